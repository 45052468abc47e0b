import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def oracle_lib():
    """The C restatement of the reference CPU library (built on demand)."""
    from fp2lib import Fp2Lib, ORACLE_LIB
    if not os.path.exists(ORACLE_LIB):
        subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "all"])
    return Fp2Lib(ORACLE_LIB, "oracle_fp2_")


@pytest.fixture(scope="session")
def golden():
    import numpy as np
    return np.load(os.path.join(ROOT, "tests", "golden", "native_fp2_golden.npz"))


@pytest.fixture(scope="session")
def circuits():
    import numpy as np
    return np.load(os.path.join(ROOT, "tests", "golden", "circuits.npz"))
