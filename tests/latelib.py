"""The late-round golden cases (tests/golden/late_golden.npz) and helpers to
feed them to the oracle (oracle/gkr_late_oracle.py) and to the device."""
from __future__ import annotations

import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import gkr_late_oracle as oracle  # noqa: E402


def pairs(a):
    return [(int(x), int(y)) for x, y in np.asarray(a).reshape(-1, 2)]


def golden_cases():
    g = np.load(os.path.join(ROOT, "tests", "golden", "late_golden.npz"))
    names = sorted(k[:-6] for k in g.files if k.endswith("_shape"))
    for n in names:
        n_in_bits, n_copies = json.loads(g[n + "_shape"].tobytes().decode())
        d = {k[len(n) + 1:]: g[k] for k in g.files if k.startswith(n + "_")}
        d.update(name=n, n_in_bits=n_in_bits, n_copies=n_copies)
        d["n_copy_bits"] = (n_copies - 1).bit_length()
        yield d
