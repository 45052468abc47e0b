"""Virgo sumcheck round on the GPU (tp_virgo_sumcheck_update_dev) against the
reference's zk_prover::sumcheck_phase{1,2}_update (tests/golden/orion_golden.npz)
and the oracle, bit for bit."""
import os

import numpy as np
import pytest

from orionlib import P61, ROOT, OrionOracle, digest, elements, virgo_inputs

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib():
    from truepix_b200 import native
    return native.gkr()


def run(lib, vma, addv, ams, r, bit):
    import torch
    dev = torch.device("cuda", 0)
    n = vma.size // 4
    t = [torch.from_numpy(a.view(np.int64)).to(dev) for a in (vma, addv, ams)]
    outs = [torch.empty(2 * n, dtype=torch.int64, device=dev) for _ in range(3)]
    ret = torch.empty(6, dtype=torch.int64, device=dev)
    s = torch.cuda.current_stream().cuda_stream
    rc = lib.tp_virgo_sumcheck_update_dev(t[0].data_ptr(), t[1].data_ptr(), t[2].data_ptr(), n,
                                          int(r[1]), int(r[0]), bit, outs[0].data_ptr(),
                                          outs[1].data_ptr(), outs[2].data_ptr(), ret.data_ptr(), s)
    assert rc == 0, lib.tp_last_error()
    torch.cuda.synchronize()
    return [o.cpu().numpy().view(np.uint64) for o in outs], ret.cpu().numpy().view(np.uint64)


def test_update_matches_reference(lib):
    og = np.load(os.path.join(ROOT, "tests", "golden", "orion_golden.npz"))
    for k in og.files:
        if not k.startswith("virgocase_"):
            continue
        phase, n, bit, seed = (int(v) for v in og[k])
        key = k[len("virgocase_"):]
        outs, ret = run(lib, *virgo_inputs(n, seed), bit)
        assert b"".join(digest(o) for o in outs) == og["virgotables_" + key].tobytes(), key
        np.testing.assert_array_equal(ret, og["virgoret_" + key])


def test_update_rounds_match_oracle(lib):
    """Several rounds in a row (the tables shrink to one entry), both bits, edge values."""
    orc = OrionOracle()
    n = 1 << 12
    vma, addv, ams, r = virgo_inputs(n, 77)
    vma[:8] = P61 - 1
    ams[8:16] = 0
    for rnd in range(12):
        bit = 0 if rnd == 0 else 1
        r = elements(1000 + rnd, 1)
        want, wret = orc.virgo_update(vma, addv, ams, r, bit)
        got, gret = run(lib, vma, addv, ams, r, bit)
        for g, w in zip(got, want):
            np.testing.assert_array_equal(g, w)
        np.testing.assert_array_equal(gret, wret)
        vma, addv, ams = want


def test_update_rejects_odd_sizes(lib):
    import torch
    buf = torch.zeros(64, dtype=torch.int64, device="cuda")
    p = buf.data_ptr()
    assert lib.tp_virgo_sumcheck_update_dev(p, p, p, 3, 0, 0, 1, p, p, p, p, None) == -1
    assert lib.tp_virgo_sumcheck_update_dev(p, p, p, 4, P61, 0, 1, p, p, p, p, None) == -1
