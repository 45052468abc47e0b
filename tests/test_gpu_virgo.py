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


# ---- layer inits (tp_virgo_layer_create, tp_virgo_phase{1,2}_init_dev) ----

def _vp(a):
    import ctypes
    return ctypes.c_void_p(a.ctypes.data)


def layer_of(lib, L):
    h = lib.tp_virgo_layer_create(L["length_g"], L["length_u"], _vp(L["ty"]), _vp(L["u"]), _vp(L["v"]),
                                  _vp(L["comb_ptr"]), _vp(L["comb_src"]), _vp(L["comb_w"]))
    assert h, lib.tp_last_error()
    return h


def device_init(lib, phase, L, h=None, d_vma0=None):
    """the three tables after the init of `phase` on the device (numpy words)"""
    import torch
    dev = torch.device("cuda", 0)
    own = h is None
    h = h or layer_of(lib, L)
    U = 1 << L["length_u"]
    vals = torch.from_numpy(L["values"].view(np.int64)).to(dev)
    outs = [torch.full((4 * U,), -1, dtype=torch.int64, device=dev) for _ in range(3)]
    s = torch.cuda.current_stream().cuda_stream
    try:
        if phase == 1:
            rc = lib.tp_virgo_phase1_init_dev(h, vals.data_ptr(), _vp(L["r0"]), _vp(L["r1"]), _vp(L["alpha"]),
                                              _vp(L["beta"]), *[o.data_ptr() for o in outs], s)
        else:
            if d_vma0 is None:
                d_vma0 = torch.from_numpy(L["vma0"].view(np.int64)).to(dev)
            rc = lib.tp_virgo_phase2_init_dev(h, vals.data_ptr(), _vp(L["r0"]), _vp(L["r1"]), _vp(L["alpha"]),
                                              _vp(L["beta"]), d_vma0.data_ptr(), _vp(L["prev_r"]), _vp(L["r_u"]),
                                              *[o.data_ptr() for o in outs], s)
        assert rc == 0, lib.tp_last_error()
        torch.cuda.synchronize()
    finally:
        if own:
            lib.tp_virgo_layer_destroy(h)
    return [o.cpu().numpy().view(np.uint64) for o in outs]


def test_layer_inits_match_reference(lib):
    """Every gate type, both phases, against the reference's zk_prover tables
    (tests/golden/virgo_init_golden.npz)."""
    from orionlib import virgo_layer
    g = np.load(os.path.join(ROOT, "tests", "golden", "virgo_init_golden.npz"))
    for k in g.files:
        if not k.startswith("vinitcase_"):
            continue
        phase, seed, lg, lu = (int(x) for x in g[k])
        outs = device_init(lib, phase, virgo_layer(seed, lg, lu))
        assert b"".join(digest(o) for o in outs) == g["vinit_" + k[len("vinitcase_"):]].tobytes(), k


@pytest.mark.parametrize("lg,lu,types", [(20, 18, None), (16, 20, None), (18, 18, (0, 1, 8, 14)), (14, 14, (5, 12))])
def test_layer_inits_match_oracle_at_larger_sizes(lib, lg, lu, types):
    from orionlib import VIRGO_TYPES, virgo_layer
    orc = OrionOracle()
    L = virgo_layer(lg * 100 + lu, lg, lu, types or VIRGO_TYPES)
    for phase in (1, 2):
        got = device_init(lib, phase, L)
        want = orc.virgo_init(phase, L)
        for a, b in zip(got, want):
            np.testing.assert_array_equal(a, b)


def test_layer_sumcheck_end_to_end_matches_oracle(lib):
    """init -> length_u rounds of phase 1 -> phase-2 init from the one-entry
    V_mult_add the rounds leave -> length_u rounds of phase 2: every round
    polynomial and the final tables against the oracle's same chain."""
    import torch
    from orionlib import virgo_layer
    orc = OrionOracle()
    lg, lu = 12, 10
    L = virgo_layer(4242, lg, lu)
    h = layer_of(lib, L)
    try:
        tabs = device_init(lib, 1, L, h)
        otabs = list(orc.virgo_init(1, L))
        assert all(np.array_equal(a, b) for a, b in zip(tabs, otabs))
        rands = [elements(500 + k, 1) for k in range(2 * lu + 1)]
        for phase in (1, 2):
            if phase == 2:
                vma0 = tabs[0][:4].copy()
                L2 = dict(L, vma0=vma0, prev_r=rands[lu])
                d_vma0 = torch.from_numpy(vma0.view(np.int64)).to("cuda")
                tabs = device_init(lib, 2, L2, h, d_vma0)
                otabs = list(orc.virgo_init(2, L2))
                assert all(np.array_equal(a, b) for a, b in zip(tabs, otabs))
            for rnd in range(lu):
                r = rands[lu * (phase - 1) + rnd] if rnd else rands[0]
                bit = 0 if rnd == 0 else 1
                got, gret = run(lib, *tabs, r, bit)
                want, wret = orc.virgo_update(*otabs, r, bit)
                np.testing.assert_array_equal(gret, wret)
                tabs, otabs = got, want
    finally:
        lib.tp_virgo_layer_destroy(h)


def test_layer_create_rejects_gates_outside_the_layer(lib):
    from orionlib import virgo_layer
    L = virgo_layer(9, 6, 6, types=(0, 4))
    L["u"][3] = 1 << 6
    L["ty"][3] = 0
    assert not lib.tp_virgo_layer_create(6, 6, _vp(L["ty"]), _vp(L["u"]), _vp(L["v"]), None, None, None)
    assert b"outside the layer" in lib.tp_last_error()
