"""Fp2 NTT / IFFT and the Reed-Solomon commit on the GPU (include/orion_gpu.h)
against the reference's outputs (tests/golden/orion_golden.npz) and the oracle,
bit for bit; full-size transforms through round trips and linearity."""
import ctypes
import os

import numpy as np
import pytest

from orionlib import P61, ROOT, OrionOracle, digest, elements

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib():
    from truepix_b200 import native
    return native.gkr()


@pytest.fixture(scope="module")
def orc():
    return OrionOracle()


@pytest.fixture(scope="module")
def og():
    return np.load(os.path.join(ROOT, "tests", "golden", "orion_golden.npz"))


def vp(a):
    return ctypes.c_void_p(a.ctypes.data)


def fft(lib, coef, order):
    out = np.zeros(2 * order, np.uint64)
    assert lib.tp_fft(vp(coef), coef.size // 2, order, vp(out)) == 0, lib.tp_last_error()
    return out


def ifft(lib, evals, coef_len):
    out = np.zeros(2 * coef_len, np.uint64)
    assert lib.tp_ifft(vp(evals), coef_len, evals.size // 2, vp(out)) == 0, lib.tp_last_error()
    return out


def test_fft_ifft_match_reference(lib, og):
    for k in og.files:
        if not k.startswith("fft_"):
            continue
        m, o = (int(v) for v in k.split("_")[1:])
        r = fft(lib, elements(200 + m + o, m), o)
        np.testing.assert_array_equal(r[:16], og["ffthead_%d_%d" % (m, o)][:r[:16].size])
        assert digest(r) == og[k].tobytes(), (m, o)
        ri = ifft(lib, elements(300 + m + o, o), m)
        assert digest(ri) == og["ifft_%d_%d" % (m, o)].tobytes(), (m, o)


@pytest.mark.parametrize("m,o", [(1 << 10, 1 << 11), (1 << 11, 1 << 11), (1 << 7, 1 << 13), (1 << 15, 1 << 20),
                                 (1 << 21, 1 << 21), (1 << 16, 1 << 22)])
def test_fft_ifft_match_oracle(lib, orc, m, o):
    coef = elements(m + 3 * o, m)
    np.testing.assert_array_equal(fft(lib, coef, o), orc.fft(coef, o))
    ev = elements(m + 5 * o, o)
    np.testing.assert_array_equal(ifft(lib, ev, m), orc.ifft(ev, m))


def test_edge_values(lib, orc):
    for kind in ("zero", "max", "small"):
        a = elements(4, 1 << 12, kind)
        np.testing.assert_array_equal(fft(lib, a, 1 << 14), orc.fft(a, 1 << 14))


def test_size_2_24_round_trip_and_linearity(lib):
    """2^24 (the largest transform of the microbenchmark): ifft(fft(a)) == a, and
    fft(a + b) == fft(a) + fft(b), on the device."""
    import torch
    n = 1 << 24
    dev = torch.device("cuda", 0)
    a = torch.from_numpy(elements(31, n).view(np.int64)).to(dev)
    b = torch.from_numpy(elements(32, n).view(np.int64)).to(dev)
    s = torch.cuda.current_stream().cuda_stream
    fa, fb, fab, back = (torch.empty_like(a) for _ in range(4))
    for x, y in ((a, fa), (b, fb)):
        assert lib.tp_fft_dev(x.data_ptr(), n, n, y.data_ptr(), 1, 0, 0, s) == 0, lib.tp_last_error()
    assert lib.tp_ifft_dev(fa.data_ptr(), n, n, back.data_ptr(), 1, 0, 0, s) == 0
    torch.cuda.synchronize()
    an, bn = a.cpu().numpy().view(np.uint64), b.cpu().numpy().view(np.uint64)
    np.testing.assert_array_equal(back.cpu().numpy().view(np.uint64), an)
    abn = (an + bn) % np.uint64(P61)
    dab = torch.from_numpy(abn.view(np.int64)).to(dev)
    assert lib.tp_fft_dev(dab.data_ptr(), n, n, fab.data_ptr(), 1, 0, 0, s) == 0
    torch.cuda.synchronize()
    got = fab.cpu().numpy().view(np.uint64)
    want = (fa.cpu().numpy().view(np.uint64) + fb.cpu().numpy().view(np.uint64)) % np.uint64(P61)
    np.testing.assert_array_equal(got, want)
    assert int(got.max()) < P61


def test_size_2_28_round_trip_and_linearity_on_device(lib):
    """The largest supported transform (2^28 points; the reference asserts beyond
    2^27): ifft(fft(a)) == a and fft(a + b) == fft(a) + fft(b), inputs drawn and
    results compared on the device."""
    import torch
    n = 1 << 28
    dev = torch.device("cuda", 0)
    g = torch.Generator(device=dev)
    g.manual_seed(28)
    p = (1 << 61) - 1
    a = torch.randint(0, p, (2 * n,), dtype=torch.int64, device=dev, generator=g)
    b = torch.randint(0, p, (2 * n,), dtype=torch.int64, device=dev, generator=g)
    s = torch.cuda.current_stream().cuda_stream
    fa, fb = torch.empty_like(a), torch.empty_like(a)
    assert lib.tp_fft_dev(a.data_ptr(), n, n, fa.data_ptr(), 1, 0, 0, s) == 0, lib.tp_last_error()
    assert lib.tp_fft_dev(b.data_ptr(), n, n, fb.data_ptr(), 1, 0, 0, s) == 0, lib.tp_last_error()
    back = torch.empty_like(a)
    assert lib.tp_ifft_dev(fa.data_ptr(), n, n, back.data_ptr(), 1, 0, 0, s) == 0, lib.tp_last_error()
    torch.cuda.synchronize()
    assert torch.equal(back, a)
    del back
    ab = a + b
    ab = torch.where(ab >= p, ab - p, ab)
    fab = torch.empty_like(a)
    assert lib.tp_fft_dev(ab.data_ptr(), n, n, fab.data_ptr(), 1, 0, 0, s) == 0, lib.tp_last_error()
    want = fa + fb
    want = torch.where(want >= p, want - p, want)
    torch.cuda.synchronize()
    assert torch.equal(fab, want)
    assert int(fab.max()) < p and int(fab.min()) >= 0


def test_batched_device_transforms(lib, orc):
    import torch
    m, o, batch = 1 << 8, 1 << 13, 64
    src = elements(41, m * batch)
    dev = torch.device("cuda", 0)
    d_in = torch.from_numpy(src.view(np.int64)).to(dev)
    d_out = torch.empty(2 * o * batch, dtype=torch.int64, device=dev)
    s = torch.cuda.current_stream().cuda_stream
    assert lib.tp_fft_dev(d_in.data_ptr(), m, o, d_out.data_ptr(), batch, m, o, s) == 0
    torch.cuda.synchronize()
    out = d_out.cpu().numpy().view(np.uint64).reshape(batch, 2 * o)
    for b in (0, 1, 37, 63):
        np.testing.assert_array_equal(out[b], orc.fft(np.ascontiguousarray(src.reshape(batch, 2 * m)[b]), o))


def test_rs_commit_matches_reference(lib, og):
    for k in og.files:
        if not k.startswith("rs_"):
            continue
        lg = int(k.split("_")[1])
        src = elements(400 + lg, 1 << lg)
        cw = np.zeros(2 << (lg + 5), np.uint64)
        tree = np.zeros((1 << (lg - 1), 32), np.uint8)
        assert lib.tp_rs_commit(vp(src), lg, vp(cw), vp(tree)) == 0, lib.tp_last_error()
        assert digest(cw) == og["rscw_%d" % lg].tobytes(), lg
        assert tree[1].tobytes() == og[k].tobytes(), lg
        assert not tree[0].any()


def test_rs_codeword_contains_the_input_at_2_22(lib):
    """Rate 2^-5: slice i's evaluations on every 32nd point of its 2^(L-1)-point
    domain are the slice's own inputs (the original domain is a subgroup)."""
    import torch
    lg = 22
    n, real_cnt, slice_len = 1 << lg, 1 << (lg - 6), 1 << (lg - 1)
    dev = torch.device("cuda", 0)
    src = torch.from_numpy(elements(9, n).view(np.int64)).to(dev)
    cw = torch.empty(2 << (lg + 5), dtype=torch.int64, device=dev)
    tree = torch.empty(32 << (lg - 1), dtype=torch.uint8, device=dev)
    s = torch.cuda.current_stream().cuda_stream
    assert lib.tp_rs_commit_dev(src.data_ptr(), lg, cw.data_ptr(), tree.data_ptr(), s) == 0
    torch.cuda.synchronize()
    sub = cw.view(64, slice_len, 2)[:, ::32, :]
    assert torch.equal(sub, src.view(64, real_cnt, 2))
    assert bool(((cw >= 0) & (cw < P61)).all())


def test_transform_argument_errors(lib):
    a = elements(1, 16)
    out = np.zeros(64, np.uint64)
    assert lib.tp_fft(vp(a), 3, 16, vp(out)) == -1
    assert lib.tp_fft(vp(a), 32, 16, vp(out)) == -1
    bad = a.copy()
    bad[3] = P61
    assert lib.tp_fft(vp(bad), 8, 16, vp(out)) == -1
    assert b"canonical" in lib.tp_last_error()
    assert lib.tp_rs_commit(vp(a), 5, None, vp(out)) == -1


def test_autotuned_splits_give_the_same_transform(lib, orc):
    """The autotuner only changes how the passes are cut; outputs stay bit-identical."""
    import ctypes
    for lg, m in ((14, 1 << 14), (21, 1 << 17)):
        digits = (ctypes.c_int * 3)()
        ms = ctypes.c_float()
        p = lib.tp_ntt_autotune(lg, 1, digits, ctypes.byref(ms))
        assert p >= 1, lib.tp_last_error()
        assert sum(digits[:p]) == lg and all(3 <= d <= 10 for d in digits[:p]) and ms.value > 0
        coef = elements(lg, m)
        np.testing.assert_array_equal(fft(lib, coef, 1 << lg), orc.fft(coef, 1 << lg))
        ev = elements(lg + 1, 1 << lg)
        np.testing.assert_array_equal(ifft(lib, ev, 1 << lg), orc.ifft(ev, 1 << lg))
    assert lib.tp_ntt_autotune(40, 1, None, None) == -1


def _fri_dev(lib, w, lm, r):
    import torch
    dev = torch.device("cuda", 0)
    d_w = torch.from_numpy(w.view(np.int64)).to(dev)
    d_next = torch.empty(w.size // 2, dtype=torch.int64, device=dev)
    d_tree = torch.empty(32 * (1 << (lm - 1)), dtype=torch.uint8, device=dev)
    rc = lib.tp_fri_commit_step_dev(d_w.data_ptr(), lm, int(r[1]), int(r[0]), d_next.data_ptr(),
                                    d_tree.data_ptr(), torch.cuda.current_stream().cuda_stream)
    assert rc == 0, lib.tp_last_error()
    torch.cuda.synchronize()
    return d_next.cpu().numpy().view(np.uint64), d_tree.cpu().numpy().reshape(-1, 32)


def test_fri_step_matches_reference(lib, og):
    for k in og.files:
        if not k.startswith("fricase_"):
            continue
        lm, seed = (int(v) for v in og[k])
        nxt, tree = _fri_dev(lib, elements(seed, (1 << lm) * 64), lm, elements(seed + 1, 1))
        assert digest(nxt) == og["frinext_%d" % lm].tobytes(), lm
        assert tree[1].tobytes() == og["friroot_%d" % lm].tobytes(), lm


def test_fri_steps_chained_match_oracle(lib, orc):
    """Consecutive steps down to one leaf, each fed the previous step's output."""
    w = elements(61, (1 << 12) * 64)
    for lm in range(12, 1, -1):
        r = elements(700 + lm, 1)
        want, wroot = orc.fri_step(w, lm, r)
        got, tree = _fri_dev(lib, w, lm, r)
        np.testing.assert_array_equal(got, want)
        assert tree[1].tobytes() == wroot
        w = want
    assert lib.tp_fri_commit_step_dev(None, 1, 0, 0, None, None, None) == -1
