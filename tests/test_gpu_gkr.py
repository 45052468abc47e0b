"""GPU parity of the GKR kernels, called through the C ABI, against the oracle
(and, through the golden fixtures, against the reference library itself).
Field arithmetic is exact: every comparison is bit-for-bit."""
import ctypes

import numpy as np
import pytest

from fp2lib import GPU_LIB, P61, Fp2Lib, rand_fp, run_session, u64p, i32p
from golden_cases import check_all

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu_lib():
    from truepix_b200 import build
    build.build()
    lib = Fp2Lib(GPU_LIB, "native_fp2_")
    assert lib.init() == 0
    assert lib.cuda_available() == 1, "CUDA library loaded but no usable device"
    return lib


def test_gpu_matches_reference_golden(gpu_lib, golden):
    check_all(gpu_lib, golden)


def _circuit_table(rng, circuits, name, n_wires, n_copies):
    n_in = int(circuits[name + "_ninputs"][0])
    vr = np.zeros((n_wires, n_copies), np.uint64)
    vr[:min(n_in, n_wires)] = rng.integers(0, 256, size=(min(n_in, n_wires), n_copies),
                                           dtype=np.uint64)
    for idx, val in circuits[name + "_consts"]:
        if idx < n_wires:
            vr[idx] = val
    return vr.reshape(-1).copy(), np.zeros(n_wires * n_copies, np.uint64)


def _compare_sessions(gpu, oracle, gt, i0, i1, n_copies, n_wires, vre, vim, rng):
    G = gt.size
    zr, zi = rand_fp(rng, G), rand_fp(rng, G)
    br, bi = rand_fp(rng, n_copies), rand_fp(rng, n_copies)
    nr = int(np.log2(n_copies))
    chal = np.stack([rand_fp(rng, 2) for _ in range(nr)])
    a = run_session(gpu, gt, i0, i1, zr, zi, n_copies, n_wires, vre, vim, br, bi, chal)
    b = run_session(oracle, gt, i0, i1, zr, zi, n_copies, n_wires, vre, vim, br, bi, chal)
    assert np.array_equal(a[0], b[0]), "claims differ"
    assert np.array_equal(a[1], b[1]) and np.array_equal(a[2], b[2]), "final wires differ"
    assert a[3] == b[3], "final beta differs"
    assert a[4] == b[4], "n_copies sequence differs"
    assert a[0].any()


@pytest.mark.parametrize("name,n_copies", [("gray", 1024), ("inv", 256), ("mask", 512),
                                           ("Crop", 512), ("gray", 2), ("Crop", 4)])
def test_session_reference_circuits(gpu_lib, oracle_lib, circuits, name, n_copies):
    rng = np.random.default_rng(hash((name, n_copies)) & 0xFFFF)
    vre, vim = _circuit_table(rng, circuits, name, 512, n_copies)
    _compare_sessions(gpu_lib, oracle_lib, circuits[name + "_type"], circuits[name + "_in0"],
                      circuits[name + "_in1"], n_copies, 512, vre, vim, rng)


@pytest.mark.parametrize("seed,n_gates,n_wires,n_copies", [
    (1, 1, 1, 2), (2, 13, 3, 4), (3, 200, 37, 64), (4, 700, 129, 128), (5, 64, 512, 256),
    (6, 3000, 64, 32), (7, 384, 512, 2048)])
def test_session_random_circuits(gpu_lib, oracle_lib, seed, n_gates, n_wires, n_copies):
    rng = np.random.default_rng(seed)
    gt = rng.integers(-1, 14, size=n_gates).astype(np.int32)
    i0 = rng.integers(0, n_wires, size=n_gates).astype(np.int32)
    i1 = rng.integers(0, n_wires, size=n_gates).astype(np.int32)
    vre, vim = rand_fp(rng, n_wires * n_copies), rand_fp(rng, n_wires * n_copies)
    _compare_sessions(gpu_lib, oracle_lib, gt, i0, i1, n_copies, n_wires, vre, vim, rng)


@pytest.mark.parametrize("name", ["gray", "Crop"])
def test_session_1080p_full_size(gpu_lib, oracle_lib, circuits, name):
    """One 1920x1080x3 frame = 16,200 copies -> 16,384 x 512 wires (2^23)."""
    rng = np.random.default_rng(1080)
    vre, vim = _circuit_table(rng, circuits, name, 512, 16384)
    _compare_sessions(gpu_lib, oracle_lib, circuits[name + "_type"], circuits[name + "_in0"],
                      circuits[name + "_in1"], 16384, 512, vre, vim, rng)


def test_session_call_orders(gpu_lib, oracle_lib):
    """claim twice, fold twice without a claim, finish with a fold pending."""
    rng = np.random.default_rng(11)
    W, C, G = 20, 64, 50
    gt = rng.integers(0, 13, size=G).astype(np.int32)
    i0 = rng.integers(0, W, size=G).astype(np.int32)
    i1 = rng.integers(0, W, size=G).astype(np.int32)
    zr, zi = rand_fp(rng, G), rand_fp(rng, G)
    vr, vi = rand_fp(rng, W * C), rand_fp(rng, W * C)
    br, bi = rand_fp(rng, C), rand_fp(rng, C)
    outs = []
    for lib in (gpu_lib, oracle_lib):
        h = lib.early_create(gt, i0, i1, zr, zi, C, W, vr, vi, br, bi)
        assert h
        log = []
        r = np.random.default_rng(5)
        log.append(lib.early_claim(h)[1])
        log.append(lib.early_claim(h)[1])
        assert lib.early_fold(h, rand_fp(r, 2)) == 0
        assert lib.early_fold(h, rand_fp(r, 2)) == 0
        log.append(lib.early_n_copies(h))
        log.append(lib.early_claim(h)[1])
        assert lib.early_fold(h, rand_fp(r, 2)) == 0
        rc, wre, wim, beta = lib.early_finish(h, W)
        assert rc == 0
        log += [wre, wim, beta, lib.early_n_wires(h)]
        lib.early_destroy(h)
        outs.append(log)
    for x, y in zip(*outs):
        if isinstance(x, np.ndarray):
            assert np.array_equal(x, y)
        else:
            assert x == y


def test_batch_ops_vs_oracle(gpu_lib, oracle_lib):
    rng = np.random.default_rng(99)
    for n_out in (1, 3, 1000, 1 << 20):
        re, im, r = rand_fp(rng, 2 * n_out), rand_fp(rng, 2 * n_out), rand_fp(rng, 2)
        a, b = gpu_lib.fold(re, im, r), oracle_lib.fold(re, im, r)
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    for n_src, nc in ((1, 1), (7, 5), (4096, 64)):
        re, im = rand_fp(rng, n_src), rand_fp(rng, n_src)
        a, b = gpu_lib.expand(re, im, nc), oracle_lib.expand(re, im, nc)
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    for n_z in (1, 2, 3, 8, 13, 16):
        zr, zi, init = rand_fp(rng, n_z), rand_fp(rng, n_z), rand_fp(rng, 2)
        a, b = gpu_lib.compute_beta(zr, zi, init), oracle_lib.compute_beta(zr, zi, init)
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]), n_z
    for n_z in (0, 1, 2, 3, 4, 9, 15, 20):
        x = rng.integers(0, 1 << 64, size=1 << n_z, dtype=np.uint64)
        x[rng.random(x.size) < 0.2] = 0
        zr, zi = rand_fp(rng, n_z), rand_fp(rng, n_z)
        assert gpu_lib.mle_eval_base(x, zr, zi) == oracle_lib.mle_eval_base(x, zr, zi), n_z
    for (G, W, C) in ((20, 4, 2), (300, 40, 64), (1000, 100, 256)):
        gt = rng.integers(-1, 14, size=G).astype(np.int32)
        i0 = rng.integers(0, W, size=G).astype(np.int32)
        i1 = rng.integers(0, W, size=G).astype(np.int32)
        args = [gt, i0, i1, rand_fp(rng, G), rand_fp(rng, G), C, W,
                rand_fp(rng, W * C), rand_fp(rng, W * C)] + \
               [rand_fp(rng, W * C // 2) for _ in range(4)] + \
               [rand_fp(rng, C), rand_fp(rng, C)] + [rand_fp(rng, C // 2) for _ in range(4)]
        assert np.array_equal(gpu_lib.sumcheck_early(*args), oracle_lib.sumcheck_early(*args))


def test_mle_at_1080p_size(gpu_lib, oracle_lib):
    """MLE of the 2^23 copy-major input vector (config: one 1080p frame)."""
    rng = np.random.default_rng(23)
    x = rng.integers(0, 256, size=1 << 23, dtype=np.uint64)
    zr, zi = rand_fp(rng, 23), rand_fp(rng, 23)
    assert gpu_lib.mle_eval_base(x, zr, zi) == oracle_lib.mle_eval_base(x, zr, zi)


def test_error_paths(gpu_lib):
    rng = np.random.default_rng(3)
    W, C = 4, 8
    gt = np.array([0, 1], np.int32)
    i0 = np.array([0, 1], np.int32)
    i1 = np.array([2, 7], np.int32)   # 7 is outside [0, 4)
    z = rand_fp(rng, 2)
    v = rand_fp(rng, W * C)
    b = rand_fp(rng, C)
    assert not gpu_lib.early_create(gt, i0, i1, z, z, C, W, v, v, b, b)
    assert b"outside" in gpu_lib._err()
    i1[1] = 3
    assert not gpu_lib.early_create(gt, i0, i1, z, z, 6, W, v, v, b, b)   # not a power of two
    h = gpu_lib.early_create(gt, i0, i1, z, z, C, W, v, v, b, b)
    assert h
    assert gpu_lib.early_fold(h, (P61, 0)) == -1                         # non-canonical challenge
    for _ in range(3):
        assert gpu_lib.early_fold(h, (1, 2)) == 0
    assert gpu_lib.early_n_copies(h) == 1
    assert gpu_lib.early_claim(h)[0] == -1                               # nothing left to claim
    assert gpu_lib.early_fold(h, (1, 2)) == -1
    gpu_lib.early_destroy(h)
    assert gpu_lib._claim(None, u64p(np.zeros(8, np.uint64))) == -1
    # batch entry points report instead of silently falling back
    with pytest.raises(RuntimeError):
        gpu_lib.sumcheck_early(gt, i0, np.array([2, 9], np.int32), z, z, C, W, v, v,
                               v[:W * C // 2].copy(), v[:W * C // 2].copy(),
                               v[:W * C // 2].copy(), v[:W * C // 2].copy(), b, b,
                               b[:C // 2].copy(), b[:C // 2].copy(), b[:C // 2].copy(),
                               b[:C // 2].copy())


def test_device_buffer_api(gpu_lib, oracle_lib, circuits):
    """tp_early_create_dev / tp_early_claim_dev / tp_early_finish_dev on torch buffers."""
    import torch
    lib = gpu_lib.lib
    lib.tp_early_create_dev.restype = ctypes.c_void_p
    lib.tp_early_create_dev.argtypes = [ctypes.c_int] + [ctypes.c_void_p] * 5 + \
        [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
    lib.tp_early_claim_dev.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
    lib.tp_early_finish_dev.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    lib.native_fp2_early_fold.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint64]
    rng = np.random.default_rng(21)
    W, C = 512, 256
    gt, i0, i1 = (np.ascontiguousarray(circuits["gray_" + k]) for k in ("type", "in0", "in1"))
    zr, zi = rand_fp(rng, gt.size), rand_fp(rng, gt.size)
    vre, vim = _circuit_table(rng, circuits, "gray", W, C)
    br_, bi_ = rand_fp(rng, C), rand_fp(rng, C)
    packed = np.stack([vre, vim], axis=1).reshape(-1)
    dv = torch.from_numpy(packed.view(np.int64)).cuda()
    db = torch.from_numpy(np.stack([br_, bi_], axis=1).reshape(-1).view(np.int64)).cuda()
    nr = 8
    claims = torch.zeros(nr * 8, dtype=torch.int64, device="cuda")
    fin = torch.zeros(2 * (W + 1), dtype=torch.int64, device="cuda")
    chal = np.stack([rand_fp(rng, 2) for _ in range(nr)])
    stream = torch.cuda.current_stream().cuda_stream
    h = lib.tp_early_create_dev(gt.size, gt.ctypes.data, i0.ctypes.data, i1.ctypes.data,
                                zr.ctypes.data, zi.ctypes.data, C, W, dv.data_ptr(),
                                db.data_ptr(), 1, stream)
    assert h
    for k in range(nr):
        assert lib.tp_early_claim_dev(h, claims.data_ptr() + 64 * k) == 0
        assert lib.native_fp2_early_fold(h, int(chal[k][0]), int(chal[k][1])) == 0
    assert lib.tp_early_finish_dev(h, fin.data_ptr(), fin.data_ptr() + 16 * W) == 0
    torch.cuda.synchronize()
    lib.native_fp2_early_destroy(ctypes.c_void_p(h))
    want = run_session(oracle_lib, gt, i0, i1, zr, zi, C, W, vre, vim, br_, bi_, chal)
    got_claims = claims.cpu().numpy().view(np.uint64).reshape(nr, 8)
    assert np.array_equal(got_claims, want[0])
    f = fin.cpu().numpy().view(np.uint64).reshape(W + 1, 2)
    assert np.array_equal(f[:W, 0], want[1]) and np.array_equal(f[:W, 1], want[2])
    assert (int(f[W, 0]), int(f[W, 1])) == want[3]


@pytest.mark.parametrize("name,hw,mode", [
    ("gray", (1080, 1920), "pixels"), ("gray", (1080, 1920), "table"),
    ("Crop", (240, 426), "pixels"), ("Crop", (240, 426), "table"),
    ("inv", (360, 640), "pixels"), ("mask", (8, 8), "pixels"), ("gray", (4, 8), "pixels"),
    ("Crop", (2, 64), "pixels"), ("gray", (720, 1280), "pixels"),
    ("gray", (2160, 3840), "pixels")])    # 4K: 64,800 copies -> 2^25 input wires, the largest serving frame
def test_frame_prover_vs_oracle(oracle_lib, circuits, name, hw, mode):
    """The device-resident frame path (bytes -> beta -> rounds -> MLE) in both modes:
    straight from the bytes, and through the materialised table."""
    import torch
    from truepix_b200.frame import FrameLayout, GkrInputLayerProver, pack_fp2
    rng = np.random.default_rng(4242)
    const = {"gray": (384, 128), "Crop": (385, 128), "inv": (384, 255), "mask": (-1, 0)}[name]
    cs = 385 if name == "Crop" else 384
    layout = FrameLayout.for_frame(hw[0], hw[1], copy_size=cs, const_idx=const[0],
                                   const_val=const[1])
    gt, i0, i1 = (circuits[name + "_" + k] for k in ("type", "in0", "in1"))
    C, W, nb = layout.padded_copies, layout.n_wires, layout.n_copy_bits
    pix = rng.integers(0, 256, size=layout.copies * cs, dtype=np.uint8)
    z1 = np.stack([rand_fp(rng, gt.size), rand_fp(rng, gt.size)])
    z2 = np.stack([rand_fp(rng, nb), rand_fp(rng, nb)], axis=1)
    point = np.stack([rand_fp(rng, nb + 9), rand_fp(rng, nb + 9)], axis=1)
    chal = np.stack([rand_fp(rng, nb), rand_fp(rng, nb)], axis=1)
    dev = torch.device("cuda", 0)
    prover = GkrInputLayerProver(layout, gt, i0, i1, mode=mode)
    prover.prove(torch.from_numpy(pix).to(dev), z1,
                 torch.from_numpy(pack_fp2(z2[:, 0], z2[:, 1])).to(dev),
                 torch.from_numpy(pack_fp2(point[:, 0], point[:, 1])).to(dev), chal)
    torch.cuda.synchronize()
    claims, wires, beta, mle = prover.results()
    # oracle on the same inputs
    vals = np.zeros((C, W), np.uint64)
    vals[:layout.copies, :cs] = pix.reshape(layout.copies, cs)
    if const[0] >= 0:
        vals[:layout.copies, const[0]] = const[1]
    table = np.ascontiguousarray(vals.T).reshape(-1)
    bre, bim = oracle_lib.compute_beta(np.ascontiguousarray(z2[:, 0]),
                                       np.ascontiguousarray(z2[:, 1]), (1, 0))
    oc, wre, wim, ob, _ = run_session(oracle_lib, gt, i0, i1, z1[0].copy(), z1[1].copy(), C, W,
                                      table, np.zeros_like(table), bre, bim, chal)
    om = oracle_lib.mle_eval_base(vals.reshape(-1).copy(), np.ascontiguousarray(point[:, 0]),
                                  np.ascontiguousarray(point[:, 1]))
    assert np.array_equal(claims, oc)
    assert np.array_equal(wires[:, 0], wre) and np.array_equal(wires[:, 1], wim)
    assert beta == ob and mle == om


def _oracle_frame(oracle_lib, gt, i0, i1, layout, pix, z1, z2, point, chal):
    C, W, cs = layout.padded_copies, layout.n_wires, layout.copy_size
    vals = np.zeros((C, W), np.uint64)
    vals[:layout.copies, :cs] = pix.reshape(layout.copies, cs)
    if layout.const_idx >= 0:
        vals[:layout.copies, layout.const_idx] = layout.const_val
    table = np.ascontiguousarray(vals.T).reshape(-1)
    bre, bim = oracle_lib.compute_beta(np.ascontiguousarray(z2[:, 0]),
                                       np.ascontiguousarray(z2[:, 1]), (1, 0))
    oc, wre, wim, ob, _ = run_session(oracle_lib, gt, i0, i1, z1[0].copy(), z1[1].copy(), C, W,
                                      table, np.zeros_like(table), bre, bim, chal)
    om = oracle_lib.mle_eval_base(vals.reshape(-1).copy(), np.ascontiguousarray(point[:, 0]),
                                  np.ascontiguousarray(point[:, 1]))
    return oc, wre, wim, ob, om


@pytest.mark.parametrize("name", ["gray", "Crop"])
def test_batch_uneven_frames_vs_oracle(oracle_lib, circuits, name):
    """A batch of frames of uneven size (1 to 16,200 copies): every frame's claims,
    wires, beta and MLE equal the oracle's for that frame alone."""
    import torch
    from truepix_b200.frame import BatchFrameProver, FrameLayout, pack_fp2
    rng = np.random.default_rng(77)
    cs = 385 if name == "Crop" else 384
    const = (385, 128) if name == "Crop" else (384, 128)
    copies = [1, 2, 5, 100, 1000, 3000, 16200] if name == "gray" else [1, 7, 64, 700]
    layouts = [FrameLayout(copies=c, copy_size=cs, const_idx=const[0], const_val=const[1])
               for c in copies]
    gt, i0, i1 = (circuits[name + "_" + k] for k in ("type", "in0", "in1"))
    dev = torch.device("cuda", 0)
    prover = BatchFrameProver(layouts, gt, i0, i1)
    R, B = prover.max_rounds, len(layouts)
    for rep in range(2):   # the same batch object serves consecutive batches
        pix, z1s, z2s, pts = [], [], [], []
        for L in layouts:
            pix.append(rng.integers(0, 256, size=L.copies * cs, dtype=np.uint8))
            z1s.append(np.stack([rand_fp(rng, gt.size), rand_fp(rng, gt.size)]))
            nb = L.n_copy_bits
            z2s.append(np.stack([rand_fp(rng, nb), rand_fp(rng, nb)], axis=1))
            pts.append(np.stack([rand_fp(rng, nb + 9), rand_fp(rng, nb + 9)], axis=1))
        chal = rng.integers(0, P61, size=(R, B, 2), dtype=np.uint64)
        z2d, ptd = {}, {}
        for C, fs in prover.groups.items():
            z2d[C] = torch.from_numpy(np.concatenate(
                [pack_fp2(z2s[f][:, 0], z2s[f][:, 1]) for f in fs])).to(dev)
            ptd[C] = torch.from_numpy(np.concatenate(
                [pack_fp2(pts[f][:, 0], pts[f][:, 1]) for f in fs])).to(dev)
        prover.prove([torch.from_numpy(p).to(dev) for p in pix], z1s, z2d, ptd, chal)
        torch.cuda.synchronize()
        _check_batch(oracle_lib, gt, i0, i1, layouts, prover, pix, z1s, z2s, pts, chal)


def _check_batch(oracle_lib, gt, i0, i1, layouts, prover, pix, z1s, z2s, pts, chal):
    for f, L in enumerate(layouts):
        claims, wires, beta, mle = prover.results(f)
        nb = L.n_copy_bits
        oc, wre, wim, ob, om = _oracle_frame(oracle_lib, gt, i0, i1, L, pix[f], z1s[f], z2s[f],
                                             pts[f], chal[:nb, f])
        assert np.array_equal(claims, oc), f"frame {f} ({L.copies} copies): claims"
        assert np.array_equal(wires[:, 0], wre) and np.array_equal(wires[:, 1], wim), f"frame {f}"
        assert beta == ob and mle == om, f"frame {f}"
