"""The reference's own CUDA library (TruePix-main/native_fp2/native_fp2.cu,
built for sm_100a by `make -C oracle ref` into oracle/_ref) run beside ours on
the same inputs through the same 14-symbol C ABI: every output bit-identical.
The reference library takes its GPU path at these sizes (its host fallback is
only for tiny jobs or when CUDA is absent; native_fp2.cu:36-40)."""
import os

import numpy as np
import pytest

from fp2lib import GPU_LIB, P61, REF_GPU_LIB, Fp2Lib, rand_fp, run_session

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not os.path.exists(REF_GPU_LIB), reason="reference GPU library not built")]

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def libs():
    ours, ref = Fp2Lib(GPU_LIB), Fp2Lib(REF_GPU_LIB)
    ours.init()
    ref.init()
    assert ours.cuda_available() == 1 and ref.cuda_available() == 1
    return ours, ref


def circuit(name="gray"):
    c = np.load(os.path.join(ROOT, "tests", "golden", "circuits.npz"))
    return (np.ascontiguousarray(c[name + "_type"], np.int32), np.ascontiguousarray(c[name + "_in0"], np.int32),
            np.ascontiguousarray(c[name + "_in1"], np.int32))


def frame_table(rng, C, W=512, cs=384, const=(384, 128)):
    v = np.zeros((W, C), np.uint64)
    v[:cs] = rng.integers(0, 256, size=(cs, C), dtype=np.uint64)
    if const:
        v[const[0]] = const[1]
    return v.reshape(-1).copy()


@pytest.mark.parametrize("name,C", [("gray", 256), ("inv", 2048), ("mask", 1024), ("gray", 16384)])
def test_early_sessions_match_the_reference_gpu_library(libs, name, C):
    ours, ref = libs
    rng = np.random.default_rng(C + len(name))
    gt, i0, i1 = circuit(name)
    W = 512
    vr = frame_table(rng, C, const=None if name == "mask" else (384, 255 if name == "inv" else 128))
    vi = np.zeros_like(vr)
    zr, zi = rand_fp(rng, gt.size), rand_fp(rng, gt.size)
    br, bi = rand_fp(rng, C), rand_fp(rng, C)
    chal = np.stack([rand_fp(rng, 2) for _ in range(int(np.log2(C)))])
    a = run_session(ours, gt, i0, i1, zr, zi, C, W, vr, vi, br, bi, chal)
    b = run_session(ref, gt, i0, i1, zr, zi, C, W, vr, vi, br, bi, chal)
    assert np.array_equal(a[0], b[0])
    assert np.array_equal(a[1], b[1]) and np.array_equal(a[2], b[2]) and a[3] == b[3]


def test_batch_entry_points_match_the_reference_gpu_library(libs):
    ours, ref = libs
    rng = np.random.default_rng(11)
    re, im = rand_fp(rng, 1 << 16), rand_fp(rng, 1 << 16)
    r = rand_fp(rng, 2)
    for x, y in zip(ours.fold(re, im, r), ref.fold(re, im, r)):
        assert np.array_equal(x, y)
    for x, y in zip(ours.expand(re[:512], im[:512], 8), ref.expand(re[:512], im[:512], 8)):
        assert np.array_equal(x, y)
    zr, zi = rand_fp(rng, 14), rand_fp(rng, 14)
    for x, y in zip(ours.compute_beta(zr, zi, (1, 0)), ref.compute_beta(zr, zi, (1, 0))):
        assert np.array_equal(x, y)
    inputs = rng.integers(0, 256, size=1 << 20, dtype=np.uint64)
    zr, zi = rand_fp(rng, 20), rand_fp(rng, 20)
    assert ours.mle_eval_base(inputs, zr, zi) == ref.mle_eval_base(inputs, zr, zi)
    # the explicit-table claim (sumcheck_early) at 256 copies
    gt, i0, i1 = circuit("inv")
    C, W = 256, 512
    v = frame_table(rng, C, const=(384, 255))
    vi = np.zeros_like(v)
    half = C // 2
    v2 = v.reshape(W, C)
    f0 = ((2 * v2[:, 0::2] + 2 * P61 - v2[:, 1::2]) % P61).reshape(-1).astype(np.uint64)
    f1 = ((2 * v2[:, 1::2] + 2 * P61 - v2[:, 0::2]) % P61).reshape(-1).astype(np.uint64)
    zr, zi = rand_fp(rng, gt.size), rand_fp(rng, gt.size)
    br, bi = rand_fp(rng, C), rand_fp(rng, C)
    bf0, bf1 = rand_fp(rng, half), rand_fp(rng, half)
    z = np.zeros(W * half, np.uint64)
    args = (gt, i0, i1, zr, zi, C, W, v, vi, f0, z, f1, z, br, bi, bf0, z[:half], bf1, z[:half])
    assert np.array_equal(ours.sumcheck_early(*args), ref.sumcheck_early(*args))
