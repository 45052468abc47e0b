"""tp_mle_eval_base_noalloc: the MLE entry point for callers that cannot
allocate device memory (their GPU memory is owned by another allocator, or a
time-critical loop cannot afford cudaMalloc/cudaFree). It uses a fixed scratch
array compiled into the library; this file checks it against the allocating
entry point tp_mle_eval_base_dev through the C ABI, on consecutive calls that
share that scratch. Collected last on purpose."""
import ctypes

import numpy as np
import pytest

from fp2lib import P61, rand_fp

pytestmark = pytest.mark.gpu


def _packed(zr, zi):
    return np.stack([zr, zi], axis=1).reshape(-1).view(np.int64)


def test_noalloc_mle_equals_allocating_entry_point():
    import torch
    from truepix_b200 import native
    lib = native.gkr()
    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(2026)
    # two calls in a row on the shared scratch, then a smaller and a larger size
    for n_z in (20, 20, 3, 23):
        x = rng.integers(0, 1 << 64, size=1 << n_z, dtype=np.uint64)   # incl. values >= p
        x[rng.random(x.size) < 0.1] = 0
        zr, zi = rand_fp(rng, n_z), rand_fp(rng, n_z)
        dx = torch.from_numpy(x.view(np.int64)).to(dev)
        dz = torch.from_numpy(_packed(zr, zi)).to(dev)
        want = torch.zeros(2, dtype=torch.int64, device=dev)
        got = torch.full((2,), -1, dtype=torch.int64, device=dev)
        s = torch.cuda.current_stream().cuda_stream
        assert lib.tp_mle_eval_base_dev(dx.data_ptr(), dz.data_ptr(), n_z, want.data_ptr(), s) == 0
        rc = lib.tp_mle_eval_base_noalloc(dx.data_ptr(), dz.data_ptr(), n_z, got.data_ptr(), s)
        assert rc == 0, lib.tp_last_error()
        torch.cuda.synchronize()
        a = want.cpu().numpy().view(np.uint64)
        b = got.cpu().numpy().view(np.uint64)
        assert int(a[0]) < P61 and int(a[1]) < P61
        assert np.array_equal(a, b), (n_z, a, b)   # exact field arithmetic: bit-for-bit


def test_noalloc_mle_rejects_sizes_beyond_its_scratch():
    import torch
    from truepix_b200 import native
    lib = native.gkr()
    buf = torch.zeros(64, dtype=torch.int64, device="cuda")
    p = buf.data_ptr()
    assert lib.tp_mle_eval_base_noalloc(p, p, 27, p, None) == -1
    assert b"2^26" in lib.tp_last_error()
    assert lib.tp_mle_eval_base_noalloc(p, p, 0, p, None) == -1
