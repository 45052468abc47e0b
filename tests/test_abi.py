"""The C-ABI library loads on a host without a GPU and exports every symbol
that include/*.h declares; host-only logic is checked here, compute on the GPU."""
import ctypes
import glob
import os
import re
import subprocess

import numpy as np
import pytest

from fp2lib import GPU_LIB, P61, rand_fp, u64p, i32p

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared(header):
    text = open(header).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return set(re.findall(r"\b((?:native_fp2|tp|orion|ntt|merkle)_\w+)\s*\(", text))


def _libs():
    from truepix_b200 import build
    build.build()
    return {os.path.basename(p): p for p in glob.glob(os.path.join(build.LIBDIR, "*.so"))}


def test_every_declared_symbol_is_exported():
    libs = _libs()
    exported = set()
    for path in libs.values():
        out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True,
                             text=True, check=True).stdout
        exported |= {l.split()[-1] for l in out.splitlines() if " T " in l}
    headers = glob.glob(os.path.join(ROOT, "include", "*.h"))
    assert headers
    for h in headers:
        missing = _declared(h) - exported
        assert not missing, f"{os.path.basename(h)} declares unexported {sorted(missing)}"


def test_reference_symbol_set_present():
    names = ["init", "cuda_available", "fold", "expand", "sumcheck_early", "compute_beta",
             "mle_eval_base", "early_create", "early_claim", "early_fold", "early_finish",
             "early_n_copies", "early_n_wires", "early_destroy"]
    lib = ctypes.CDLL(GPU_LIB)
    for n in names:
        assert hasattr(lib, "native_fp2_" + n), n


def test_init_without_device_reports_unavailable():
    lib = ctypes.CDLL(GPU_LIB)
    lib.native_fp2_init.restype = ctypes.c_int
    lib.native_fp2_cuda_available.restype = ctypes.c_int
    assert lib.native_fp2_init() == 0
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if not has_gpu:
        assert lib.native_fp2_cuda_available() == 0
        # a session cannot be created without a device: NULL, never a CPU fallback
        lib.native_fp2_early_create.restype = ctypes.c_void_p
        one = np.zeros(4, np.uint64)
        g = np.zeros(1, np.int32)
        h = lib.native_fp2_early_create(1, i32p(g), i32p(g), i32p(g), u64p(one), u64p(one), 2, 1,
                                        u64p(one), u64p(one), u64p(one), u64p(one))
        assert not h


# ---- gate decomposition (host code of the library, no GPU) ----------------

def _gate_py(tp, x, y):
    mul = lambda a, b: ((a[0] * b[0] - a[1] * b[1]) % P61, (a[0] * b[1] + a[1] * b[0]) % P61)
    add = lambda a, b: ((a[0] + b[0]) % P61, (a[1] + b[1]) % P61)
    sub = lambda a, b: ((a[0] - b[0]) % P61, (a[1] - b[1]) % P61)
    one, two = (1, 0), (2, 0)
    return {0: lambda: mul(x, y), 1: lambda: add(x, y), 2: lambda: sub(x, y), 3: lambda: x,
            4: lambda: y, 5: lambda: sub(add(x, y), mul(x, y)),
            6: lambda: sub(add(x, y), mul(two, mul(x, y))), 7: lambda: sub(one, x),
            8: lambda: sub(one, mul(x, y)), 9: lambda: sub(add(one, mul(x, y)), add(x, y)),
            10: lambda: sub(add(one, mul(two, mul(x, y))), add(x, y)),
            11: lambda: mul(sub(one, x), y)}.get(tp, lambda: x)()


def _form(lib, gt, i0, i1, zr, zi, W, max_terms=4096):
    k0 = np.zeros(2, np.uint64)
    lin = np.zeros(2 * W, np.uint64)
    ab = np.zeros(2 * max_terms, np.int32)
    c = np.zeros(2 * max_terms, np.uint64)
    nt = lib.tp_gate_form(gt.size, i32p(gt), i32p(i0), i32p(i1), u64p(zr), u64p(zi), W,
                          u64p(k0), u64p(lin), max_terms, i32p(ab), u64p(c))
    return nt, k0, lin, ab, c


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_gate_form_equals_gate_sum(seed):
    lib = ctypes.CDLL(GPU_LIB)
    lib.tp_gate_form.restype = ctypes.c_int
    rng = np.random.default_rng(seed)
    W, G = 9, 60
    gt = rng.integers(-2, 15, size=G).astype(np.int32)
    i0 = rng.integers(0, W, size=G).astype(np.int32)
    i1 = rng.integers(0, W, size=G).astype(np.int32)
    zr, zi = rand_fp(rng, G), rand_fp(rng, G)
    nt, k0, lin, ab, c = _form(lib, gt, i0, i1, zr, zi, W)
    assert nt >= 0
    for _ in range(5):
        V = [(int(a), int(b)) for a, b in zip(rand_fp(rng, W), rand_fp(rng, W))]
        want = (0, 0)
        for g in range(G):
            val = _gate_py(int(gt[g]), V[i0[g]], V[i1[g]])
            z = (int(zr[g]), int(zi[g]))
            t = ((val[0] * z[0] - val[1] * z[1]) % P61, (val[0] * z[1] + val[1] * z[0]) % P61)
            want = ((want[0] + t[0]) % P61, (want[1] + t[1]) % P61)
        got = [int(k0[0]), int(k0[1])]
        for w in range(W):
            l = (int(lin[2 * w]), int(lin[2 * w + 1]))
            got[0] = (got[0] + l[0] * V[w][0] - l[1] * V[w][1]) % P61
            got[1] = (got[1] + l[0] * V[w][1] + l[1] * V[w][0]) % P61
        for t in range(nt):
            a, b = ab[2 * t], ab[2 * t + 1]
            cc = (int(c[2 * t]), int(c[2 * t + 1]))
            xy = ((V[a][0] * V[b][0] - V[a][1] * V[b][1]) % P61,
                  (V[a][0] * V[b][1] + V[a][1] * V[b][0]) % P61)
            got[0] = (got[0] + cc[0] * xy[0] - cc[1] * xy[1]) % P61
            got[1] = (got[1] + cc[0] * xy[1] + cc[1] * xy[0]) % P61
        assert tuple(got) == want


def test_gate_form_groups_crop_products_by_shared_wire(circuits):
    lib = ctypes.CDLL(GPU_LIB)
    lib.tp_gate_form.restype = ctypes.c_int
    rng = np.random.default_rng(7)
    gt, i0, i1 = circuits["Crop_type"], circuits["Crop_in0"], circuits["Crop_in1"]
    zr, zi = rand_fp(rng, gt.size), rand_fp(rng, gt.size)
    nt, k0, lin, ab, c = _form(lib, gt, i0, i1, zr, zi, 512)
    nonzero = int(((zr != 0) | (zi != 0)).sum())       # zero-weight gates drop out
    assert nt == nonzero and nt >= 380
    assert set(ab[1:2 * nt:2].tolist()) == {384}      # one group keyed by the mask wire
    assert not lin.any() and not k0.any()


def test_gate_form_rejects_bad_wire_index():
    lib = ctypes.CDLL(GPU_LIB)
    lib.tp_gate_form.restype = ctypes.c_int
    lib.tp_last_error.restype = ctypes.c_char_p
    gt = np.array([0], np.int32)
    i0 = np.array([3], np.int32)
    i1 = np.array([9], np.int32)
    z = np.ones(1, np.uint64)
    k0 = np.zeros(2, np.uint64)
    lin = np.zeros(8, np.uint64)
    ab = np.zeros(2, np.int32)
    cc = np.zeros(2, np.uint64)
    assert lib.tp_gate_form(1, i32p(gt), i32p(i0), i32p(i1), u64p(z), u64p(z), 4, u64p(k0),
                            u64p(lin), 1, i32p(ab), u64p(cc)) == -1
    assert b"outside" in lib.tp_last_error()
    # an unused operand may be anything (the pass gate ignores in1), as in the reference
    gt[0] = 12
    assert lib.tp_gate_form(1, i32p(gt), i32p(i0), i32p(i1), u64p(z), u64p(z), 4, u64p(k0),
                            u64p(lin), 1, i32p(ab), u64p(cc)) == 0


def test_library_without_device_fails_loudly():
    """With no usable device the library's loader raises instead of falling back
    to a CPU path, and a reference-facing session call returns NULL."""
    from truepix_b200 import native
    lib = native.gkr(require_device=False)
    lib.native_fp2_init()
    if lib.native_fp2_cuda_available():
        pytest.skip("a device is present")
    native._cache.pop("gkr", None)
    with pytest.raises(RuntimeError):
        native.gkr()
    lib = native.gkr(require_device=False)
    gt = np.array([12], np.int32)
    z = np.array([1], np.uint64)
    v = np.array([1, 2], np.uint64)
    h = lib.native_fp2_early_create(1, i32p(gt), i32p(gt * 0), i32p(gt * 0), u64p(z), u64p(z * 0), 2, 1,
                                    u64p(v), u64p(v * 0), u64p(v), u64p(v * 0))
    assert not h


def test_orion_sizes_without_device():
    """tp_orion_codeword_len / tp_orion_tree_leaves are host arithmetic: they
    match the oracle's encode_output_len and the tree padding with no GPU."""
    from orionlib import OrionOracle
    from truepix_b200 import native
    lib = native.gkr(require_device=False)
    orc = OrionOracle()
    for n in (1, 2, 13, 14, 64, 100, 1000, 8192, 65536, 1 << 18):
        assert lib.tp_orion_codeword_len(n) == orc.encode_len(n), n
    assert lib.tp_orion_tree_leaves(128 * 100) == 256
    assert lib.tp_orion_tree_leaves(1 << 23) == 1 << 17
    assert lib.tp_orion_tree_leaves(100) == 0


def test_launcher_handle_keeps_the_lock_and_shares_the_library():
    """native.gkr_launcher(): the same library bound as a PyDLL (calls keep the
    interpreter lock), with the same signatures and the same error state"""
    import ctypes
    from truepix_b200 import native
    lib, quick = native.gkr(require_device=False), native.gkr_launcher()
    assert isinstance(quick, ctypes.PyDLL) and not isinstance(lib, ctypes.PyDLL)
    assert quick.tp_host_sha_mb_available() == lib.tp_host_sha_mb_available()
    bad = np.array([(1 << 61) - 1, 0], np.uint64)
    assert quick.tp_eq_table_host(bad.ctypes.data, 1, np.empty(4, np.uint64).ctypes.data) == -1
    assert lib.tp_last_error_code() != 0 and lib.tp_last_error()
