"""ctypes bindings shared by the tests, the smoke check and the bench.

`bind(path, prefix)` loads a shared library that exports the native_fp2 symbol
set (reference names `native_fp2_*`, or the oracle's `oracle_fp2_*`) and wraps
every entry point in a numpy-friendly helper. The prototypes are those of
TruePix-main/native_fp2/native_fp2.cpp:11-160 (ctypes types as in
TruePix-main/libTruePix/native_fp2_bridge.py:48-113).
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

P61 = (1 << 61) - 1
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_LIB = os.path.join(ROOT, "oracle", "liboracle_fp2.so")
REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libnative_fp2_ref.so")
# the reference's GPU library (TruePix-main/native_fp2/native_fp2.cu for sm_100a)
REF_GPU_LIB = os.path.join(ROOT, "oracle", "_ref", "libnative_fp2_ref_gpu.so")
GPU_LIB = os.path.join(ROOT, "truepix_b200", "lib", "libnative_fp2_gpu.so")

_U64P = ctypes.POINTER(ctypes.c_uint64)
_I32P = ctypes.POINTER(ctypes.c_int)
_U64 = ctypes.c_uint64
_I32 = ctypes.c_int
_SZ = ctypes.c_size_t
_VP = ctypes.c_void_p


def u64p(a: np.ndarray):
    assert a.dtype == np.uint64 and a.flags["C_CONTIGUOUS"], (a.dtype, a.flags)
    return a.ctypes.data_as(_U64P)


def i32p(a: np.ndarray):
    assert a.dtype == np.int32 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_I32P)


class Fp2Lib:
    """One loaded library exposing the 14 native_fp2 entry points."""

    def __init__(self, path: str, prefix: str = "native_fp2_"):
        self.path = path
        self.lib = ctypes.CDLL(path)
        self.prefix = prefix
        L, p = self.lib, prefix

        def f(name, res, args):
            fn = getattr(L, p + name)
            fn.restype = res
            fn.argtypes = args
            return fn

        if hasattr(L, p + "init"):
            self._init = f("init", ctypes.c_int, [])
            self._avail = f("cuda_available", ctypes.c_int, [])
        else:
            self._init = self._avail = None
        self._fold = f("fold", None, [_U64P, _U64P, _SZ, _U64, _U64, _U64P, _U64P])
        self._expand = f("expand", None, [_U64P, _U64P, _SZ, _SZ, _U64P, _U64P])
        self._sc = f("sumcheck_early", None,
                     [_I32, _I32P, _I32P, _I32P, _U64P, _U64P, _I32, _I32]
                     + [_U64P] * 12 + [_U64P])
        self._beta = f("compute_beta", None, [_U64P, _U64P, _I32, _U64, _U64, _U64P, _U64P])
        self._mle = f("mle_eval_base", None, [_U64P, _U64P, _U64P, _I32, _U64P, _U64P])
        self._create = f("early_create", _VP,
                         [_I32, _I32P, _I32P, _I32P, _U64P, _U64P, _I32, _I32,
                          _U64P, _U64P, _U64P, _U64P])
        self._claim = f("early_claim", ctypes.c_int, [_VP, _U64P])
        self._efold = f("early_fold", ctypes.c_int, [_VP, _U64, _U64])
        self._finish = f("early_finish", ctypes.c_int, [_VP, _U64P, _U64P, _U64P, _U64P])
        self._ncop = f("early_n_copies", ctypes.c_int, [_VP])
        self._nw = f("early_n_wires", ctypes.c_int, [_VP])
        self._destroy = f("early_destroy", None, [_VP])
        self._err = None
        if hasattr(L, "tp_last_error"):
            self._err = L.tp_last_error
            self._err.restype = ctypes.c_char_p
            self._err.argtypes = []
            self._errc = L.tp_last_error_code
            self._errc.restype = ctypes.c_int
            self._errc.argtypes = []

    # -- error state of the product library (absent in oracle / reference) --
    def check(self):
        if self._err is not None and self._errc() != 0:
            raise RuntimeError("native_fp2: " + self._err().decode())

    def init(self) -> int:
        return self._init() if self._init else 0

    def cuda_available(self) -> int:
        return self._avail() if self._avail else 0

    def fold(self, re, im, r):
        n_out = re.size // 2
        ore = np.zeros(n_out, np.uint64)
        oim = np.zeros(n_out, np.uint64)
        self._fold(u64p(re), u64p(im), n_out, int(r[0]), int(r[1]), u64p(ore), u64p(oim))
        self.check()
        return ore, oim

    def expand(self, re, im, ncopies):
        n = re.size
        ore = np.zeros(n * ncopies, np.uint64)
        oim = np.zeros(n * ncopies, np.uint64)
        self._expand(u64p(re), u64p(im), n, ncopies, u64p(ore), u64p(oim))
        self.check()
        return ore, oim

    def sumcheck_early(self, gt, i0, i1, z1re, z1im, n_copies, n_wires, vre, vim,
                       f0re, f0im, f1re, f1im, bre, bim, bf0re, bf0im, bf1re, bf1im):
        out = np.zeros(8, np.uint64)
        self._sc(gt.size, i32p(gt), i32p(i0), i32p(i1), u64p(z1re), u64p(z1im),
                 n_copies, n_wires, u64p(vre), u64p(vim), u64p(f0re), u64p(f0im),
                 u64p(f1re), u64p(f1im), u64p(bre), u64p(bim), u64p(bf0re), u64p(bf0im),
                 u64p(bf1re), u64p(bf1im), u64p(out))
        self.check()
        return out

    def compute_beta(self, zre, zim, init):
        n = 1 << zre.size
        ore = np.zeros(n, np.uint64)
        oim = np.zeros(n, np.uint64)
        self._beta(u64p(zre), u64p(zim), zre.size, int(init[0]), int(init[1]),
                   u64p(ore), u64p(oim))
        self.check()
        return ore, oim

    def mle_eval_base(self, inputs, zre, zim):
        ore = np.zeros(1, np.uint64)
        oim = np.zeros(1, np.uint64)
        self._mle(u64p(inputs), u64p(zre), u64p(zim), zre.size, u64p(ore), u64p(oim))
        self.check()
        return int(ore[0]), int(oim[0])

    # -- early session --
    def early_create(self, gt, i0, i1, z1re, z1im, n_copies, n_wires, vre, vim, bre, bim):
        h = self._create(gt.size, i32p(gt), i32p(i0), i32p(i1), u64p(z1re), u64p(z1im),
                         n_copies, n_wires, u64p(vre), u64p(vim), u64p(bre), u64p(bim))
        return h

    def early_claim(self, h):
        out = np.zeros(8, np.uint64)
        rc = self._claim(h, u64p(out))
        return rc, out

    def early_fold(self, h, r):
        return self._efold(h, int(r[0]), int(r[1]))

    def early_finish(self, h, n_wires):
        wre = np.zeros(n_wires, np.uint64)
        wim = np.zeros(n_wires, np.uint64)
        bre = np.zeros(1, np.uint64)
        bim = np.zeros(1, np.uint64)
        rc = self._finish(h, u64p(wre), u64p(wim), u64p(bre), u64p(bim))
        return rc, wre, wim, (int(bre[0]), int(bim[0]))

    def early_n_copies(self, h):
        return self._ncop(h)

    def early_n_wires(self, h):
        return self._nw(h)

    def early_destroy(self, h):
        self._destroy(h)


def run_session(lib: Fp2Lib, gt, i0, i1, z1re, z1im, n_copies, n_wires, vre, vim, bre, bim,
                challenges):
    """Drive claim/fold for every copy bit, then finish; returns all outputs."""
    h = lib.early_create(gt, i0, i1, z1re, z1im, n_copies, n_wires, vre, vim, bre, bim)
    if not h:
        lib.check()
        raise RuntimeError("early_create returned NULL")
    claims = []
    ncs = []
    try:
        k = 0
        while lib.early_n_copies(h) > 1:
            rc, out = lib.early_claim(h)
            if rc != 0:
                lib.check()
                raise RuntimeError("early_claim failed")
            claims.append(out)
            rc = lib.early_fold(h, challenges[k])
            if rc != 0:
                lib.check()
                raise RuntimeError("early_fold failed")
            ncs.append(lib.early_n_copies(h))
            k += 1
        rc, wre, wim, beta = lib.early_finish(h, n_wires)
        if rc != 0:
            lib.check()
            raise RuntimeError("early_finish failed")
    finally:
        lib.early_destroy(h)
    return np.stack(claims) if claims else np.zeros((0, 8), np.uint64), wre, wim, beta, ncs


def rand_fp(rng, n):
    """Uniform canonical base-field elements with the edge values mixed in."""
    x = rng.integers(0, P61, size=n, dtype=np.uint64)
    if n >= 4:
        x[0] = 0
        x[1] = P61 - 1
        x[2] = 1
        x[3] = (1 << 60)
    return x
