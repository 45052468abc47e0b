"""Helpers shared by the Orion tests, the golden generator and the bench.

Field elements are 16 bytes in the reference's memory order: u64 img, then
u64 real (TruePix-main/Orion/Orion_nonzk/include/linear_gkr/prime_field.h).
Arrays of n elements are numpy uint64 arrays of 2n words [img0, re0, img1, ...].

`elements(seed, n)` makes seeded inputs without depending on numpy's
generator streams (splitmix64 of seed:index), so fixtures stay valid across
numpy versions.
"""
from __future__ import annotations

import ctypes
import hashlib
import os

import numpy as np

P61 = (1 << 61) - 1
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORION_ORACLE_LIB = os.path.join(ROOT, "oracle", "liborion_oracle.so")
ORION_REF_LIB = os.path.join(ROOT, "oracle", "_ref", "liborion_ref.so")
ORION_ZK_REF_LIB = os.path.join(ROOT, "oracle", "_ref", "liborion_zk_ref.so")

_V = ctypes.c_void_p
_LL = ctypes.c_longlong
_I = ctypes.c_int


def splitmix64(x: np.ndarray) -> np.ndarray:
    with np.errstate(over="ignore"):
        z = x + np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


def elements(seed: int, n: int, kind: str = "random") -> np.ndarray:
    """n canonical Fp2 elements (2n u64 words). kind: random | zero | max | small."""
    if kind == "zero":
        return np.zeros(2 * n, np.uint64)
    if kind == "max":
        return np.full(2 * n, P61 - 1, np.uint64)
    idx = np.arange(2 * n, dtype=np.uint64) + (np.uint64(seed) << np.uint64(40))
    v = splitmix64(idx)
    if kind == "small":
        return v & np.uint64(0xFF)
    return (v >> np.uint64(3)) % np.uint64(P61)


def frame_bytes(seed: int, n: int) -> np.ndarray:
    """n seeded uniform bytes (splitmix64 of seed:index)."""
    idx = np.arange((n + 7) // 8, dtype=np.uint64) + (np.uint64(seed) << np.uint64(40))
    return splitmix64(idx).view(np.uint8)[:n].copy()


def frame_elements(pix: np.ndarray, copies: int, cs: int, W: int, const_idx: int, const_val: int,
                   padded: int) -> np.ndarray:
    """The commit input of a frame (include/truepix/truepix_gkr.h:154-206): element
    copy * W + wire = pixel for wire < cs, const_val at const_idx, zero elsewhere;
    real part only (img 0)."""
    v = np.zeros((padded, W), np.uint64)
    v[:copies, :cs] = pix.reshape(copies, cs)
    if const_idx >= 0:
        v[:copies, const_idx] = const_val
    out = np.zeros(2 * padded * W, np.uint64)
    out[1::2] = v.reshape(-1)
    return out


def virgo_inputs(n: int, seed: int):
    """Three linear_poly tables of n entries {a, b} (4 words each) and a random."""
    return (elements(seed, 2 * n), elements(seed + 1, 2 * n), elements(seed + 2, 2 * n),
            elements(seed + 3, 1))


VIRGO_TYPES = (0, 1, 2, 4, 5, 6, 7, 8, 9, 10, 12, 13, 14)


def virgo_layer(seed: int, length_g: int, length_u: int, types=VIRGO_TYPES) -> dict:
    """A seeded two-layer circuit slice for the Virgo inits: 2^length_g gates of the
    given types over 2^length_u values (ranges of sum / exp-sum gates at most 8
    long, 1-4 (src, weight) terms per custom-comb gate), the randoms r0, r1
    (length_g), alpha, beta, and for phase 2 vma0 ({a, b}), prev_r and r_u
    (length_u). Element arrays as everywhere here: u64 words [img, real, ...]."""
    rng = np.random.default_rng(seed)
    G, U = 1 << length_g, 1 << length_u
    ty = rng.choice(np.array(types, np.int32), size=G).astype(np.int32)
    u = rng.integers(0, U, size=G, dtype=np.int64)
    v = rng.integers(0, U, size=G, dtype=np.int64)
    span = rng.integers(0, 8, size=G, dtype=np.int64)
    u[ty == 4] = rng.integers(0, min(G, U), size=int((ty == 4).sum()), dtype=np.int64)   # a gate and a value index
    lo = rng.integers(0, max(1, U - 8), size=G, dtype=np.int64)
    r5, r12 = ty == 5, ty == 12
    u[r5], v[r5] = lo[r5], np.minimum(lo[r5] + span[r5], U)
    u[r12], v[r12] = lo[r12], np.minimum(lo[r12] + span[r12], U - 1)
    n_terms = np.where(ty == 14, rng.integers(1, 5, size=G), 0)
    comb_ptr = np.zeros(G + 1, np.int32)
    comb_ptr[1:] = np.cumsum(n_terms)
    comb_src = rng.integers(0, U, size=max(1, int(comb_ptr[-1])), dtype=np.int64).astype(np.int32)
    comb_w = elements(seed + 7, max(1, int(comb_ptr[-1])))
    return dict(length_g=length_g, length_u=length_u, ty=ty, u=u, v=v, comb_ptr=comb_ptr, comb_src=comb_src,
                comb_w=comb_w, values=elements(seed + 1, U), r0=elements(seed + 2, length_g),
                r1=elements(seed + 3, length_g), alpha=elements(seed + 4, 1), beta=elements(seed + 5, 1),
                vma0=elements(seed + 6, 2), prev_r=elements(seed + 8, 1), r_u=elements(seed + 9, max(1, length_u)))


def digest(a: np.ndarray) -> bytes:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).digest()


def _vp(a: np.ndarray):
    assert a.flags["C_CONTIGUOUS"]
    return ctypes.c_void_p(a.ctypes.data)


class OrionOracle:
    """ctypes view of oracle/orion_oracle.c (the C restatement)."""

    def __init__(self, path: str = ORION_ORACLE_LIB):
        L = self.lib = ctypes.CDLL(path)
        L.oracle_sha256_64.argtypes = [ctypes.c_char_p, _V]
        L.oracle_glibc_stream.argtypes = [ctypes.c_uint32, _I, _V]
        L.oracle_encode_len.argtypes = [_LL]
        L.oracle_encode_len.restype = _LL
        L.oracle_orion_commit.argtypes = [_V, _LL, _V, _V]
        L.oracle_fft.argtypes = [_V, _LL, _LL, _V]
        L.oracle_ifft.argtypes = [_V, _LL, _LL, _V]
        L.oracle_rs_commit.argtypes = [_V, _I, _V, _V]
        L.oracle_encode.argtypes = [_V, _LL, _V]
        L.oracle_encode.restype = _LL
        L.oracle_orion_combine.argtypes = [_V, _LL, _V, _V, _V, _V, _V]
        L.oracle_fri_step.argtypes = [_V, _I, _V, _V, _V]
        L.oracle_virgo_update.argtypes = [_V, _V, _V, _LL, _V, _I, _V, _V, _V, _V]
        L.oracle_virgo_phase1_init.argtypes = [_LL, _V, _V, _V, _V, _V, _V, _I, _I, _V, _V, _V, _V, _V, _V, _V, _V]
        L.oracle_virgo_phase2_init.argtypes = [_LL, _V, _V, _V, _V, _V, _V, _I, _I, _V, _V, _V, _V, _V, _V, _V, _V,
                                               _V, _V, _V]
        L.oracle_frame_vector.argtypes = [_V, _I, _I, _I, _I, _I, ctypes.c_uint64, ctypes.c_uint64, _I, _V]

    def sha256_64(self, msg: bytes) -> bytes:
        assert len(msg) == 64
        out = ctypes.create_string_buffer(32)
        self.lib.oracle_sha256_64(msg, out)
        return out.raw

    def glibc_rand(self, seed: int, n: int) -> list:
        out = (ctypes.c_int * n)()
        self.lib.oracle_glibc_stream(seed, n, out)
        return list(out)

    def encode_len(self, n: int) -> int:
        return self.lib.oracle_encode_len(n)

    def encode(self, src: np.ndarray) -> np.ndarray:
        n = src.size // 2
        out = np.zeros(2 * self.encode_len(n), np.uint64)
        assert self.lib.oracle_encode(_vp(src), n, _vp(out)) == out.size // 2
        return out

    def commit(self, src: np.ndarray, leaves: bool = False):
        n = src.size // 2
        root = ctypes.create_string_buffer(32)
        lv = np.zeros(2 * (n // 128) * 32, np.uint8) if leaves else None
        rc = self.lib.oracle_orion_commit(_vp(src), n, root, _vp(lv) if leaves else None)
        if rc != 0:
            raise ValueError("oracle_orion_commit: %d" % rc)
        return (root.raw, lv.reshape(-1, 32)) if leaves else root.raw

    def frame_vector(self, pix: np.ndarray, copies: int, cs: int, W: int, const_idx: int, const_val: int,
                     padded: int, seed: int = 0, mode: int = 0) -> np.ndarray:
        """The frame's polynomial as base-field values (mode 0 plain, 1 masked, 2 mask)."""
        out = np.zeros(padded * W, np.uint64)
        pix = np.ascontiguousarray(pix, np.uint8)
        rc = self.lib.oracle_frame_vector(_vp(pix), copies, padded, cs, W, const_idx, const_val, seed, mode,
                                          _vp(out))
        if rc != 0:
            raise ValueError("oracle_frame_vector: %d" % rc)
        return out

    def zk_commit(self, pix: np.ndarray, copies: int, cs: int, W: int, const_idx: int, const_val: int,
                  padded: int, seed: int):
        """(masked root, mask root) of the ZK commit pair of a frame."""
        roots = []
        for mode in (1, 2):
            v = self.frame_vector(pix, copies, cs, W, const_idx, const_val, padded, seed, mode)
            src = np.zeros(2 * v.size, np.uint64)
            src[1::2] = v
            roots.append(self.commit(src))
        return tuple(roots)

    def virgo_init(self, phase: int, L: dict):
        """(V_mult_add, addV_array, add_mult_sum) after sumcheck_phase{1,2}_init."""
        U = 1 << L["length_u"]
        outs = [np.zeros(4 * U, np.uint64) for _ in range(3)]
        common = [1 << L["length_g"], _vp(L["ty"]), _vp(L["u"]), _vp(L["v"]), _vp(L["comb_ptr"]), _vp(L["comb_src"]),
                  _vp(L["comb_w"]), L["length_g"], L["length_u"], _vp(L["values"]), _vp(L["r0"]), _vp(L["r1"]),
                  _vp(L["alpha"]), _vp(L["beta"])]
        if phase == 1:
            rc = self.lib.oracle_virgo_phase1_init(*common, *[_vp(o) for o in outs])
        else:
            rc = self.lib.oracle_virgo_phase2_init(*common, _vp(L["vma0"]), _vp(L["prev_r"]), _vp(L["r_u"]),
                                                   *[_vp(o) for o in outs])
        if rc != 0:
            raise ValueError("oracle_virgo_phase%d_init: %d" % (phase, rc))
        return tuple(outs)

    def combine(self, src: np.ndarray, r0: np.ndarray, r1: np.ndarray):
        """(combined codeword, root of its tree, answer) of the opening passes."""
        n = src.size // 2
        comb = np.zeros(2 * self.encode_len(n // 128), np.uint64)
        root = ctypes.create_string_buffer(32)
        ans = np.zeros(2, np.uint64)
        rc = self.lib.oracle_orion_combine(_vp(src), n, _vp(r0), _vp(r1), _vp(comb), root, _vp(ans))
        assert rc == 0
        return comb, root.raw, ans

    def fri_step(self, w: np.ndarray, log_m: int, r: np.ndarray):
        """(next interleaved witness, root) of one FRI commit-phase step."""
        nxt = np.zeros(w.size // 2, np.uint64)
        root = ctypes.create_string_buffer(32)
        assert self.lib.oracle_fri_step(_vp(w), log_m, _vp(r), _vp(nxt), root) == 0
        return nxt, root.raw

    def virgo_update(self, vma, addv, ams, r, bit):
        """(folded tables x3, ret [6 words]) of one Virgo sumcheck round."""
        n = vma.size // 4
        outs = [np.zeros(2 * n, np.uint64) for _ in range(3)]
        ret = np.zeros(6, np.uint64)
        rc = self.lib.oracle_virgo_update(_vp(vma), _vp(addv), _vp(ams), n, _vp(r), bit,
                                          *[_vp(o) for o in outs], _vp(ret))
        assert rc == 0
        return outs, ret

    def fft(self, coef: np.ndarray, order: int) -> np.ndarray:
        out = np.zeros(2 * order, np.uint64)
        assert self.lib.oracle_fft(_vp(coef), coef.size // 2, order, _vp(out)) == 0
        return out

    def ifft(self, evals: np.ndarray, coef_len: int) -> np.ndarray:
        out = np.zeros(2 * coef_len, np.uint64)
        assert self.lib.oracle_ifft(_vp(evals), coef_len, evals.size // 2, _vp(out)) == 0
        return out

    def rs_commit(self, src: np.ndarray, log_len: int, want_codeword: bool = False):
        root = ctypes.create_string_buffer(32)
        cw = np.zeros(2 << (log_len + 5), np.uint64) if want_codeword else None
        rc = self.lib.oracle_rs_commit(_vp(src), log_len, root, _vp(cw) if want_codeword else None)
        assert rc == 0
        return (root.raw, cw) if want_codeword else root.raw
