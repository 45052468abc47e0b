"""ctypes bridge to the B200 GKR kernels (libnative_fp2_gpu.so).

Mirror of TruePix-main/libTruePix/native_fp2_bridge.py: same module flags
(ENABLE_GPU, AVAILABLE, GPU_ACTIVE, GPU_FAIL_REASON), same functions and classes
(Fp2Buf, fold_values, sumcheck_early, EarlySession, early_session_create,
cache_gate_tables, resolve_gate_type_idx, compute_beta, mle_eval_base) with the
same arguments and return types, so LayerProver / LayerComputeV / VerifierIOMLExt
can import it unchanged.

Differences, on purpose:
  * One library only. There is no CPU library and no CPU fallback: when the CUDA
    library or the device is missing, AVAILABLE and GPU_ACTIVE are False and
    every entry point raises RuntimeError naming the reason.
  * Every native call is checked; a failure inside the library raises
    RuntimeError with the library's message instead of returning silently.
"""
from __future__ import annotations

import array as _array
import ctypes
import os
from typing import List, Optional, Sequence, Tuple

try:  # inside the TruePix tree use its field type, so values pickle identically
    from libTruePix.extfield import BASE_PRIME_61, Fp2, _raw  # type: ignore
except Exception:  # standalone
    from .fp2 import BASE_PRIME_61, Fp2, _raw


def _env_enable_gpu() -> bool:
    v = os.environ.get("TRUEPIX_ENABLE_GPU", "").strip().lower()
    return v not in ("0", "false", "no", "off")


ENABLE_GPU = _env_enable_gpu()

_LIB = None
_GPU_LIB = None
AVAILABLE = False
GPU_ACTIVE = False
GPU_FAIL_REASON = ""

_U64 = ctypes.c_uint64
_I32 = ctypes.c_int
_SIZE = ctypes.c_size_t
_VOID_P = ctypes.c_void_p
_PU64 = ctypes.POINTER(_U64)
_PI32 = ctypes.POINTER(_I32)

HERE = os.path.dirname(os.path.realpath(__file__))
DEFAULT_LIB = os.path.join(HERE, "lib", "libnative_fp2_gpu.so")


def _bind(lib) -> None:
    sig = {
        "native_fp2_init": (ctypes.c_int, []),
        "native_fp2_cuda_available": (ctypes.c_int, []),
        "native_fp2_fold": (None, [_PU64, _PU64, _SIZE, _U64, _U64, _PU64, _PU64]),
        "native_fp2_expand": (None, [_PU64, _PU64, _SIZE, _SIZE, _PU64, _PU64]),
        "native_fp2_sumcheck_early": (None, [_I32, _PI32, _PI32, _PI32, _PU64, _PU64, _I32, _I32]
                                      + [_PU64] * 13),
        "native_fp2_compute_beta": (None, [_PU64, _PU64, _I32, _U64, _U64, _PU64, _PU64]),
        "native_fp2_mle_eval_base": (None, [_PU64, _PU64, _PU64, _I32, _PU64, _PU64]),
        "native_fp2_early_create": (_VOID_P, [_I32, _PI32, _PI32, _PI32, _PU64, _PU64, _I32, _I32,
                                              _PU64, _PU64, _PU64, _PU64]),
        "native_fp2_early_claim": (ctypes.c_int, [_VOID_P, _PU64]),
        "native_fp2_early_fold": (ctypes.c_int, [_VOID_P, _U64, _U64]),
        "native_fp2_early_finish": (ctypes.c_int, [_VOID_P, _PU64, _PU64, _PU64, _PU64]),
        "native_fp2_early_n_copies": (ctypes.c_int, [_VOID_P]),
        "native_fp2_early_n_wires": (ctypes.c_int, [_VOID_P]),
        "native_fp2_early_destroy": (None, [_VOID_P]),
        "tp_last_error_code": (ctypes.c_int, []),
        "tp_last_error": (ctypes.c_char_p, []),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args


def _load() -> None:
    global _LIB, _GPU_LIB, AVAILABLE, GPU_ACTIVE, GPU_FAIL_REASON
    if not ENABLE_GPU:
        GPU_FAIL_REASON = "TRUEPIX_ENABLE_GPU disabled (this library has no CPU path)"
        return
    path = os.environ.get("TRUEPIX_NATIVE_FP2_GPU_LIB", DEFAULT_LIB)
    if not os.path.isfile(path):
        GPU_FAIL_REASON = "missing %s (python -m truepix_b200.build)" % path
        return
    try:
        lib = ctypes.CDLL(path)
        _bind(lib)
    except (OSError, AttributeError) as exc:
        GPU_FAIL_REASON = "cannot load %s: %s" % (path, exc)
        return
    if lib.native_fp2_init() != 0 or not lib.native_fp2_cuda_available():
        GPU_FAIL_REASON = "no usable CUDA device: %s" % lib.tp_last_error().decode()
        return
    _LIB = _GPU_LIB = lib
    AVAILABLE = GPU_ACTIVE = True
    GPU_FAIL_REASON = ""


_load()


def _require():
    if _LIB is None:
        raise RuntimeError("native_fp2 GPU library not available: " + GPU_FAIL_REASON)
    return _LIB


def _check(lib) -> None:
    if lib.tp_last_error_code() != 0:
        raise RuntimeError("native_fp2: " + lib.tp_last_error().decode())


def cuda_available() -> bool:
    return GPU_ACTIVE


def early_session_supported() -> bool:
    return GPU_ACTIVE and _GPU_LIB is not None


class Fp2Buf:
    """Contiguous Fp2 vector (real[], imag[]) with list-like access."""
    __slots__ = ("real", "imag", "n")

    def __init__(self, real, imag, n: Optional[int] = None):
        self.real = real
        self.imag = imag
        self.n = int(n if n is not None else len(real))

    def __len__(self) -> int:
        return self.n

    def __getitem__(self, idx):
        if isinstance(idx, slice):
            start, stop, step = idx.indices(self.n)
            if step != 1:
                return [_raw(self.real[i], self.imag[i], BASE_PRIME_61)
                        for i in range(start, stop, step)]
            n = stop - start
            if n <= 0:
                return Fp2Buf((_U64 * 0)(), (_U64 * 0)(), 0)
            rr = (_U64 * n)()
            ii = (_U64 * n)()
            ctypes.memmove(rr, ctypes.byref(self.real, start * 8), n * 8)
            ctypes.memmove(ii, ctypes.byref(self.imag, start * 8), n * 8)
            return Fp2Buf(rr, ii, n)
        return _raw(self.real[idx], self.imag[idx], BASE_PRIME_61)

    def __iter__(self):
        for i in range(self.n):
            yield _raw(self.real[i], self.imag[i], BASE_PRIME_61)

    def to_list(self) -> List[Fp2]:
        return list(self)


def _as_fp2_challenge(val) -> Fp2:
    if isinstance(val, Fp2):
        return val
    return _raw(int(val) % BASE_PRIME_61, 0, BASE_PRIME_61)


def _coords_from_values(values: Sequence):
    if isinstance(values, Fp2Buf):
        return values.real, values.imag, values.n
    n = len(values)
    re = (_U64 * n)()
    im = (_U64 * n)()
    p = BASE_PRIME_61
    for i, v in enumerate(values):
        if isinstance(v, Fp2):
            re[i] = v.real
            im[i] = v.imag
        else:
            re[i] = int(v) % p
    return re, im, n


def _pack_wire_rows(rows: Sequence, n_wires: int, n_cols: int):
    p = BASE_PRIME_61
    re = (_U64 * (n_wires * n_cols))()
    im = (_U64 * (n_wires * n_cols))()
    for w in range(n_wires):
        row = rows[w]
        base = w * n_cols
        if isinstance(row, Fp2Buf):
            ctypes.memmove(ctypes.byref(re, base * 8), row.real, n_cols * 8)
            ctypes.memmove(ctypes.byref(im, base * 8), row.imag, n_cols * 8)
            continue
        for c in range(n_cols):
            v = row[c]
            if isinstance(v, Fp2):
                re[base + c] = v.real
                im[base + c] = v.imag
            else:
                re[base + c] = int(v) % p
    return re, im


def _z1_arrays(z1: Sequence, n_gates: int):
    p = BASE_PRIME_61
    z1r = (_U64 * n_gates)()
    z1i = (_U64 * n_gates)()
    for g, z in enumerate(z1):
        if isinstance(z, Fp2):
            z1r[g] = z.real
            z1i[g] = z.imag
        else:
            z1r[g] = int(z) % p
    return z1r, z1i


def fold_values(values: Sequence, challenge, expand_ncopies: int = 1) -> Tuple[Fp2Buf, Fp2Buf]:
    """Fold pairs; returns (outputs, scratch) as Fp2Buf."""
    lib = _require()
    chal = _as_fp2_challenge(challenge)
    in_r, in_i, n_in = _coords_from_values(values)
    n_out = n_in // 2
    out_r = (_U64 * n_out)()
    out_i = (_U64 * n_out)()
    lib.native_fp2_fold(in_r, in_i, _SIZE(n_out), _U64(chal.real), _U64(chal.imag), out_r, out_i)
    _check(lib)
    scratch = Fp2Buf(out_r, out_i, n_out)
    if expand_ncopies <= 1:
        return scratch, scratch
    n_exp = n_out * expand_ncopies
    exp_r = (_U64 * n_exp)()
    exp_i = (_U64 * n_exp)()
    lib.native_fp2_expand(out_r, out_i, _SIZE(n_out), _SIZE(expand_ncopies), exp_r, exp_i)
    _check(lib)
    return Fp2Buf(exp_r, exp_i, n_exp), scratch


def sumcheck_early(gate_type, in0, in1, z1, n_copies: int, n_wires: int, values, fact0, fact1,
                   beta, beta_f0, beta_f1) -> List[Fp2]:
    lib = _require()
    n_gates = len(gate_type)
    half_n = n_copies >> 1
    p = BASE_PRIME_61
    gt = (_I32 * n_gates)(*gate_type)
    i0a = (_I32 * n_gates)(*in0)
    i1a = (_I32 * n_gates)(*in1)
    z1r, z1i = _z1_arrays(z1, n_gates)
    vr, vi = _pack_wire_rows(values, n_wires, n_copies)
    f0r, f0i = _pack_wire_rows(fact0, n_wires, half_n)
    f1r, f1i = _pack_wire_rows(fact1, n_wires, half_n)
    br, bi, _ = _coords_from_values(beta)
    bf0r, bf0i, _ = _coords_from_values(beta_f0)
    bf1r, bf1i, _ = _coords_from_values(beta_f1)
    out8 = (_U64 * 8)()
    lib.native_fp2_sumcheck_early(_I32(n_gates), gt, i0a, i1a, z1r, z1i, _I32(n_copies),
                                  _I32(n_wires), vr, vi, f0r, f0i, f1r, f1i, br, bi, bf0r, bf0i,
                                  bf1r, bf1i, out8)
    _check(lib)
    return [_raw(out8[0], out8[1], p), _raw(out8[2], out8[3], p),
            _raw(out8[4], out8[5], p), _raw(out8[6], out8[7], p)]


class EarlySession:
    """Resident early-round GKR session on the device."""

    __slots__ = ("_handle", "_n_wires")

    def __init__(self, handle, n_wires: int):
        self._handle = handle
        self._n_wires = int(n_wires)

    @property
    def n_copies(self) -> int:
        return int(_GPU_LIB.native_fp2_early_n_copies(self._handle))

    @property
    def n_wires(self) -> int:
        return self._n_wires

    def claim(self) -> List[Fp2]:
        out8 = (_U64 * 8)()
        if _GPU_LIB.native_fp2_early_claim(self._handle, out8) != 0:
            raise RuntimeError("native_fp2_early_claim failed: " + _GPU_LIB.tp_last_error().decode())
        p = BASE_PRIME_61
        return [_raw(out8[0], out8[1], p), _raw(out8[2], out8[3], p),
                _raw(out8[4], out8[5], p), _raw(out8[6], out8[7], p)]

    def fold(self, challenge) -> None:
        chal = _as_fp2_challenge(challenge)
        if _GPU_LIB.native_fp2_early_fold(self._handle, _U64(chal.real), _U64(chal.imag)) != 0:
            raise RuntimeError("native_fp2_early_fold failed: " + _GPU_LIB.tp_last_error().decode())

    def finish(self) -> Tuple[List[Fp2], Fp2]:
        n = self._n_wires
        wr = (_U64 * n)()
        wi = (_U64 * n)()
        br = _U64()
        bi = _U64()
        if _GPU_LIB.native_fp2_early_finish(self._handle, wr, wi, ctypes.byref(br),
                                            ctypes.byref(bi)) != 0:
            raise RuntimeError("native_fp2_early_finish failed: " + _GPU_LIB.tp_last_error().decode())
        p = BASE_PRIME_61
        return [_raw(wr[i], wi[i], p) for i in range(n)], _raw(br.value, bi.value, p)

    def destroy(self) -> None:
        if self._handle:
            _GPU_LIB.native_fp2_early_destroy(self._handle)
            self._handle = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


def early_session_create(gate_type, in0, in1, z1, n_copies: int, n_wires: int, values,
                         beta) -> EarlySession:
    if not early_session_supported():
        raise RuntimeError("native_fp2 early session API not available: " + GPU_FAIL_REASON)
    n_gates = len(gate_type)
    gt = (_I32 * n_gates)(*gate_type)
    i0a = (_I32 * n_gates)(*in0)
    i1a = (_I32 * n_gates)(*in1)
    z1r, z1i = _z1_arrays(z1, n_gates)
    vr, vi = _pack_wire_rows(values, n_wires, n_copies)
    br, bi, _ = _coords_from_values(beta)
    handle = _GPU_LIB.native_fp2_early_create(_I32(n_gates), gt, i0a, i1a, z1r, z1i,
                                              _I32(n_copies), _I32(n_wires), vr, vi, br, bi)
    if not handle:
        raise RuntimeError("native_fp2_early_create failed: " + _GPU_LIB.tp_last_error().decode())
    return EarlySession(handle, n_wires)


def resolve_gate_type_idx(gate) -> int:
    """Gate object -> native type index (needs TruePix's gateprover module)."""
    from libTruePix import gateprover as gp  # type: ignore
    tp = type(gate)
    if tp is gp.MuxGateProver:
        bit = gate.layer.circuit.muxbits[gate.muxbit]
        return 4 if bit else 3
    idx = getattr(gate, "gate_type_idx", None)
    if idx is not None:
        return int(idx)
    mapping = {
        gp.MulGateProver: 0, gp.AddGateProver: 1, gp.SubGateProver: 2, gp.OrGateProver: 5,
        gp.XorGateProver: 6, gp.NotGateProver: 7, gp.NandGateProver: 8, gp.NorGateProver: 9,
        gp.NxorGateProver: 10, gp.NaabGateProver: 11, gp.PassGateProver: 12,
    }
    return mapping.get(tp, 12)


def cache_gate_tables(gates) -> Tuple[List[int], List[int], List[int]]:
    return ([resolve_gate_type_idx(g) for g in gates], [g.in0 for g in gates],
            [g.in1 for g in gates])


def compute_beta(z: Sequence, init=1) -> Fp2Buf:
    """Beta table over Fp2 challenges; returns Fp2Buf of length 2^len(z)."""
    lib = _require()
    n = len(z)
    if n == 0:
        return Fp2Buf((_U64 * 0)(), (_U64 * 0)(), 0)
    zr, zi, _ = _coords_from_values(z)
    out_n = 1 << n
    out_r = (_U64 * out_n)()
    out_i = (_U64 * out_n)()
    if isinstance(init, Fp2):
        ir, ii = init.real, init.imag
    else:
        ir, ii = int(init) % BASE_PRIME_61, 0
    lib.native_fp2_compute_beta(zr, zi, _I32(n), _U64(ir), _U64(ii), out_r, out_i)
    _check(lib)
    return Fp2Buf(out_r, out_i, out_n)


def mle_eval_base(inputs: Sequence, z: Sequence) -> Fp2:
    """MLE of base-field inputs (zero-padded to 2^len(z)) at the Fp2 point z."""
    lib = _require()
    n_z = len(z)
    n = 1 << n_z
    p = BASE_PRIME_61
    lim = min(len(inputs), n)
    if lim and type(inputs[0]) is int:
        a = _array.array("Q")
        if lim == len(inputs) and lim == n:
            try:
                a.fromlist(inputs if isinstance(inputs, list) else list(inputs))
            except (TypeError, OverflowError):
                a = _array.array("Q", (int(v) % p for v in inputs))
        else:
            a.extend(int(inputs[i]) % p for i in range(lim))
            if lim < n:
                a.extend([0] * (n - lim))
        buf = (_U64 * n).from_buffer(a)
    else:
        buf = (_U64 * n)()
        for i in range(lim):
            v = inputs[i]
            if isinstance(v, Fp2):
                if v.imag != 0:
                    raise TypeError("mle_eval_base expects base-field inputs")
                buf[i] = v.real
            else:
                buf[i] = int(v) % p
    zr, zi, _ = _coords_from_values(z)
    out_r = _U64()
    out_i = _U64()
    lib.native_fp2_mle_eval_base(buf, zr, zi, _I32(n_z), ctypes.byref(out_r), ctypes.byref(out_i))
    _check(lib)
    return _raw(out_r.value, out_i.value, p)
