"""The circuit-output golden cases (tests/golden/circuit_outputs_golden.npz) and
the oracle's restatement of the reference circuit evaluator
(oracle_circuit_outputs in oracle/liboracle_fp2.so)."""
from __future__ import annotations

import ctypes
import json
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_LIB = os.path.join(ROOT, "oracle", "liboracle_fp2.so")


def golden_cases():
    g = np.load(os.path.join(ROOT, "tests", "golden", "circuit_outputs_golden.npz"))
    names = sorted(k[:-4] for k in g.files if k.endswith("_pix"))
    for n in names:
        copies, padded, cs, n_wires, ci, cv = json.loads(g[n + "_layout"].tobytes().decode())
        gates = g[n + "_gates"]
        yield dict(name=n, pix=g[n + "_pix"], copies=copies, padded=padded, cs=cs, n_wires=n_wires,
                   const_idx=ci, const_val=int(cv), gt=np.ascontiguousarray(gates[0]),
                   i0=np.ascontiguousarray(gates[1]), i1=np.ascontiguousarray(gates[2]), out=g[n + "_out"])


def oracle_outputs(pix, copies, padded, cs, n_wires, const_idx, const_val, gt, i0, i1):
    lib = ctypes.CDLL(ORACLE_LIB)
    f = lib.oracle_circuit_outputs
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                  ctypes.c_uint64, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    bits = (len(gt) - 1).bit_length()
    out = np.empty(padded << bits, np.uint64)
    pix = np.ascontiguousarray(pix, np.uint8)
    gt, i0, i1 = (np.ascontiguousarray(a, np.int32) for a in (gt, i0, i1))
    assert f(pix.ctypes.data, copies, padded, cs, n_wires, const_idx, const_val, len(gt), gt.ctypes.data,
             i0.ctypes.data, i1.ctypes.data, out.ctypes.data) == 0
    return out
