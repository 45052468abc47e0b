"""Replay of the Fiat-Shamir golden scripts (tests/golden/fs_golden.npz).

`replay_python` restates the reference transcript's binary format with Python's
hashlib (test infrastructure: it checks the golden vectors on CPU);
`replay_lib` drives the library's tp_fs_* host entry points through ctypes."""
from __future__ import annotations

import ctypes
import hashlib
import json
import os
import struct

import numpy as np

P61 = (1 << 61) - 1
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def golden():
    return np.load(os.path.join(ROOT, "tests", "golden", "fs_golden.npz"))


def scripts(g):
    for k in sorted(g.files):
        if k.startswith("fsscript_"):
            name = k[len("fsscript_"):]
            protocol, ops = json.loads(g[k].tobytes().decode())
            yield name, protocol, ops


def py_value(x, fp2=lambda re, im: ("fp2", re, im)):
    """the JSON form of a put() argument in the golden scripts -> Python values:
    {"fp2": [re, im]} is an Fp2 (built by `fp2`), {"tuple": [...]} a tuple,
    {"dict": [[k, v], ...]} a dict"""
    if isinstance(x, dict):
        if "fp2" in x:
            return fp2(int(x["fp2"][0]), int(x["fp2"][1]))
        if "tuple" in x:
            return tuple(py_value(v, fp2) for v in x["tuple"])
        return {k: py_value(v, fp2) for k, v in x["dict"]}
    if isinstance(x, list):
        return [py_value(v, fp2) for v in x]
    return x


def _flat(vals):
    for v in vals:
        if isinstance(v, (list, tuple)) and not (isinstance(v, tuple) and v[:1] == ("fp2",)):
            yield from _flat(v)
        else:
            yield v


def encode_put(x):
    """bytes a reference transcript absorbs for put(x) (fiatshamir.py:101-138, 168-186)"""
    vals = py_value(x)
    if isinstance(vals, dict):
        vals = list(vals.items())
    elif not isinstance(vals, list):
        vals = [vals]
    if vals and type(vals[0]) is int and all(type(v) is int and 0 <= v < 1 << 64 for v in vals):
        return b"\x01" + struct.pack("<I", len(vals)) + b"".join(struct.pack("<Q", v) for v in vals)
    out = b""
    for e in _flat(vals):
        if type(e) is int:
            out += b"\x02" + struct.pack("<Q", e & ((1 << 64) - 1))
        elif isinstance(e, tuple):
            out += b"\x03" + struct.pack("<QQ", e[1], e[2])
        elif isinstance(e, str):
            out += b"\x04" + struct.pack("<I", len(e.encode())) + e.encode()
        else:
            assert e is None
            out += b"\x05"
    return out


class PyTranscript:
    def __init__(self, protocol):
        self.h = hashlib.sha256(b"TruePix," + protocol.encode() + b"," + b"binhash1,")
        self.rnum = 0

    def u64s(self, v):
        self.h.update(b"\x01" + struct.pack("<I", len(v)) + b"".join(struct.pack("<Q", x) for x in v))

    def fp2(self, re, im):
        self.h.update(b"\x03" + struct.pack("<QQ", re, im))

    def str(self, s):
        b = s.encode()
        self.h.update(b"\x04" + struct.pack("<I", len(b)) + b)

    def scalar(self):
        while True:
            self.u64s([self.rnum])
            self.rnum += 1
            v = int.from_bytes(self.h.digest(), "big") & P61
            if v < P61:
                return v

    def ext(self, label):
        self.str("ext"), self.str(label), self.str("real")
        re = self.scalar()
        self.str("ext"), self.str(label), self.str("imag")
        return re, self.scalar()


def replay_python(protocol, ops):
    t = PyTranscript(protocol)
    outs, digs = [], b""
    for op in ops:
        if op[0] == "u64s":
            t.u64s(op[1])
        elif op[0] == "fp2s":
            for re, im in op[1]:
                t.fp2(re, im)
        elif op[0] == "str":
            t.str(op[1])
        elif op[0] == "put_py":
            t.h.update(encode_put(op[1]))
        elif op[0] == "ext":
            outs += list(t.ext(op[1]))
        elif op[0] == "scalar":
            outs.append(t.scalar())
        elif op[0] == "digest":
            digs += t.h.digest()
    return np.array(outs, np.uint64), digs


def replay_lib(lib, protocol, ops, state=None):
    """(outputs, digests, state buffer) through tp_fs_*; `state` continues a given one"""
    st = state if state is not None else ctypes.create_string_buffer(lib.tp_fs_state_bytes())
    if state is None:
        assert lib.tp_fs_init(st, protocol.encode()) == 0
    outs, digs = [], b""
    re, im = ctypes.c_uint64(), ctypes.c_uint64()
    d = ctypes.create_string_buffer(32)
    for op in ops:
        if op[0] == "u64s":
            a = np.array(op[1], np.uint64)
            assert lib.tp_fs_put_u64s(st, a.ctypes.data, a.size) == 0
        elif op[0] == "fp2s":
            a = np.array(op[1], np.uint64).reshape(-1, 2)
            r, i = np.ascontiguousarray(a[:, 0]), np.ascontiguousarray(a[:, 1])
            assert lib.tp_fs_put_fp2s(st, r.ctypes.data, i.ctypes.data, r.size) == 0
        elif op[0] == "str":
            assert lib.tp_fs_put_str(st, op[1].encode()) == 0
        elif op[0] == "put_py":
            b = encode_put(op[1])
            assert lib.tp_fs_absorb(st, b, len(b)) == 0
        elif op[0] == "ext":
            assert lib.tp_fs_rand_ext(st, op[1].encode(), ctypes.byref(re), ctypes.byref(im)) == 0
            outs += [re.value, im.value]
        elif op[0] == "scalar":
            assert lib.tp_fs_rand_scalar(st, ctypes.byref(re)) == 0
            outs.append(re.value)
        elif op[0] == "digest":
            assert lib.tp_fs_digest(st, d) == 0
            digs += d.raw
    return np.array(outs, np.uint64), digs, st


# ---- VOLE-committed sumcheck round (circuitnizkvec_vole.py:396-418) ----------
HALF, THIRD = 1152921504606846976, 1537228672809129301   # 2^-1, 3^-1 mod p


def f2add(a, b): return ((a[0] + b[0]) % P61, (a[1] + b[1]) % P61)
def f2sub(a, b): return ((a[0] - b[0]) % P61, (a[1] - b[1]) % P61)
def f2mul(a, b): return ((a[0] * b[0] - a[1] * b[1]) % P61, (a[0] * b[1] + a[1] * b[0]) % P61)
def f2scale(a, k): return (a[0] * k % P61, a[1] * k % P61)


def interpolate_cubic(f0, f1, fm1, f2):
    """util.interpolate_cubic: coefficients from the values at 0, 1, -1, 2"""
    a = f2sub((0, 0), fm1)
    b = f2scale(f2add(f1, fm1), HALF)
    c = f2scale(f2add(f1, a), HALF)
    d = f2scale(f2add(f2, a), THIRD)
    c2 = f2sub(b, f0)
    c3 = f2scale(f2sub(f2sub(d, c), c2), HALF)
    return [f0, f2sub(c, c3), c2, c3]


def vole_rounds_python(g, name):
    """Replay of a golden case (tests/golden/vole_round_golden.npz)"""
    T = PyTranscript("truepix")
    T.u64s([int(x) for x in g[name + "_prefix"]])
    u, v = g[name + "_u"], g[name + "_v"]
    idx = int(g[name + "_start"][0])
    prev = tuple(int(x) for x in g[name + "_prev0"]) if int(g[name + "_has_prev"][0]) else None
    chals, vzs = [], []
    for cl in g[name + "_claims"]:
        f = [(int(a), int(b)) for a, b in cl]
        outs = interpolate_cubic(*f)
        tags = []
        for c in outs:
            tags.append((int(v[idx, 0]), int(v[idx, 1])))
            d = f2sub(c, (int(u[idx, 0]), int(u[idx, 1])))
            idx += 1
            T.fp2(*d)
        zp1 = f2add(f2add(f2add(f2add(tags[0], tags[1]), tags[2]), tags[3]), tags[0])
        ch = T.ext("eq")
        vz = f2mul(zp1, ch) if prev is None else f2mul(f2sub(prev, zp1), ch)
        T.fp2(*vz)
        vzs.append(vz)
        r = T.ext("sc-0-%d" % len(chals))
        chals.append(r)
        prev = f2add(f2mul(f2add(f2mul(f2add(f2mul(tags[3], r), tags[2]), r), tags[1]), r), tags[0])
    return np.array(chals, np.uint64), np.array(vzs, np.uint64), prev, T.h.digest(), idx
