"""The whole-layer VOLE golden cases (tests/golden/layer_vole_golden.npz) and
the states the late rounds start from: the transcript after the prefix and the
early rounds, replayed through the library's host transcript from the golden
values, and the VOLE state between the phases."""
from __future__ import annotations

import ctypes
import json
import os
import struct

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def cases():
    g = np.load(os.path.join(ROOT, "tests", "golden", "layer_vole_golden.npz"))
    for n in sorted(k[:-6] for k in g.files if k.endswith("_shape")):
        n_in_bits, n_copies = json.loads(g[n + "_shape"].tobytes().decode())
        d = {k[len(n) + 1:]: g[k] for k in g.files if k.startswith(n + "_")}
        d.update(name=n, n_in_bits=n_in_bits, n_copies=n_copies, nb=(n_copies - 1).bit_length())
        yield d


def early_transcript(lib, c):
    """the frame's transcript state after the prefix and the early rounds (host
    library calls), and the early challenges it drew"""
    st = ctypes.create_string_buffer(lib.tp_fs_state_bytes())
    assert lib.tp_fs_init(st, b"truepix") == 0
    pre = np.ascontiguousarray(c["prefix"], np.uint64)
    assert lib.tp_fs_put_u64s(st, pre.ctypes.data, pre.size) == 0
    re, im = ctypes.c_uint64(), ctypes.c_uint64()
    chals = []
    for rd in range(c["nb"]):
        d = np.ascontiguousarray(c["d"][4 * rd:4 * rd + 4], np.uint64)
        r, i = np.ascontiguousarray(d[:, 0]), np.ascontiguousarray(d[:, 1])
        assert lib.tp_fs_put_fp2s(st, r.ctypes.data, i.ctypes.data, 4) == 0
        assert lib.tp_fs_rand_ext(st, b"eq", ctypes.byref(re), ctypes.byref(im)) == 0
        vz = c["vz"][rd]
        r, i = np.array([vz[0]], np.uint64), np.array([vz[1]], np.uint64)
        assert lib.tp_fs_put_fp2s(st, r.ctypes.data, i.ctypes.data, 1) == 0
        assert lib.tp_fs_rand_ext(st, ("sc-0-%d" % rd).encode(), ctypes.byref(re), ctypes.byref(im)) == 0
        chals.append((re.value, im.value))
    return st, chals


def vole_state_mid(c):
    """the 160-byte VOLE state between the phases: next correlation, previous
    value, running sums of tags and coefficients"""
    b = struct.pack("<QII", int(c["used_mid"][0]), 1, 0) + struct.pack("<QQ", *[int(x) for x in c["prev_mid"][0]])
    for k in range(4):
        b += struct.pack("<QQ", *[int(x) for x in c["v_elem_mid"][k]])
    for k in range(4):
        b += struct.pack("<QQ", *[int(x) for x in c["out_elem_mid"][k]])
    assert len(b) == 160
    return b


def vole_state_fields(b):
    idx, has_prev, bad = struct.unpack_from("<QII", b, 0)
    f = lambda off: tuple(struct.unpack_from("<QQ", b, off))
    return dict(idx=idx, has_prev=has_prev, bad=bad, prev=f(16), v_elem=[f(32 + 16 * k) for k in range(4)],
                out_elem=[f(96 + 16 * k) for k in range(4)])


def closing_python(T, line, prev, idx, v_elem, out_elem, u, v, w1, w2, w3, z2, zg, gates, layer=0, zk=False):
    """The layer's closing proofs (circuitnizkvec_vole.py:433-500, one layer)
    restated on the hashlib transcript T: create_final_prod_pok on the line's
    coefficients, eval_mlext with GateFunctionsPC, the equality proof, tau, the
    input point and its tag, create_pok_final, the point put, the input value
    proof. zk: the zero-knowledge prover's product proof (circuitnizkvec_vole_ZK.py
    :188-247), with three mask commitments of 1 and their product proof.
    Returns (closing values in put order, point, tag, correlations used)."""
    from fslib import f2add, f2mul, f2sub
    import struct as _st
    n = len(line) - 1
    out = []

    def put(x):
        T.fp2(*x)
        out.append(x)

    def commit(m):
        nonlocal idx
        t, d = v[idx], f2sub(m, u[idx])
        idx += 1
        return t, d

    sval = (0, 0)
    for x in line:
        sval = f2add(sval, x)
    prod = f2mul(line[0], sval)
    v1, d1 = commit(line[0])
    v3, d3 = commit(prod)
    put(d1), put(d3)
    tags = [v1]
    rest_sum = rest_v = (0, 0)
    for x in line[1:]:
        t, d = commit(x)
        tags.append(t)
        put(d)
        rest_sum, rest_v = f2add(rest_sum, x), f2add(rest_v, t)
    c = T.ext("pok-vec")
    put(f2mul(rest_sum, c)), put(f2mul(rest_v, c))
    vsum = (0, 0)
    for t in tags:
        vsum = f2add(vsum, t)
    if zk:
        mask = [commit((1, 0)) for _ in range(3)]
        for _, d in mask:
            put(d)
    put(f2mul(v1, vsum))
    put(f2sub(f2add(f2mul(line[0], vsum), f2mul(sval, v1)), v3))
    if zk:
        (m1, _), (m2, _), (m3, _) = mask
        put(f2mul(m1, m2))
        put(f2sub(f2add(m2, m1), m3))
    pr = (v1, vsum, v3)
    one = (1, 0)

    def pc(t, x, y, xy):
        if t == 0: return xy
        if t == 1: return f2add(x, y)
        if t == 2: return f2sub(x, y)
        if t == 3: return x
        if t == 4: return y
        if t == 5: return f2sub(f2add(x, y), xy)
        if t == 6: return f2sub(f2add(x, y), f2add(xy, xy))
        if t == 7: return f2sub(one, x)
        if t == 8: return f2sub(one, xy)
        if t == 9: return f2sub(f2add(one, xy), f2add(x, y))
        if t == 10: return f2sub(f2add(one, f2add(xy, xy)), f2add(x, y))
        if t == 11: return f2sub(y, xy)
        return x

    gt, i0, i1 = gates
    tv = (0, 0)
    for g in range(len(gt)):
        e = zg[g]
        for j in range(n):
            e = f2mul(e, w1[j] if (i0[g] >> j) & 1 else f2sub(one, w1[j]))
            e = f2mul(e, w2[j] if (i1[g] >> j) & 1 else f2sub(one, w2[j]))
        tv = f2add(tv, f2mul(e, pc(gt[g], *pr)))
    mz = one
    for wk, zk in zip(w3, z2):
        mz = f2mul(mz, f2sub(f2add(f2add(f2mul(wk, zk), f2mul(wk, zk)), one), f2add(wk, zk)))
    tv = f2mul(tv, mz)
    e = T.ext("eq")
    put(f2mul(f2sub(prev, tv), e))
    tau = T.ext("tau-%d" % layer)
    tag = tags[-1]
    for t in reversed(tags[:-1]):
        tag = f2add(f2mul(tag, tau), t)
    point = [f2add(a, f2mul(f2sub(b, a), tau)) for a, b in zip(w1, w2)] + list(w3)
    osum = vs = (0, 0)
    for k in range(len(out_elem)):
        osum, vs = f2add(osum, out_elem[k]), f2add(vs, v_elem[k])
    c = T.ext("pok-final")
    put(f2mul(osum, c)), put(f2mul(vs, c))
    T.str("gkr_input_point")
    T.h.update(b"".join(b"\x02" + _st.pack("<Q", x) for p in point for x in p))
    c = T.ext("input-val")
    put(f2mul(tag, c))
    return out, point, tag, idx
