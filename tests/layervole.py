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
