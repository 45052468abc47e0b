"""The opening's host logic against opening proofs written by the reference's
own linearPC_multi_prove programs (tests/golden/opening_golden.npz): a
restatement of the Orion transcript draws each proof's 1222 queried columns from
the point's eq tables (split as truepix_b200.opening.split_point splits the
point), and those tables reproduce the proof's answer (r1 against the combined
message) and its column checks (r0 against queried columns); the proof file
layout round trip. Host code only."""
import hashlib
import json
import os
import struct
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
P61 = (1 << 61) - 1


def f2mul(a, b):
    return ((a[0] * b[0] - a[1] * b[1]) % P61, (a[0] * b[1] + a[1] * b[0]) % P61)


def eq(coords):
    t = [(1, 0)]
    for z in coords:
        one_m = ((1 - z[0]) % P61, (-z[1]) % P61)
        t = [f2mul(x, one_m) for x in t] + [f2mul(x, z) for x in t]
    return t


class OrionTranscript:
    """restatement of truepix_orion::FsTranscript (Orion src/truepix/orion_fs.cpp:20-105):
    a 32-byte state; each absorb of up to 32 bytes replaces it by SHA-256(state ||
    bytes || zero pad to 64); draws take 8 bytes at a time from a pool
    SHA-256(state || 0x01 || 0^31), after which the state is SHA-256(state || 0x02 || 0^31)"""

    def __init__(self):
        self.state, self.pool = bytes(32), bytes(32)
        self.absorb(b"truepix/orion-fs/v1")

    def absorb(self, data):
        for off in range(0, len(data), 32):
            chunk = data[off:off + 32]
            self.state = hashlib.sha256(self.state + chunk + bytes(32 - len(chunk))).digest()
        self.used = 32

    def absorb_u64(self, x):
        self.absorb(struct.pack("<Q", x))

    def absorb_field(self, re, im):
        self.absorb(struct.pack("<Q", re))
        self.absorb(struct.pack("<Q", im))

    def squeeze_index(self, bound):
        if self.used + 8 > 32:
            self.pool = hashlib.sha256(self.state + b"\x01" + bytes(31)).digest()
            self.state = hashlib.sha256(self.state + b"\x02" + bytes(31)).digest()
            self.used = 0
        v = struct.unpack_from("<Q", self.pool, self.used)[0]
        self.used += 8
        return v % bound


def query_columns(T, cw_len, group, count):
    if group < 0:
        return [T.squeeze_index(cw_len) for _ in range(count)]
    size = (cw_len + 1) // 2 if group == 0 else cw_len // 2
    return [2 * T.squeeze_index(size) + group for _ in range(count)]


def cases():
    g = np.load(os.path.join(ROOT, "tests", "golden", "opening_golden.npz"))
    for n in sorted(k[:-4] for k in g.files if k.endswith("_pix")):
        d = {k[len(n) + 1:]: g[k] for k in g.files if k.startswith(n + "_")}
        d["name"] = n
        yield d


def dot(ws, els):
    """sum of w * e over (real, imag) weights and (img, real) elements"""
    s = (0, 0)
    for w, (im, re) in zip(ws, els):
        p = f2mul(w, (int(re), int(im)))
        s = ((s[0] + p[0]) % P61, (s[1] + p[1]) % P61)
    return s


def test_transcript_and_tables_match_reference_openings():
    """plain openings and both openings of the zero-knowledge pair (the masked
    polynomial's over the even columns, the mask's over the odd ones)"""
    from truepix_b200.opening import query_count, split_point
    n = 0
    for c in cases():
        zk = json.loads(c["layout"].tobytes().decode())[4] is not None
        for tag in (["", "mask_"] if zk else [""]):
            version, group1, N, cs, msg_len, cw_len, qc = (int(x) for x in c[tag + "header"])
            assert (version, group1, cs, qc) == (2, 0 if tag else 1, 128, query_count())
            pt = [(int(a), int(b)) for a, b in c["point"]]
            c0, c1 = split_point(pt)
            r0, r1 = eq(c0), eq(c1)
            assert len(r0) == 128 and len(r1) == msg_len
            T = OrionTranscript()
            T.absorb(b"tensor-open")
            T.absorb(c[tag + "com_root"].tobytes())
            T.absorb_u64(N)
            T.absorb_u64(group1)
            for re, im in r0 + r1:
                T.absorb_field(re, im)
            col_q = query_columns(T, cw_len, -1 if not zk else (1 if tag else 0), qc)
            np.testing.assert_array_equal(np.array(col_q), c[tag + "col_q"], err_msg=c["name"] + tag)
            im, re = (int(x) for x in c[tag + "answer"][0])
            assert dot(r1, c[tag + "message"]) == (re, im)
            for k in range(3):
                im, re = (int(x) for x in c[tag + "combined3"][k])
                assert dot(r0, c[tag + "cols3"][k]) == (re, im)
            n += 1
    assert n == 4


def test_proof_file_layout_round_trip():
    """opening_bytes writes the reference's layout: parsed back by the
    fixture generator's own reader"""
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    from gen_opening_golden import parse
    from truepix_b200.opening import opening_bytes
    rng = np.random.default_rng(3)
    cw, msg, qc = 40, 16, 5
    comb = rng.integers(0, P61, size=(cw, 2), dtype=np.uint64)
    cols = rng.integers(0, P61, size=(qc * 128, 2), dtype=np.uint64)
    b = opening_bytes(2048, msg, cw, np.array([3, 4], np.uint64), bytes(range(32)), bytes(32), [1, 2, 3, 4, 39],
                      cols, comb, ([5, 9], [b"a" * 32, b"b" * 32]), ([7], [b"c" * 32]))
    f = parse(b)
    assert list(f["header"]) == [2, 1, 2048, 128, msg, cw, qc]
    assert list(f["col_q"]) == [1, 2, 3, 4, 39] and list(f["sparse"]) == [2, 1]
    np.testing.assert_array_equal(f["message"], comb[:msg])
    np.testing.assert_array_equal(f["cols"].reshape(-1, 2), cols)


def _addrs(arrays):
    return np.array([a.ctypes.data for a in arrays], np.uint64)


def test_library_transcript_draws_single_and_lockstep():
    """the library's opening transcript (tp_orion_open_queries2 and its lockstep
    form tp_orion_open_queries_multi: SHA-256 chains hashed in the 16 and 8 lanes
    of the multi-buffer compression, in pairs, an odd one alone) against the
    restatement above: the queried columns of every group and the second batch of
    draws (the EC(y1) positions), for 1 to 25 transcripts in one call, and
    the reference's own openings drawn as a lockstep pair"""
    from truepix_b200 import native
    lib = native.gkr(require_device=False)
    rng = np.random.default_rng(11)
    N, n_r0, n_r1, cw_len, count = 128 * 16, 128, 16, 41, 37
    specs = []
    for i in range(25):
        root = rng.integers(0, 256, 32, dtype=np.uint8)
        r0 = rng.integers(0, P61, (n_r0, 2), dtype=np.uint64)
        r1 = rng.integers(0, P61, (n_r1, 2), dtype=np.uint64)
        specs.append((root, i % 2, r0, r1, (-1, 0, 1)[i % 3]))
    expect = []
    for root, g1, r0, r1, group in specs:
        T = OrionTranscript()
        T.absorb(b"tensor-open")
        T.absorb(root.tobytes())
        T.absorb_u64(N)
        T.absorb_u64(g1)
        for re, im in np.concatenate([r0, r1]).tolist():
            T.absorb_field(re, im)
        col = query_columns(T, cw_len, group, count)
        ec = [T.squeeze_index(cw_len) for _ in range(count)]
        expect.append((col, ec))
    for (root, g1, r0, r1, group), (col, ec) in zip(specs, expect):
        q, q2 = np.zeros(count, np.int64), np.zeros(count, np.int64)
        native.check(lib, lib.tp_orion_open_queries2(root.tobytes(), N, g1, r0.ctypes.data, n_r0, r1.ctypes.data,
                                                     n_r1, cw_len, group, count, q.ctypes.data, q2.ctypes.data),
                     "tp_orion_open_queries2")
        assert q.tolist() == col and q2.tolist() == ec
    for n in (1, 2, 3, 5, 8, 16, 17, 25):
        sp = specs[:n]
        qs = [np.zeros(count, np.int64) for _ in range(n)]
        q2s = [np.zeros(count, np.int64) for _ in range(n)]
        g1s = np.array([s[1] for s in sp], np.int32)
        groups = np.array([s[4] for s in sp], np.int32)
        # the pointer arrays stay referenced until the call returns
        a_root, a_r0, a_r1 = _addrs([s[0] for s in sp]), _addrs([s[2] for s in sp]), _addrs([s[3] for s in sp])
        a_q, a_q2 = _addrs(qs), _addrs(q2s)
        native.check(lib, lib.tp_orion_open_queries_multi(n, a_root.ctypes.data, N, g1s.ctypes.data, a_r0.ctypes.data,
                                                          n_r0, a_r1.ctypes.data, n_r1, cw_len, groups.ctypes.data,
                                                          count, a_q.ctypes.data, a_q2.ctypes.data),
                     "tp_orion_open_queries_multi")
        for (col, ec), q, q2 in zip(expect, qs, q2s):
            assert q.tolist() == col and q2.tolist() == ec
    # the zero-knowledge golden openings: the masked polynomial's and the mask's
    # transcripts of one proof drawn as a pair
    from truepix_b200.opening import split_point
    pairs = 0
    for c in cases():
        if json.loads(c["layout"].tobytes().decode())[4] is None:
            continue
        pt = [(int(a), int(b)) for a, b in c["point"]]
        c0, c1 = split_point(pt)
        r0 = np.array(eq(c0), np.uint64)
        r1 = np.array(eq(c1), np.uint64)
        hdr = [[int(x) for x in c[tag + "header"]] for tag in ("", "mask_")]
        assert hdr[0][2] == hdr[1][2] and hdr[0][5] == hdr[1][5]
        N, cw_len, qc = hdr[0][2], hdr[0][5], hdr[0][6]
        roots = [np.frombuffer(c[tag + "com_root"].tobytes(), np.uint8).copy() for tag in ("", "mask_")]
        qs = [np.zeros(qc, np.int64) for _ in range(2)]
        a_root, a_r0, a_r1, a_q = _addrs(roots), _addrs([r0, r0]), _addrs([r1, r1]), _addrs(qs)
        g1s, groups = np.array([1, 0], np.int32), np.array([0, 1], np.int32)
        native.check(lib, lib.tp_orion_open_queries_multi(2, a_root.ctypes.data, N, g1s.ctypes.data, a_r0.ctypes.data,
                                                          len(r0), a_r1.ctypes.data, len(r1), cw_len,
                                                          groups.ctypes.data, qc, a_q.ctypes.data, None),
                     "tp_orion_open_queries_multi")
        np.testing.assert_array_equal(qs[0], c["col_q"], err_msg=c["name"])
        np.testing.assert_array_equal(qs[1], c["mask_col_q"], err_msg=c["name"])
        pairs += 1
    assert pairs >= 1
