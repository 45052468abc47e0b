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
