"""Golden proofs of the reference prover (tests/golden/prover_golden.npz), the
pickle form of its Fp2 values, and the restated proof of a frame (oracle early
rounds, restated VOLE rounds, oracle late rounds, restated closing proofs) used
to check the host side of truepix_b200.prover on the same inputs."""
from __future__ import annotations

import json
import os
import sys
import types

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
P61 = (1 << 61) - 1


def fp2_type():
    """The class the reference's proofs pickle their Fp2 values as:
    libTruePix.extfield.Fp2 with state (real, imag, p). The reference's own when
    it is importable, else a class with the same name and state."""
    try:
        from libTruePix.extfield import Fp2
        return Fp2
    except ImportError:
        pass
    if "libTruePix.extfield" not in sys.modules:
        pkg = sys.modules.setdefault("libTruePix", types.ModuleType("libTruePix"))
        mod = types.ModuleType("libTruePix.extfield")

        class Fp2:
            __slots__ = ("real", "imag", "p")

            def __init__(self, real, imag, p=P61):
                self.real, self.imag, self.p = int(real) % p, int(imag) % p, p

            def __getstate__(self):
                return (self.real, self.imag, self.p)

            def __setstate__(self, state):
                self.real, self.imag, self.p = state

            def __eq__(self, other):
                return (self.real, self.imag) == (other.real, other.imag)

        Fp2.__module__ = "libTruePix.extfield"
        Fp2.__qualname__ = "Fp2"
        mod.Fp2 = Fp2
        pkg.extfield = mod
        sys.modules["libTruePix.extfield"] = mod
    return sys.modules["libTruePix.extfield"].Fp2


def cases():
    g = np.load(os.path.join(ROOT, "tests", "golden", "prover_golden.npz"))
    for n in sorted(k[:-4] for k in g.files if k.endswith("_pix")):
        circ, copies, cs, ci, cv, pid, zk = json.loads(g[n + "_layout"].tobytes().decode())
        d = {k[len(n) + 1:]: g[k] for k in g.files if k.startswith(n + "_")}
        d.update(name=n, circ=circ, copies=copies, cs=cs, ci=ci, cv=cv, pid=pid, zk=bool(zk),
                 manifest=json.loads(g[n + "_manifest"].tobytes().decode()))
        yield d


def circuit(name):
    c = np.load(os.path.join(ROOT, "tests", "golden", "circuits.npz"))
    return c[name + "_type"], c[name + "_in0"], c[name + "_in1"]


def restated_proof(c, lib_transcript):
    """The proof of golden case c with every value computed by the oracle and the
    restatements, assembled by truepix_b200.prover.LayerTranscript."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from circuitlib import oracle_outputs
    from fp2lib import ORACLE_LIB, Fp2Lib
    from fslib import f2add, f2mul, f2sub, interpolate_cubic
    from latelib import oracle
    from layervole import closing_python
    from truepix_b200 import prover
    gt, i0, i1 = circuit(c["circ"])
    copies, cs, ci, cv = c["copies"], c["cs"], c["ci"], c["cv"]
    padded = 1 << max(1, (copies - 1).bit_length())
    nb, n, W = padded.bit_length() - 1, 9, 512
    outs = oracle_outputs(c["pix"], copies, padded, cs, W, ci, cv, gt, i0, i1)
    t = lib_transcript
    z1, z2 = t.io_prefix(outs, padded * W, prover.commit_binding(c["manifest"]), 9, nb)
    # the restated round loop needs the transcript's running state: replay it in Python
    from fslib import PyTranscript, encode_put
    T = PyTranscript("truepix")
    T.h.update(encode_put(c["pid"]) + encode_put(None) + encode_put(["private_input_omitted", padded * W]))
    import struct
    T.h.update(b"\x01" + struct.pack("<I", outs.size) + outs.tobytes())
    b = prover.commit_binding(c["manifest"])
    T.h.update(encode_put(b))
    assert [T.ext("z1-%d" % i) for i in range(9)] == z1
    assert [T.ext("z2-%d" % i) for i in range(nb)] == z2
    ol = Fp2Lib(ORACLE_LIB, "oracle_fp2_")
    zr, zi = (np.ascontiguousarray([p[k] for p in z1], np.uint64) for k in (0, 1))
    wr, wi = ol.compute_beta(zr, zi, (1, 0))
    zg = [(int(a), int(b)) for a, b in zip(wr[:gt.size], wi[:gt.size])]
    zr2, zi2 = (np.ascontiguousarray([p[k] for p in z2], np.uint64) for k in (0, 1))
    br, bi = ol.compute_beta(zr2, zi2, (1, 0))
    V = np.zeros((W, padded), np.uint64)
    rows = c["pix"].reshape(copies, cs).astype(np.uint64)
    V[:cs, :copies] = rows.T
    if ci >= 0:
        V[ci, :copies] = cv
    vr = np.ascontiguousarray(V.reshape(-1))
    vi = np.zeros_like(vr)
    z1r = np.ascontiguousarray([p[0] for p in zg], np.uint64)
    z1i = np.ascontiguousarray([p[1] for p in zg], np.uint64)
    g32 = [np.ascontiguousarray(a, np.int32) for a in (gt, i0, i1)]
    h = ol.early_create(*g32, z1r, z1i, padded, W, vr, vi, np.ascontiguousarray(br), np.ascontiguousarray(bi))
    u = [(int(a), int(b)) for a, b in c["u"]]
    v = [(int(a), int(b)) for a, b in c["v"]]
    idx, prev = 0, None
    v_elem, out_elem = [(0, 0)] * 4, [(0, 0)] * 4
    early, late_vals, chals = [], [], []
    late = None
    for rd in range(nb + 2 * n):
        if rd < nb:
            rc, o8 = ol.early_claim(h)
            assert rc == 0
            cf = interpolate_cubic(*[(int(o8[2 * k]), int(o8[2 * k + 1])) for k in range(4)])
        else:
            if late is None:
                rc, wre, wim, beta = ol.early_finish(h, W)
                assert rc == 0
                ol.early_destroy(h)
                late = oracle.LateRounds([(int(a), int(b)) for a, b in zip(wre, wim)],
                                         (int(beta[0]), int(beta[1])), zg,
                                         tuple([int(x) for x in a] for a in (gt, i0, i1)), n)
            cf = late.coefs()
        tags, row = [], []
        for k, x in enumerate(cf):
            tags.append(v[idx])
            d = f2sub(x, u[idx])
            idx += 1
            T.fp2(*d)
            row.append(d)
            v_elem[k] = f2add(v_elem[k], tags[-1])
            out_elem[k] = f2add(out_elem[k], x)
        now = tags[0]
        for tt in tags:
            now = f2add(now, tt)
        e = T.ext("eq")
        vz = f2mul(now, e) if prev is None else f2mul(f2sub(prev, now), e)
        T.fp2(*vz)
        row.append(vz)
        r = T.ext("sc-0-%d" % rd)
        chals.append(r)
        p = tags[-1]
        for tt in reversed(tags[:-1]):
            p = f2add(f2mul(p, r), tt)
        prev = p
        if rd < nb:
            assert ol.early_fold(h, r) == 0
            early.append(row)
        else:
            late.next_round(r)
            late_vals.append(row)
    w3, w1, w2 = chals[:nb], chals[nb:nb + n], chals[nb + n:]
    closing, point, tag, _ = closing_python(T, late.line(), prev, idx, v_elem, out_elem, u, v, w1, w2, w3, z2, zg,
                                            tuple([int(x) for x in a] for a in (gt, i0, i1)), zk=c["zk"])
    t.record(early, late_vals, closing, point, tag, zk=c["zk"])
    return T.h.digest()
