"""Golden vectors for the VOLE-committed sumcheck round of the reference prover
(TruePix-main/libTruePix/circuitnizkvec_vole.py:396-418 with create_pok_temp
:113-128 and create_eq_proof :220-234), built from the reference's own pieces:
util.interpolate_cubic, ExtVOLECommit.commit / est_val / est_eq, FiatShamir.put /
rand_ext and util.horner_eval, imported from the reference checkout.

Per round of a layer: the round polynomial's four coefficients are interpolated
from the claims at (0, 1, -1, 2); each is committed with the next VOLE
correlation (d = c - u put into the transcript, tag v kept); the tags' value at
0 + 1 is tied to the previous round's value by an equality proof (challenge
rand_ext("eq"), (prev - now) * challenge put; the first round of the first
layer proves the value alone, tag * challenge); the fold challenge is
rand_ext("sc-<layer>-<round>") and the next round's previous value is the tags'
polynomial at it. Seeded claims and correlations; stored in
tests/golden/vole_round_golden.npz.

Run here (needs the reference checkout):
    python tests/golden/gen_vole_round_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.path.join(os.environ.get("TRUEPIX_REF", "/root/reference"), "TruePix-main")
P61 = (1 << 61) - 1
CASES = [("r3", 3, 1, False), ("r14", 14, 2, False), ("r11_prev", 11, 3, True)]   # (name, rounds, seed, has_prev)


def run(rounds, seed, has_prev):
    sys.path.insert(0, REF)
    import libTruePix.util as util
    from libTruePix.ExtVOLECommit import ExtVOLECommit
    from libTruePix.extfield import Fp2
    from libTruePix.fiatshamir import FiatShamir
    rng = np.random.default_rng(seed)
    r = lambda *shape: rng.integers(0, P61, size=shape, dtype=np.uint64)
    claims = r(rounds, 4, 2)
    n_vole = 4 * rounds + 5
    u, v = r(n_vole, 2), r(n_vole, 2)
    start = 5                                       # correlations already used earlier in the proof
    prefix = [int(x) for x in r(3)]
    prev0 = r(2)
    fs = FiatShamir(P61, protocol="truepix")
    fs.put(prefix)
    com = ExtVOLECommit(P61)
    com.u_lists = [[Fp2(int(a), int(b), P61) for a, b in u]]
    com.v_lists = [[Fp2(int(a), int(b), P61) for a, b in v]]
    com.numVOLE = start
    com.VOLEindex = n_vole - start
    prev = Fp2(int(prev0[0]), int(prev0[1]), P61) if has_prev else None
    v_elem = [Fp2(0, 0, P61)] * 4
    out_elem = [Fp2(0, 0, P61)] * 4
    chals, vzs = [], []
    for rd in range(rounds):
        f = [Fp2(int(claims[rd, k, 0]), int(claims[rd, k, 1]), P61) for k in range(4)]
        outs = util.interpolate_cubic(f)
        rvals = []
        for num, val in enumerate(outs):
            v_m, d_m = com.commit(val)
            rvals.append(v_m)
            fs.put(d_m)
            v_elem[num] = v_elem[num] + v_m
            out_elem[num] = out_elem[num] + val
        zp1 = (sum(rvals) + rvals[0]) % P61
        chal = fs.rand_ext("eq")
        v_z = com.est_val(zp1, chal) if prev is None else com.est_eq(prev, zp1, chal)
        fs.put(v_z)
        vzs.append([int(v_z.real), int(v_z.imag)])
        nrand = fs.rand_ext("sc-0-%d" % rd)
        chals.append([int(nrand.real), int(nrand.imag)])
        prev = util.horner_eval(rvals, nrand)
    pk = lambda xs: np.array([[int(x.real), int(x.imag)] for x in xs], np.uint64)
    return dict(claims=claims, u=u, v=v, start=np.array([start]), prefix=np.array(prefix, np.uint64),
                prev0=prev0, has_prev=np.array([int(has_prev)]), chals=np.array(chals, np.uint64),
                vzs=np.array(vzs, np.uint64), prev=pk([prev]), v_elem=pk(v_elem), out_elem=pk(out_elem),
                digest=np.frombuffer(fs.hash.digest(), np.uint8), used=np.array([com.numVOLE]))


def main():
    out = {}
    for name, rounds, seed, has_prev in CASES:
        for k, val in run(rounds, seed, has_prev).items():
            out["%s_%s" % (name, k)] = val
    np.savez_compressed(os.path.join(HERE, "vole_round_golden.npz"), **out)
    print("wrote", len(out), "arrays")


if __name__ == "__main__":
    main()
