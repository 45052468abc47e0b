"""Golden vectors of the input layer's whole VOLE-committed proof -- early and
late rounds and the layer's closing proofs -- made by the reference prover's
own code in the order of its loop (TruePix-main/libTruePix/circuitnizkvec_vole.py
:386-500): LayerProver (layerprover.py) for the round polynomials and the line;
CircuitProverNIZK's create_pok_temp, create_eq_proof, create_final_prod_pok,
create_pok_final, create_input_value_proof and _challenge, and
CircuitVerifier.eval_mlext, called on a prover object that carries only the
state they read (commitment, transcript, gate tables); GateFunctionsPC for the
committed gate values; ExtVOLECommit for the commitments; FiatShamir for the
transcript.

Per case: gates, inputs, z1, z2, the per-gate weights, correlations u, v and the
first one used, the transcript prefix; per round the coefficients, the values d
put, the equality value, the challenge; between the phases the wires, beta, the
previous value and the running tag / coefficient sums; after the late rounds
the line coefficients, the previous value, the sums, the correlations used and
the transcript digest; then the closing proof's Fp2 values in the order they are
put, the input point, its tag, the correlations used and the final digest.

Run here (needs the reference checkout):  python tests/golden/gen_layer_vole_golden.py
"""
from __future__ import annotations

import json
import os
import sys
import warnings

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.path.join(os.environ.get("TRUEPIX_REF", "/root/reference"), "TruePix-main")
P61 = (1 << 61) - 1


def run_case(rng, n_in_bits, n_copies, gt, i0, i1, inputs, start):
    sys.path.insert(0, REF)
    warnings.simplefilter("ignore", SyntaxWarning)
    import libTruePix.util as util
    from libTruePix.ExtVOLECommit import ExtVOLECommit
    from libTruePix.extfield import Fp2
    from libTruePix.fiatshamir import FiatShamir
    from libTruePix.circuitprover import _DummyCircuitProver
    from libTruePix.layerprover import LayerProver
    import libTruePix.gateprover as gp
    by_idx = {}
    for name in dir(gp):
        c = getattr(gp, name)
        if isinstance(c, type) and getattr(c, "gate_type_idx", None) is not None and c is not gp.MuxGateProver:
            by_idx[c.gate_type_idx] = c
    F = lambda: Fp2(int(rng.integers(0, P61)), int(rng.integers(0, P61)), P61)
    n_out_bits = max(1, (len(gt) - 1).bit_length())
    circuit = _DummyCircuitProver(n_copies)
    nb = circuit.nCopyBits
    n_rounds = nb + 2 * n_in_bits
    L = LayerProver(n_in_bits, circuit, [int(x) for x in i0], [int(x) for x in i1], [by_idx[int(t)] for t in gt])
    L.set_inputs([[int(x) for x in row] for row in inputs])
    z1 = [F() for _ in range(n_out_bits)]
    z2 = [F() for _ in range(nb)]
    L.set_z(z1, z2, None, None, True)
    zg = [g.accum_z1 for g in L.gates]

    n_vole = start + 4 * nb + 3 * 2 * n_in_bits + (n_in_bits + 2) + 1
    u = rng.integers(0, P61, size=(n_vole, 2), dtype=np.uint64)
    v = rng.integers(0, P61, size=(n_vole, 2), dtype=np.uint64)
    com = ExtVOLECommit(P61)
    com.u_lists = [[Fp2(int(a), int(b), P61) for a, b in u]]
    com.v_lists = [[Fp2(int(a), int(b), P61) for a, b in v]]
    com.numVOLE = start
    com.VOLEindex = n_vole - start
    prefix = [int(x) for x in rng.integers(0, P61, size=5, dtype=np.uint64)]
    fs = FiatShamir(P61, protocol="truepix")
    fs.put(prefix)

    from libTruePix.circuitnizkvec_vole import CircuitProverNIZK
    from libTruePix.gateprover_vole import GateFunctionsPC
    from libTruePix.extfield import serialize_point
    prv = CircuitProverNIZK.__new__(CircuitProverNIZK)      # the state its proof methods read
    prv.com, prv.fs, prv.v_elem, prv.out_elem, prv.com_q_a, prv.tV_a = com, fs, [], [], None, None
    prv.layInBits, prv.layOutBits, prv.nCopyBits = [n_in_bits], [n_out_bits], nb
    prv.in0vv, prv.in1vv, prv.muxvv = [[int(x) for x in i0]], [[int(x) for x in i1]], None
    prv.typvv = [[by_idx[int(t)] for t in gt]]

    lay = 0
    prev = None
    rec = dict(coefs=[], d=[], vz=[], chal=[])
    mid = {}
    w1, w2, w3 = [], [], []
    for rd in range(n_rounds):
        L.compute_outputs()
        outs = list(L.output)
        mark = len(fs.trans)
        rvals = prv.create_pok_temp(outs)
        rec["d"].extend(x[0] for x in list(fs.trans)[mark:])
        zp1 = (sum(rvals) + rvals[0]) % P61
        prv.create_eq_proof(prev, zp1)
        rec["vz"].append(fs.trans[-1][0])
        nrand = prv._challenge("sc-%d-%d" % (lay, rd))
        L.next_round(nrand)
        prev = util.horner_eval(rvals, nrand)
        rec["coefs"].extend(outs)
        rec["chal"].append(nrand)
        (w3 if rd < nb else w1 if rd < nb + n_in_bits else w2).append(nrand)
        if rd == nb - 1:
            mid = dict(wires=list(L.compute_v_final.inputs), beta=[L.compute_beta.prevPassValue], prev_mid=[prev],
                       v_elem_mid=list(prv.v_elem) + [0] * (4 - len(prv.v_elem)),
                       out_elem_mid=list(prv.out_elem) + [0] * (4 - len(prv.out_elem)), used_mid=[com.numVOLE])
    L.compute_outputs()
    final = list(L.output)
    v_elem, out_elem = list(prv.v_elem), list(prv.out_elem)
    late_end = dict(prev=[prev], used=np.array([com.numVOLE], np.int64),
                    digest=np.frombuffer(fs.hash.digest(), np.uint8))

    # the layer's closing proofs, circuitnizkvec_vole.py:433-500 (one layer: project_line)
    mark = len(fs.trans)
    (outs_rvals, pr_rvals) = prv.create_final_prod_pok(final)
    (mlext_evals, mlx_z2) = prv.eval_mlext(lay, z1, z2, w1, w2, w3, None, None)
    tV = 0
    for (idx, elm) in enumerate(mlext_evals):
        tV += elm * GateFunctionsPC[idx](pr_rvals[0], pr_rvals[1], pr_rvals[2], None)
        tV %= P61
    tV = tV * mlx_z2 % P61
    prv.create_eq_proof(prev, tV)
    tau = prv._challenge("tau-%d" % lay)
    tag = util.horner_eval(outs_rvals, tau)
    zz1 = [(e1 + (e2 - e1) * tau) % P61 for (e1, e2) in zip(w1, w2)]
    prv.create_pok_final()
    point = list(zz1) + list(w3)
    fs.put(["gkr_input_point", serialize_point(point)])
    prv.create_input_value_proof(tag, None)
    closing = []
    for item in list(fs.trans)[mark:]:
        for x in util.flatten(item):
            if isinstance(x, Fp2):
                closing.append(x)

    def f2(xs):
        return np.array([[int(x.real), int(x.imag)] if hasattr(x, "real") and not isinstance(x, int) else [int(x), 0]
                         for x in xs], np.uint64).reshape(-1, 2)
    out = {k: f2(vv) for k, vv in rec.items()}
    out.update({k: (f2(vv) if k != "used_mid" else np.array(vv, np.int64)) for k, vv in mid.items()})
    out.update(z1=f2(z1), z2=f2(z2), zg=f2(zg), final=f2(final), prev=f2(late_end["prev"]),
               v_elem=f2(v_elem + [0] * (4 - len(v_elem))), out_elem=f2(out_elem + [0] * (4 - len(out_elem))),
               u=u, v=v, start=np.array([start], np.int64), prefix=np.array(prefix, np.uint64),
               used=late_end["used"], digest=late_end["digest"],
               closing=f2(closing), point=f2(point), tau=f2([tau]), tag=f2([tag]),
               used_closed=np.array([com.numVOLE], np.int64),
               digest_closed=np.frombuffer(fs.hash.digest(), np.uint8))
    return out


def main():
    c = np.load(os.path.join(HERE, "circuits.npz"))
    rng = np.random.default_rng(9090)
    arrays = {}
    inputs = rng.integers(0, 256, size=(4, 512)).astype(np.uint64)
    inputs[:, 384] = 128
    inputs[:, 385:] = 0
    types = np.array([0, 1, 2, 5, 6, 7, 8, 9, 10, 11, 12], np.int32)
    gt_r = rng.choice(types, size=20).astype(np.int32)
    cases = [("gray", 9, 4, c["gray_type"], c["gray_in0"], c["gray_in1"], inputs, 11),
             ("random", 5, 8, gt_r, rng.integers(0, 32, size=20).astype(np.int32),
              rng.integers(0, 32, size=20).astype(np.int32),
              rng.integers(0, P61, size=(8, 32), dtype=np.uint64), 3)]
    for (name, n_in_bits, n_copies, gt, i0, i1, inp, start) in cases:
        r = run_case(rng, n_in_bits, n_copies, gt, i0, i1, inp, start)
        arrays[name + "_shape"] = np.array(json.dumps([n_in_bits, n_copies]).encode(), "S")
        arrays[name + "_gates"] = np.stack([gt, i0, i1]).astype(np.int32)
        arrays[name + "_inputs"] = np.ascontiguousarray(inp, np.uint64)
        for k, vv in r.items():
            arrays[name + "_" + k] = vv
    np.savez_compressed(os.path.join(HERE, "layer_vole_golden.npz"), **arrays)
    print("wrote", len(cases), "cases")


if __name__ == "__main__":
    main()
