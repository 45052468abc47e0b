"""Golden vectors of the GKR input layer's whole sumcheck -- early rounds, late
rounds and the line projection -- made by the reference's own LayerProver
(TruePix-main/libTruePix/layerprover.py with gateprover.py and layercompute.py)
driven the way its own test drives it (libTruePixtests/layer.py) and the way
circuitnizkvec_vole.py:386-402 drives it, with Fp2 challenges.

For each case: gate table (native type index, in0, in1), the copies' inputs,
z1, z2, the per-gate weights the layer starts from (accum_z1), the challenges of
every round, the prover's output of every round (4 coefficients in an early
round, 3 in a late round), the final output (the n_in_bits + 1 coefficients of
the input values on the line through the two late points), and, between the
phases, the wire values and the beta value the late rounds start from.

Run here (needs the reference checkout):  python tests/golden/gen_late_golden.py
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


def run_case(rng, n_in_bits, n_copies, gt, i0, i1, inputs):
    sys.path.insert(0, REF)
    warnings.simplefilter("ignore", SyntaxWarning)
    from libTruePix.extfield import Fp2
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
    L = LayerProver(n_in_bits, circuit, [int(x) for x in i0], [int(x) for x in i1], [by_idx[int(t)] for t in gt])
    L.set_inputs([[int(x) for x in row] for row in inputs])
    z1 = [F() for _ in range(n_out_bits)]
    z2 = [F() for _ in range(circuit.nCopyBits)]
    L.set_z(z1, z2, None, None, True)
    zg = [g.accum_z1 for g in L.gates]
    n_rounds = circuit.nCopyBits + 2 * n_in_bits
    chal = [F() for _ in range(n_rounds)]
    outs = []
    wires = beta = None
    for rd in range(n_rounds):
        L.compute_outputs()
        outs.append(list(L.output))
        L.next_round(chal[rd])
        if rd == circuit.nCopyBits - 1:
            wires = list(L.compute_v_final.inputs)
            beta = L.compute_beta.prevPassValue
    L.compute_outputs()
    final = list(L.output)
    f2 = lambda xs: np.array([[int(x.real), int(x.imag)] for x in xs], np.uint64).reshape(-1, 2)
    return dict(z1=f2(z1), z2=f2(z2), zg=f2(zg), chal=f2(chal),
                early=f2([c for o in outs[:circuit.nCopyBits] for c in o]),
                late=f2([c for o in outs[circuit.nCopyBits:] for c in o]),
                final=f2(final), wires=f2(wires), beta=f2([beta]))


def cases():
    c = np.load(os.path.join(HERE, "circuits.npz"))
    rng = np.random.default_rng(777)
    out = []
    # the gray circuit (384 gates over 512 wires) on 4 copies of bytes with the constant wire
    inputs = rng.integers(0, 256, size=(4, 512)).astype(np.uint64)
    inputs[:, 384] = 128
    inputs[:, 385:] = 0
    out.append(("gray", 9, 4, c["gray_type"], c["gray_in0"], c["gray_in1"], inputs))
    # crop (multiplications by the flag wire) on 2 copies
    inputs = rng.integers(0, 256, size=(2, 512)).astype(np.uint64)
    inputs[:, 384] = rng.integers(0, 2, size=2)
    inputs[:, 385] = 128
    inputs[:, 386:] = 0
    out.append(("crop", 9, 2, c["Crop_type"], c["Crop_in0"], c["Crop_in1"], inputs))
    # random circuits of every non-multiplexer type, field-size inputs
    types = np.array([0, 1, 2, 5, 6, 7, 8, 9, 10, 11, 12], np.int32)
    for k, (n_in_bits, n_copies, n_gates) in enumerate([(4, 8, 13), (6, 4, 64), (3, 2, 5), (5, 16, 40)]):
        W = 1 << n_in_bits
        gt = rng.choice(types, size=n_gates).astype(np.int32)
        i0 = rng.integers(0, W, size=n_gates).astype(np.int32)
        i1 = rng.integers(0, W, size=n_gates).astype(np.int32)
        inputs = rng.integers(0, P61, size=(n_copies, W), dtype=np.uint64)
        out.append(("random%d" % k, n_in_bits, n_copies, gt, i0, i1, inputs))
    return out, rng


def main():
    arrays = {}
    cs, rng = cases()
    for (name, n_in_bits, n_copies, gt, i0, i1, inputs) in cs:
        r = run_case(rng, n_in_bits, n_copies, gt, i0, i1, inputs)
        arrays[name + "_shape"] = np.array(json.dumps([n_in_bits, n_copies]).encode(), "S")
        arrays[name + "_gates"] = np.stack([gt, i0, i1]).astype(np.int32)
        arrays[name + "_inputs"] = np.ascontiguousarray(inputs, np.uint64)
        for k, v in r.items():
            arrays[name + "_" + k] = v
    np.savez_compressed(os.path.join(HERE, "late_golden.npz"), **arrays)
    print("wrote", len(cs), "cases")


if __name__ == "__main__":
    main()
