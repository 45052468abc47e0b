"""Golden output vectors of the TruePix circuits, made by the reference's own
circuit evaluator (TruePix-main/libTruePix/arithcircuitbuilder.py
ArithCircuitBuilder over the gate classes of gateprover.py / arithcircuit.py).

For each case: the frame bytes, the layout (copies, padded copies, copy size,
wires, constant wire and value), the gate table (native type index, in0, in1)
and the output vector the prover puts into its transcript
(circuitnizkvec_vole.py:351-355): the per-copy outputs, each padded to
2^ceil(log2 gates), concatenated, padded with zeros to the padded copy count.
Cases: the four circuits of tests/golden/circuits.npz on small frames, random
gate tables of every non-multiplexer type with a large constant, one gate, one
copy.

Run here (needs the reference checkout):  python tests/golden/gen_circuit_golden.py
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.path.join(os.environ.get("TRUEPIX_REF", "/root/reference"), "TruePix-main")
P61 = (1 << 61) - 1


def reference_outputs(pix, copies, padded, cs, n_wires, const_idx, const_val, gt, i0, i1):
    sys.path.insert(0, REF)
    from libTruePix.defs import Defs
    import libTruePix.gateprover as gp
    from libTruePix.arithcircuitbuilder import ArithCircuitBuilder
    assert Defs.prime == P61
    by_idx = {}
    for name in dir(gp):
        c = getattr(gp, name)
        if isinstance(c, type) and getattr(c, "gate_type_idx", None) is not None and c is not gp.MuxGateProver:
            by_idx[c.gate_type_idx] = c
    typev = [by_idx[int(t)] for t in gt]
    b = ArithCircuitBuilder(copies, n_wires, [[int(x) for x in i0]], [[int(x) for x in i1]], [typev])
    inputs = []
    for c in range(copies):
        row = [int(x) for x in pix[c * cs:(c + 1) * cs]] + [0] * (n_wires - cs)
        if const_idx >= 0:
            row[const_idx] = const_val
        inputs.append(row)
    (ckt_outputs, _) = b.run(inputs)
    outvals = [int(v) for copy in ckt_outputs for v in copy]
    n_out_bits = (len(gt) - 1).bit_length()
    outvals += [0] * ((padded << n_out_bits) - len(outvals))
    return np.array(outvals, dtype=np.uint64)


def cases():
    c = np.load(os.path.join(HERE, "circuits.npz"))
    rng = np.random.default_rng(424242)
    out = []
    layout = {"gray": (384, 384, 128), "inv": (384, 384, 255), "mask": (384, -1, 0), "Crop": (385, 385, 128)}
    for name, copies, padded in (("gray", 5, 8), ("inv", 6, 8), ("mask", 3, 4), ("Crop", 7, 8)):
        cs, ci, cv = layout[name]
        pix = rng.integers(0, 256, size=copies * cs, dtype=np.uint8)
        out.append((name, pix, copies, padded, cs, 512, ci, cv, c[name + "_type"], c[name + "_in0"],
                    c[name + "_in1"]))
    types = np.array([0, 1, 2, 5, 6, 7, 8, 9, 10, 11, 12], np.int32)
    for k, (n_gates, copies, padded, cs, n_wires, ci, cv) in enumerate(
            [(100, 3, 4, 300, 512, 400, P61 - 5), (384, 4, 4, 384, 512, 384, 1 << 60),
             (1, 1, 1, 16, 32, -1, 0), (33, 2, 2, 40, 64, 63, 7)]):
        pix = rng.integers(0, 256, size=copies * cs, dtype=np.uint8)
        gt = rng.choice(types, size=n_gates).astype(np.int32)
        i0 = rng.integers(0, n_wires, size=n_gates, dtype=np.int32)
        i1 = rng.integers(0, n_wires, size=n_gates, dtype=np.int32)
        if ci >= 0:
            i1[: n_gates // 4] = ci   # some gates read the constant
        out.append(("random%d" % k, pix, copies, padded, cs, n_wires, ci, cv, gt, i0, i1))
    return out


def main():
    arrays = {}
    for (name, pix, copies, padded, cs, n_wires, ci, cv, gt, i0, i1) in cases():
        arrays[name + "_pix"] = pix
        arrays[name + "_layout"] = np.array(json.dumps([copies, padded, cs, n_wires, ci, str(cv)]).encode(), "S")
        arrays[name + "_gates"] = np.stack([gt, i0, i1]).astype(np.int32)
        arrays[name + "_out"] = reference_outputs(pix, copies, padded, cs, n_wires, ci, cv, gt, i0, i1)
    np.savez_compressed(os.path.join(HERE, "circuit_outputs_golden.npz"), **arrays)
    print("wrote", len(arrays) // 4, "cases")


if __name__ == "__main__":
    main()
