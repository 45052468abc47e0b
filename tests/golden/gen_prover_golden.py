"""Golden proofs of the reference prover itself: CircuitProverNIZK.run
(TruePix-main/libTruePix/circuitnizkvec_vole.py:265-500, and its
zero-knowledge variant circuitnizkvec_vole_ZK.py:293-520, TruePix's default) on
small frames of the gray, inv and crop circuits, with a fixed process id, a VOLE prover file in the
reference's binary format (ExtVOLEGen.py:25-50, 130-186) holding seeded
correlations, and an Orion commitment manifest (fp2_link.py:426-504) with fixed
roots.

Per case: the frame bytes and layout, pid, the correlations u, v, the manifest,
the proof bytes run() returns (FiatShamir.to_string()), and, for checks that
cannot import the reference, every Fp2 value of the transcript's trans queue in
order (with each entry's length), the input point, its tag and the transcript's
final digest.

Run here (needs the reference checkout):  python tests/golden/gen_prover_golden.py
"""
from __future__ import annotations

import json
import os
import struct
import sys
import tempfile
import warnings

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.path.join(os.environ.get("TRUEPIX_REF", "/root/reference"), "TruePix-main")
P61 = (1 << 61) - 1
LAYOUT_ID = "copy-major-384-const128-pad512-v1"

# name, circuit, copies, copy_size, const_idx, const_val, pid, zk manifest, zero-knowledge prover
CASES = [("gray4", "gray", 4, 384, 384, 128, 4242, True, False),
         ("inv7", "inv", 7, 384, 384, 255, 777, False, False),
         ("crop3", "Crop", 3, 385, 385, 128, 31337, True, False),
         ("gray4zk", "gray", 4, 384, 384, 128, 5151, True, True),
         ("crop5zk", "Crop", 5, 385, 385, 128, 2718, True, True)]


def run_case(rng, circ, copies, cs, ci, cv, pid, zk, zk_prover, workdir):
    sys.path.insert(0, REF)
    warnings.simplefilter("ignore", SyntaxWarning)
    if zk_prover:      # TruePix's default mode: circuitnizkvec_vole_ZK.py
        import libTruePix.circuitnizkvec_vole_ZK as cnv
    else:
        import libTruePix.circuitnizkvec_vole as cnv
    import libTruePix.gateprover as gp
    import libTruePix.util as util
    from libTruePix.extfield import Fp2
    by_idx = {}
    for name in dir(gp):
        k = getattr(gp, name)
        if isinstance(k, type) and getattr(k, "gate_type_idx", None) is not None and k is not gp.MuxGateProver:
            by_idx[k.gate_type_idx] = k
    c = np.load(os.path.join(HERE, "circuits.npz"))
    gt, i0, i1 = c[circ + "_type"], c[circ + "_in0"], c[circ + "_in1"]
    pix = rng.integers(0, 256, size=copies * cs, dtype=np.uint8)
    if circ == "Crop":
        pix.reshape(copies, cs)[:, 384] = rng.integers(0, 2, size=copies)   # the crop flag byte
    inputs = [[int(x) for x in pix[i * cs:(i + 1) * cs]] + [cv] for i in range(copies)]
    n_vole = 200
    u = rng.integers(0, P61, size=(n_vole, 2), dtype=np.uint64)
    v = rng.integers(0, P61, size=(n_vole, 2), dtype=np.uint64)
    padded = 1 << max(1, (copies - 1).bit_length())
    manifest = dict(protocol="truepix", layout=LAYOUT_ID, zk=zk, copies=copies, padded_copies=padded,
                    copy_size=cs, padded_copy_size=512, const_idx=ci, const_val=cv, n=padded * 512,
                    lg_n=(padded * 512).bit_length() - 1, masked_root=bytes(rng.integers(0, 256, 32, np.uint8)).hex(),
                    mask_root=bytes(rng.integers(0, 256, 32, np.uint8)).hex() if zk else "")
    cwd = os.getcwd()
    os.chdir(workdir)
    try:
        with open("vole_ext_prover_%d.json" % pid, "wb") as fh:
            fh.write(struct.pack("<4sIIIIQ", b"EVOL", 1, 1, 1, n_vole, P61))
            for a in (u[:, 0], u[:, 1], v[:, 0], v[:, 1]):
                fh.write(np.ascontiguousarray(a).tobytes())
        with open("orion_commit.json", "w") as fh:
            json.dump(manifest, fh)
        os.environ["TRUEPIX_ORION_COMMIT_FILE"] = os.path.join(workdir, "orion_commit.json")
        cnv.os.getpid = lambda: pid
        prv = cnv.CircuitProverNIZK(copies, len(inputs[0]), [[int(x) for x in i0]], [[int(x) for x in i1]],
                                    [[by_idx[int(t)] for t in gt]])
        proof = prv.run(inputs)
    finally:
        os.chdir(cwd)
    fp2s, lens = [], []
    for item in prv.fs.trans:
        vals = [x for x in util.flatten(item) if isinstance(x, Fp2)]
        fp2s += vals
        lens.append(len(vals))
    pk = lambda xs: np.array([[int(x.real), int(x.imag)] for x in xs], np.uint64).reshape(-1, 2)
    return dict(pix=pix, layout=np.array(json.dumps([circ, copies, cs, ci, cv, pid, int(zk_prover)]).encode(), "S"),
                u=u, v=v, manifest=np.array(json.dumps(manifest).encode(), "S"),
                proof=np.frombuffer(proof, np.uint8), trans_fp2=pk(fp2s), trans_lens=np.array(lens, np.int32),
                point=pk(prv.final_input_point), tag=pk([prv.final_input_tag]),
                digest=np.frombuffer(prv.fs.hash.digest(), np.uint8))


def main():
    rng = np.random.default_rng(20261204)
    arrays = {}
    with tempfile.TemporaryDirectory() as workdir:
        for (name, circ, copies, cs, ci, cv, pid, zk, zk_prover) in CASES:
            for k, val in run_case(rng, circ, copies, cs, ci, cv, pid, zk, zk_prover, workdir).items():
                arrays[name + "_" + k] = val
    np.savez_compressed(os.path.join(HERE, "prover_golden.npz"), **arrays)
    print("wrote", len(CASES), "cases")


if __name__ == "__main__":
    main()
