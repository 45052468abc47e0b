"""Golden Orion opening proofs made by the reference's own program
linearPC_multi_prove (TruePix-main/Orion/Orion_nonzk/examples/
multivariate_PC_test_prove.cpp:127-190 with src/VPD/linearPC.cpp:426-640
tensor_product_protocol, src/truepix/orion_fs.cpp transcript,
src/truepix/orion_proof.cpp:67-95 file format), built from its sources by
`make -C oracle ref` into oracle/_ref/linearPC_multi_prove and run on a frame's
input.txt, commitment manifest and GKR point file in a scratch directory.

The program's in-process EC(y1) self-check runs an external `./fft_gkr` only for
timing and proof-size statistics (src/VPD/vpd_verifier.cpp:80-90: it reads back
three numbers and adds them to its counters); the scratch directory holds a
stand-in that writes zeros there. Nothing it writes reaches the proof file. The
reference's self-check needs frames of 64 copies or more (smaller ones stop on
its FRI asserts).

The zero-knowledge case runs the Orion_zk tree's program (TruePix's default),
which opens the masked polynomial and the mask from the seed file's mask
(orion_proof_masked.bin with use_group1 = 1, orion_proof_mask.bin with 0).

Per case (and per polynomial of the zero-knowledge case, the mask's fields
prefixed mask_): the frame bytes and layout, the GKR point, the proof's SHA-256
and size, and the fields the CPU tests read: the header, the answer, both roots,
the query indices, the combined message, and three queried columns with the
combined codeword's entries at them.

Run here (needs the reference checkout and `make -C oracle ref`):
    python tests/golden/gen_opening_golden.py
"""
from __future__ import annotations

import hashlib
import json
import os
import struct
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
PROVE = os.path.join(ROOT, "oracle", "_ref", "linearPC_multi_prove")
PROVE_ZK = os.path.join(ROOT, "oracle", "_ref", "linearPC_multi_prove_zk")
P61 = (1 << 61) - 1
LAYOUT_ID = "copy-major-384-const128-pad512-v1"

# name, copies, copy_size, const_idx, const_val, zero-knowledge (mask seed) or None
CASES = [("gray64", 64, 384, 384, 128, None), ("crop100", 100, 385, 385, 128, None),
         ("gray80zk", 80, 384, 384, 128, 0x1234ABCD5678EF01)]


def parse(proof: bytes) -> dict:
    """orion_proof.cpp:67-95"""
    assert proof[:8] == b"ORIONPV1"
    version, use_group1, N, column_size, msg_len, cw_len, qc = struct.unpack_from("<IIQQQQI", proof, 8)
    off = 8 + struct.calcsize("<IIQQQQI")
    el = lambda o, n: np.frombuffer(proof, np.uint64, count=2 * n, offset=o).reshape(n, 2)   # (img, real)
    answer = el(off, 1); off += 16
    com_root = proof[off:off + 32]; off += 32
    comb_root = proof[off:off + 32]; off += 32
    col_q = np.frombuffer(proof, np.int64, count=qc, offset=off); off += 8 * qc
    cols = el(off, qc * column_size); off += 16 * qc * column_size
    combined = el(off, cw_len); off += 16 * cw_len
    message = el(off, msg_len); off += 16 * msg_len
    sparse = []
    for _ in range(2):
        (n,) = struct.unpack_from("<Q", proof, off)
        off += 8 + n * 36
        sparse.append(n)
    assert off == len(proof)
    return dict(header=np.array([version, use_group1, N, column_size, msg_len, cw_len, qc], np.int64),
                answer=answer, com_root=np.frombuffer(com_root, np.uint8), comb_root=np.frombuffer(comb_root, np.uint8),
                col_q=col_q, cols=cols.reshape(qc, column_size, 2), combined=combined, message=message,
                sparse=np.array(sparse, np.int64))


def fields(proof: bytes) -> dict:
    f = parse(proof)
    q3 = [0, len(f["col_q"]) // 2, len(f["col_q"]) - 1]
    return dict(sha256=np.frombuffer(hashlib.sha256(proof).digest(), np.uint8), size=np.array([len(proof)]),
                header=f["header"], answer=f["answer"], com_root=f["com_root"], comb_root=f["comb_root"],
                col_q=f["col_q"], message=f["message"], cols3=f["cols"][q3],
                combined3=f["combined"][f["col_q"][q3]], sparse=f["sparse"])


def run_case(rng, copies, cs, ci, cv, seed):
    pix = rng.integers(0, 256, size=copies * cs, dtype=np.uint8)
    padded = 1 << max(1, (copies - 1).bit_length())
    n = padded * 512
    lg = n.bit_length() - 1
    point = rng.integers(0, P61, size=(lg, 2), dtype=np.uint64)
    with tempfile.TemporaryDirectory() as d:
        rows = pix.reshape(copies, cs)
        with open(os.path.join(d, "input.txt"), "w") as fh:
            fh.write("\n".join(" ".join(str(int(x)) for x in row) for row in rows) + "\n")
        with open(os.path.join(d, "gkr_point_prover.txt"), "w") as fh:
            fh.write("%d\n" % lg + "".join("%d %d\n" % (a, b) for a, b in point))
        with open(os.path.join(d, "orion_commit.json"), "w") as fh:
            json.dump(dict(protocol="truepix", layout=LAYOUT_ID, zk=seed is not None, copies=copies,
                           padded_copies=padded, copy_size=cs, padded_copy_size=512, const_idx=ci, const_val=cv,
                           n=n, lg_n=lg, masked_root="00" * 32, mask_root="00" * 32 if seed is not None else ""), fh)
        if seed is not None:
            with open(os.path.join(d, "orion_mask_seed.txt"), "w") as fh:
                fh.write("%d\n" % seed)
        stub = os.path.join(d, "fft_gkr")
        with open(stub, "w") as fh:
            fh.write('#!/bin/sh\necho "0 0 0" > "$2"\n')
        os.chmod(stub, 0o755)
        env = dict(os.environ, TRUEPIX_PROTOCOL="truepix", TRUEPIX_COPY_SIZE=str(cs), TRUEPIX_CONST_IDX=str(ci),
                   TRUEPIX_CONST_VAL=str(cv), TRUEPIX_GKR_POINT_FILE=os.path.join(d, "gkr_point_prover.txt"))
        env.pop("TRUEPIX_ORION_MODE", None)
        env.pop("TRUEPIX_ORION_PROOF_FILE", None)
        prog = PROVE if seed is None else PROVE_ZK
        r = subprocess.run([prog, str(copies), "0"], cwd=d, env=env, capture_output=True, text=True, timeout=600)
        names = ["orion_proof.bin"] if seed is None else ["orion_proof_masked.bin", "orion_proof_mask.bin"]
        proofs = []
        for nm in names:
            path = os.path.join(d, nm)
            assert os.path.exists(path), r.stdout[-3000:] + r.stderr[-2000:]
            with open(path, "rb") as fh:
                proofs.append(fh.read())
    out = dict(pix=pix, layout=np.array(json.dumps([copies, cs, ci, cv, seed]).encode(), "S"), point=point)
    for tag, proof in zip(["", "mask_"] if seed is not None else [""], proofs):
        for k, v in fields(proof).items():
            out[tag + k] = v
    return out


def main():
    rng = np.random.default_rng(8080)
    arrays = {}
    for (name, copies, cs, ci, cv, seed) in CASES:
        for k, v in run_case(rng, copies, cs, ci, cv, seed).items():
            arrays[name + "_" + k] = v
    np.savez_compressed(os.path.join(HERE, "opening_golden.npz"), **arrays)
    print("wrote", len(CASES), "cases")


if __name__ == "__main__":
    main()
