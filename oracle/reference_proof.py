"""The reference implementation's CPU work for one proved frame, for the CPU
baseline and the reference arm of bench.py (test infrastructure: it measures the
reference, it is not the product path).

One frame of TruePix's prover phase with the plain (-z 2) prover, as
TruePix-main/run_truepix_prover.py:218-421 runs it, and the commit phase before
it (run_truepix_signer.py:29-41):

  commit   the reference's Orion commit() (oracle/_ref/liborion_ref.so, built
           from TruePix-main/Orion/Orion_nonzk's sources by oracle/Makefile)
  IO       circuit outputs (oracle_circuit_outputs, the C restatement of the
           reference evaluator), the transcript's puts and draws with hashlib as
           libTruePix/fiatshamir.py does them (tests/fslib.py PyTranscript)
  GKR      the early rounds in the reference's own native_fp2.cpp
           (oracle/_ref/libnative_fp2_ref.so), the VOLE-committed round loop,
           the late rounds (oracle/gkr_late_oracle.py, a restatement of the
           reference's Python LayerProver) and the closing proofs
           (tests/layervole.py closing_python), all in the reference prover's
           order (circuitnizkvec_vole.py:396-500)
  open     the reference's own linearPC_multi_prove program (oracle/_ref, built
           from the reference sources) on the frame's input.txt, manifest and
           GKR point, with the reference's ./fft_gkr in its working directory:
           it recommits, opens (tensor_product_protocol) and runs its EC(y1)
           self-check, and writes orion_proof.bin

The reference's own Python prover and circuit front-end are not run (this box
runs compiled reference code only); their steps are the restatements named
above, which do the same work in the same order.
"""
from __future__ import annotations

import json
import os
import struct
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
REF_DIR = os.path.join(HERE, "_ref")
P61 = (1 << 61) - 1
LAYOUT_ID = "copy-major-384-const128-pad512-v1"


def available() -> str:
    """'' when the reference builds this needs are present, else why not"""
    for name in ("libnative_fp2_ref.so", "liborion_ref.so", "linearPC_multi_prove", "fft_gkr"):
        if not os.path.exists(os.path.join(REF_DIR, name)):
            return "oracle/_ref/%s missing (make -C oracle ref)" % name
    return ""


def prove_frame(pix: np.ndarray, copies: int, cs: int, ci: int, cv: int, gt, i0, i1, pid: int, u, v,
                workdir: str = None) -> dict:
    """One proved frame (plain prover) on this process's core; returns the stage
    times (seconds) and the sizes of what it wrote."""
    import ctypes
    sys.path[:0] = [os.path.join(ROOT, "tests"), HERE]
    from circuitlib import oracle_outputs
    from fp2lib import REF_LIB, Fp2Lib
    from fslib import PyTranscript, encode_put, f2add, f2mul, f2sub, interpolate_cubic
    import gkr_late_oracle as oracle
    from layervole import closing_python
    W, n = 512, 9
    padded = 1 << max(1, (copies - 1).bit_length())
    nb = padded.bit_length() - 1
    N = padded * W
    times = {}
    t0 = time.perf_counter()
    # ---- commit phase: the reference's commit() of the input vector
    lib = ctypes.CDLL(os.path.join(REF_DIR, "liborion_ref.so"))
    V_ = ctypes.c_void_p
    lib.ref_commit.argtypes = [V_, ctypes.c_longlong, V_, V_]
    vec = np.zeros((padded, W), np.uint64)
    vec[:copies, :cs] = pix.reshape(copies, cs)
    if ci >= 0:
        vec[:copies, ci] = cv
    elems = np.zeros(2 * N, np.uint64)
    elems[1::2] = vec.reshape(-1)
    root, hx = ctypes.create_string_buffer(32), ctypes.create_string_buffer(80)
    lib.ref_commit(V_(elems.ctypes.data), N, root, hx)
    root_hex = hx.value.decode()
    manifest = dict(protocol="truepix", layout=LAYOUT_ID, zk=False, copies=copies, padded_copies=padded,
                    copy_size=cs, padded_copy_size=W, const_idx=ci, const_val=cv, n=N, lg_n=N.bit_length() - 1,
                    masked_root=root_hex, mask_root="")
    t1 = time.perf_counter()
    times["commit"] = t1 - t0
    # ---- IO transcript
    outs = oracle_outputs(pix, copies, padded, cs, W, ci, cv, gt, i0, i1)
    T = PyTranscript("truepix")
    T.h.update(encode_put(pid) + encode_put(None) + encode_put(["private_input_omitted", N]))
    T.h.update(b"\x01" + struct.pack("<I", outs.size) + outs.tobytes())
    binding = (["orion-commit", "truepix", LAYOUT_ID, 0] +
               [manifest[k] for k in ("copies", "padded_copies", "copy_size", "padded_copy_size", "const_idx",
                                      "const_val", "n", "lg_n")] + [manifest["masked_root"], ""])
    T.h.update(encode_put(binding))
    z1 = [T.ext("z1-%d" % i) for i in range(9)]
    z2 = [T.ext("z2-%d" % i) for i in range(nb)]
    t2 = time.perf_counter()
    times["io"] = t2 - t1
    # ---- GKR: early rounds in the reference library, round loop, late rounds, closing proofs
    rl = Fp2Lib(REF_LIB, "native_fp2_")
    zr, zi = (np.ascontiguousarray([p[k] for p in z1], np.uint64) for k in (0, 1))
    wr, wi = rl.compute_beta(zr, zi, (1, 0))
    zg = [(int(a), int(b)) for a, b in zip(wr[:len(gt)], wi[:len(gt)])]
    zr2, zi2 = (np.ascontiguousarray([p[k] for p in z2], np.uint64) for k in (0, 1))
    br, bi = rl.compute_beta(zr2, zi2, (1, 0))
    vr = np.ascontiguousarray(vec.T.reshape(-1))
    vi = np.zeros_like(vr)
    g32 = [np.ascontiguousarray(a, np.int32) for a in (gt, i0, i1)]
    h = rl.early_create(*g32, np.ascontiguousarray(wr[:len(gt)]), np.ascontiguousarray(wi[:len(gt)]), padded, W,
                        vr, vi, np.ascontiguousarray(br), np.ascontiguousarray(bi))
    uu = [(int(a), int(b)) for a, b in u]
    vv = [(int(a), int(b)) for a, b in v]
    idx, prev = 0, None
    v_elem, out_elem = [(0, 0)] * 4, [(0, 0)] * 4
    chals, late = [], None
    gates = tuple([int(x) for x in a] for a in (gt, i0, i1))
    for rd in range(nb + 2 * n):
        if rd < nb:
            rc, o8 = rl.early_claim(h)
            cf = interpolate_cubic(*[(int(o8[2 * k]), int(o8[2 * k + 1])) for k in range(4)])
        else:
            if late is None:
                rc, wre, wim, beta = rl.early_finish(h, W)
                rl.early_destroy(h)
                late = oracle.LateRounds([(int(a), int(b)) for a, b in zip(wre, wim)], (int(beta[0]), int(beta[1])),
                                         zg, gates, n)
            cf = late.coefs()
        tags = []
        for k, x in enumerate(cf):
            tags.append(vv[idx])
            T.fp2(*f2sub(x, uu[idx]))
            idx += 1
            v_elem[k] = f2add(v_elem[k], tags[-1])
            out_elem[k] = f2add(out_elem[k], x)
        now = tags[0]
        for tt in tags:
            now = f2add(now, tt)
        e = T.ext("eq")
        T.fp2(*(f2mul(now, e) if prev is None else f2mul(f2sub(prev, now), e)))
        r = T.ext("sc-0-%d" % rd)
        chals.append(r)
        p = tags[-1]
        for tt in reversed(tags[:-1]):
            p = f2add(f2mul(p, r), tt)
        prev = p
        if rd < nb:
            rl.early_fold(h, r)
        else:
            late.next_round(r)
    w3, w1, w2 = chals[:nb], chals[nb:nb + n], chals[nb + n:]
    closing, point, tag, _ = closing_python(T, late.line(), prev, idx, v_elem, out_elem, uu, vv, w1, w2, w3, z2, zg,
                                            gates)
    t3 = time.perf_counter()
    times["gkr"] = t3 - t2
    # ---- the reference's prove phase program: recommit, open, EC(y1) self-check
    with tempfile.TemporaryDirectory(dir=workdir) as d:
        with open(os.path.join(d, "input.txt"), "w") as fh:
            rows = pix.reshape(copies, cs)
            fh.write("\n".join(" ".join(map(str, row.tolist())) for row in rows) + "\n")
        with open(os.path.join(d, "gkr_point_prover.txt"), "w") as fh:
            fh.write("%d\n" % len(point) + "".join("%d %d\n" % (a, b) for a, b in point))
        with open(os.path.join(d, "orion_commit.json"), "w") as fh:
            json.dump(manifest, fh)
        os.symlink(os.path.join(REF_DIR, "fft_gkr"), os.path.join(d, "fft_gkr"))
        env = dict(os.environ, TRUEPIX_PROTOCOL="truepix", TRUEPIX_COPY_SIZE=str(cs), TRUEPIX_CONST_IDX=str(ci),
                   TRUEPIX_CONST_VAL=str(cv), TRUEPIX_GKR_POINT_FILE=os.path.join(d, "gkr_point_prover.txt"),
                   OMP_NUM_THREADS="1")
        env.pop("TRUEPIX_ORION_MODE", None)
        env.pop("TRUEPIX_ORION_PROOF_FILE", None)
        t4 = time.perf_counter()
        r = subprocess.run([os.path.join(REF_DIR, "linearPC_multi_prove"), str(copies), "0"], cwd=d, env=env,
                           capture_output=True, text=True, timeout=3600)
        t5 = time.perf_counter()
        path = os.path.join(d, "orion_proof.bin")
        if r.returncode != 0 or not os.path.exists(path):
            raise RuntimeError("linearPC_multi_prove failed: " + (r.stdout[-800:] + r.stderr[-800:]))
        size = os.path.getsize(path)
    times["files"] = t4 - t3
    times["open"] = t5 - t4
    times["total"] = t5 - t0
    return dict(times=times, opening_bytes=size, closing=len(closing))
