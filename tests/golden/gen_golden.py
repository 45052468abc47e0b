"""Generate the golden fixtures for the GKR Fp2 path from the reference itself.

Runs the reference CPU library built from source by `make -C oracle ref`
(oracle/_ref/libnative_fp2_ref.so <- TruePix-main/native_fp2/native_fp2.cpp) on
seeded inputs and stores inputs and outputs in tests/golden/native_fp2_golden.npz.
It also turns the reference's four circuit files (TruePix-main/pws/{gray,inv,
mask,Crop}.pws) into gate tables (type index as in
TruePix-main/libTruePix/native_fp2_bridge.py:450-472) stored in
tests/golden/circuits.npz.

Run here (needs the reference checkout):  python tests/golden/gen_golden.py
"""
from __future__ import annotations

import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
from fp2lib import Fp2Lib, REF_LIB, P61, rand_fp, run_session  # noqa: E402

REF_ROOT = os.environ.get("TRUEPIX_REF", "/root/reference")
PWS_DIR = os.path.join(REF_ROOT, "TruePix-main", "pws")

# pws operator token -> native gate type index
OPS = {"*": 0, "+": 1, "minus": 2, "OR": 5, "XOR": 6, "NOT": 7, "NAND": 8, "NOR": 9,
       "NXOR": 10, "NAAB": 11, "PASS": 12}


def parse_pws(path):
    """Flat one-layer pws: inputs `P Vk = Ij E`, constants `P Vk = c E`,
    gates `P Ok = Va OP Vb E`. Returns (n_inputs, consts{idx: val}, gates)."""
    consts, gates, n_in = {}, [], 0
    for line in open(path):
        t = line.split()
        if not t or t[0] != "P":
            continue
        if t[1].startswith("V"):
            if t[3].startswith("I"):
                n_in += 1
            else:
                consts[int(t[1][1:])] = int(t[3])
        else:
            a, op, b = t[3], t[4], t[5]
            gates.append((OPS[op], int(a[1:]), int(b[1:])))
    g = np.array(gates, dtype=np.int32)
    return n_in, consts, g


def circuits():
    out = {}
    for name in ("gray", "inv", "mask", "Crop"):
        n_in, consts, g = parse_pws(os.path.join(PWS_DIR, name + ".pws"))
        out[name + "_type"] = np.ascontiguousarray(g[:, 0])
        out[name + "_in0"] = np.ascontiguousarray(g[:, 1])
        out[name + "_in1"] = np.ascontiguousarray(g[:, 2])
        out[name + "_ninputs"] = np.array([n_in], np.int32)
        out[name + "_consts"] = np.array(sorted(consts.items()), np.int64).reshape(-1, 2)
    return out


def rand_gates(rng, n_gates, n_wires):
    gt = rng.integers(-1, 14, size=n_gates).astype(np.int32)   # includes default types
    gt[: min(14, n_gates)] = np.arange(-1, 13)[: min(14, n_gates)]
    i0 = rng.integers(0, n_wires, size=n_gates).astype(np.int32)
    i1 = rng.integers(0, n_wires, size=n_gates).astype(np.int32)
    return gt, i0, i1


def main():
    lib = Fp2Lib(REF_LIB, "native_fp2_")
    rng = np.random.default_rng(20261203)
    G = {}

    # fold
    for k, n_out in enumerate((1, 7, 1000)):
        re_, im_ = rand_fp(rng, 2 * n_out), rand_fp(rng, 2 * n_out)
        r = rand_fp(rng, 2)
        ore, oim = lib.fold(re_, im_, r)
        G.update({f"fold{k}_re": re_, f"fold{k}_im": im_, f"fold{k}_r": r,
                  f"fold{k}_ore": ore, f"fold{k}_oim": oim})

    # expand
    re_, im_ = rand_fp(rng, 5), rand_fp(rng, 5)
    ore, oim = lib.expand(re_, im_, 3)
    G.update({"exp_re": re_, "exp_im": im_, "exp_ore": ore, "exp_oim": oim})

    # sumcheck_early with explicit -1 / 2 tables
    for k, (n_gates, n_wires, n_copies) in enumerate(((14, 5, 2), (40, 16, 8), (64, 24, 32))):
        gt, i0, i1 = rand_gates(rng, n_gates, n_wires)
        z = [rand_fp(rng, n_gates) for _ in range(2)]
        v = [rand_fp(rng, n_wires * n_copies) for _ in range(2)]
        f0 = [rand_fp(rng, n_wires * n_copies // 2) for _ in range(2)]
        f1 = [rand_fp(rng, n_wires * n_copies // 2) for _ in range(2)]
        b = [rand_fp(rng, n_copies) for _ in range(2)]
        bf0 = [rand_fp(rng, n_copies // 2) for _ in range(2)]
        bf1 = [rand_fp(rng, n_copies // 2) for _ in range(2)]
        out = lib.sumcheck_early(gt, i0, i1, z[0], z[1], n_copies, n_wires, v[0], v[1],
                                 f0[0], f0[1], f1[0], f1[1], b[0], b[1], bf0[0], bf0[1],
                                 bf1[0], bf1[1])
        pre = f"sc{k}_"
        G.update({pre + "gt": gt, pre + "i0": i0, pre + "i1": i1,
                  pre + "shape": np.array([n_gates, n_wires, n_copies], np.int64),
                  pre + "z": np.stack(z), pre + "v": np.stack(v), pre + "f0": np.stack(f0),
                  pre + "f1": np.stack(f1), pre + "b": np.stack(b), pre + "bf0": np.stack(bf0),
                  pre + "bf1": np.stack(bf1), pre + "out": out})

    # compute_beta
    for k, n_z in enumerate((1, 5, 10)):
        zr, zi = rand_fp(rng, n_z), rand_fp(rng, n_z)
        init = rand_fp(rng, 2) if k else np.array([1, 0], np.uint64)
        ore, oim = lib.compute_beta(zr, zi, init)
        G.update({f"beta{k}_z": np.stack([zr, zi]), f"beta{k}_init": init,
                  f"beta{k}_ore": ore, f"beta{k}_oim": oim})

    # mle_eval_base (inputs include values >= p and zeros)
    for k, n_z in enumerate((0, 1, 2, 7, 12)):
        n = 1 << n_z
        x = rng.integers(0, 1 << 64, size=n, dtype=np.uint64)
        x[rng.random(n) < 0.3] = 0
        if n > 2:
            x[1] = P61
            x[2] = np.uint64((1 << 64) - 1)
        zr, zi = rand_fp(rng, n_z), rand_fp(rng, n_z)
        o = lib.mle_eval_base(x, zr, zi)
        G.update({f"mle{k}_x": x, f"mle{k}_z": np.stack([zr, zi]),
                  f"mle{k}_out": np.array(o, np.uint64)})

    # early sessions: random circuits and the reference circuits at small sizes
    C = circuits()
    sessions = []
    for (n_gates, n_wires, n_copies) in ((14, 4, 2), (30, 7, 16), (100, 33, 64)):
        gt, i0, i1 = rand_gates(rng, n_gates, n_wires)
        sessions.append(("rand", gt, i0, i1, n_wires, n_copies, None))
    for name, n_copies in (("gray", 8), ("inv", 4), ("mask", 8), ("Crop", 16)):
        sessions.append((name, C[name + "_type"], C[name + "_in0"], C[name + "_in1"], 512,
                         n_copies, name))
    for k, (name, gt, i0, i1, n_wires, n_copies, circ) in enumerate(sessions):
        n_gates = gt.size
        z = [rand_fp(rng, n_gates) for _ in range(2)]
        if circ is None:
            v = [rand_fp(rng, n_wires * n_copies) for _ in range(2)]
        else:
            # pixel-like private inputs, imaginary part 0, constants, zero padding
            n_in = int(C[circ + "_ninputs"][0])
            vr = np.zeros((n_wires, n_copies), np.uint64)
            vr[:n_in] = rng.integers(0, 256, size=(n_in, n_copies), dtype=np.uint64)
            for idx, val in C[circ + "_consts"]:
                if idx < n_wires:
                    vr[idx] = val
            v = [vr.reshape(-1).copy(), np.zeros(n_wires * n_copies, np.uint64)]
        b = [rand_fp(rng, n_copies) for _ in range(2)]
        n_rounds = int(np.log2(n_copies))
        chal = np.stack([rand_fp(rng, 2) for _ in range(n_rounds)]) if n_rounds else \
            np.zeros((0, 2), np.uint64)
        claims, wre, wim, beta, _ = run_session(lib, gt, i0, i1, z[0], z[1], n_copies, n_wires,
                                                v[0], v[1], b[0], b[1], chal)
        pre = f"sess{k}_"
        G.update({pre + "gt": gt, pre + "i0": i0, pre + "i1": i1,
                  pre + "shape": np.array([n_gates, n_wires, n_copies], np.int64),
                  pre + "z": np.stack(z), pre + "v": np.stack(v), pre + "b": np.stack(b),
                  pre + "chal": chal, pre + "claims": claims,
                  pre + "wires": np.stack([wre, wim]),
                  pre + "beta": np.array(beta, np.uint64)})
    G["n_sessions"] = np.array([len(sessions)])

    np.savez_compressed(os.path.join(HERE, "native_fp2_golden.npz"), **G)
    np.savez_compressed(os.path.join(HERE, "circuits.npz"), **C)
    print("wrote", len(G), "arrays;", len(C), "circuit arrays")


if __name__ == "__main__":
    main()
