"""Golden vectors for the Fiat-Shamir transcript from the reference's own class
(TruePix-main/libTruePix/fiatshamir.py, imported from the reference checkout):
seeded scripts of puts (int lists, Fp2 values, strings) and draws (rand_ext,
rand_scalar), with every drawn challenge and the final running digest, stored in
tests/golden/fs_golden.npz (each script as JSON text next to its outputs).

Run here (needs the reference checkout):
    python tests/golden/gen_fs_golden.py
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.path.join(os.environ.get("TRUEPIX_REF", "/root/reference"), "TruePix-main")
P61 = (1 << 61) - 1


def scripts():
    rng = np.random.default_rng(2026)
    r = lambda n: [int(x) for x in rng.integers(0, P61, size=n, dtype=np.uint64)]
    out = []
    # a GKR-like run: IO values, commitment labels, then per round four claims and a challenge
    ops = [["u64s", [int(x) for x in rng.integers(0, 256, size=1000, dtype=np.uint64)]],
           ["str", "gkr_input_point"], ["ext", "z1-0"], ["ext", "z2-0"]]
    for rd in range(16):
        ops.append(["fp2s", [r(2) for _ in range(4)]])
        ops.append(["ext", "sc-0-%d" % rd])
    ops += [["scalar"], ["scalar"], ["digest"]]
    out.append(("gkr_rounds", "truepix", ops))
    # block-boundary and edge values: 0, p - 1, 2^64 - 1, long and empty-ish labels
    ops = [["u64s", [0, P61 - 1, (1 << 64) - 1]], ["fp2s", [[0, 0], [P61 - 1, P61 - 1]]],
           ["str", "x" * 200], ["ext", "L" * 64], ["str", ""], ["ext", "a"]]
    for n in (1, 7, 8, 9, 55, 56, 57, 63, 64, 65, 127, 128):
        ops.append(["u64s", r(n)])
        ops.append(["scalar"])
        ops.append(["digest"])
    out.append(("boundaries", "truepix", ops))
    # put() of mixed Python values through the general encoder (fiatshamir.py:122-138):
    # {"fp2": [re, im]} stands for an Fp2, {"tuple": [...]} for a tuple, {"dict": [[k, v]...]} for a dict
    fp = lambda: {"fp2": r(2)}
    ops = [["put_py", ["private_input_omitted", 384]], ["put_py", None], ["put_py", {"tuple": [fp(), fp()]}],
           ["put_py", [fp(), [fp(), 7, "s"], {"tuple": [None, 5]}]], ["put_py", {"dict": [["a", 1], ["b", fp()]]}],
           ["put_py", 12345], ["put_py", [1, 2, (1 << 64) - 1]], ["put_py", [3, "mixed", 4]],
           ["put_py", {"fp2": [0, P61 - 1]}], ["ext", "gkr_input_point"], ["put_py", [-1, 5]], ["scalar"],
           ["digest"]]
    out.append(("mixed_puts", "truepix", ops))
    # another protocol name and many draws in a row
    ops = [["ext", "pok-%d" % k] for k in range(40)] + [["digest"]]
    out.append(("draws", "orion-opening", ops))
    return out


def py_value(x, Fp2):
    """the JSON form of a put() argument -> Python values with the given Fp2 type"""
    if isinstance(x, dict):
        if "fp2" in x:
            return Fp2(int(x["fp2"][0]), int(x["fp2"][1]), P61)
        if "tuple" in x:
            return tuple(py_value(v, Fp2) for v in x["tuple"])
        return {k: py_value(v, Fp2) for k, v in x["dict"]}
    if isinstance(x, list):
        return [py_value(v, Fp2) for v in x]
    return x


def run(protocol, ops):
    sys.path.insert(0, REF)
    from libTruePix.extfield import Fp2
    from libTruePix.fiatshamir import FiatShamir
    fs = FiatShamir(P61, protocol=protocol)
    outs, digests = [], []
    for op in ops:
        if op[0] == "u64s":
            fs.put(list(op[1]))
        elif op[0] == "fp2s":
            for re, im in op[1]:
                fs.put(Fp2(re, im, P61))
        elif op[0] == "str":
            fs.put(op[1])
        elif op[0] == "put_py":
            fs.put(py_value(op[1], Fp2))
        elif op[0] == "ext":
            c = fs.rand_ext(op[1])
            outs += [int(c.real), int(c.imag)]
        elif op[0] == "scalar":
            outs.append(int(fs.rand_scalar()))
        elif op[0] == "digest":
            digests.append(fs.hash.digest())
    return np.array(outs, np.uint64), np.frombuffer(b"".join(digests), np.uint8)


def main():
    out = {}
    for name, protocol, ops in scripts():
        vals, dig = run(protocol, ops)
        out["fsscript_" + name] = np.frombuffer(json.dumps([protocol, ops]).encode(), np.uint8)
        out["fsout_" + name] = vals
        out["fsdigest_" + name] = dig
    np.savez_compressed(os.path.join(HERE, "fs_golden.npz"), **out)
    print("wrote", len(out), "arrays")


if __name__ == "__main__":
    main()
