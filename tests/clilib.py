"""Running the process boundaries the reference's Python front end drives
(./fft_gkr and linearPC_multi_{commit,prove,open}): ours from truepix_b200/bin
and, where the oracle's reference builds are present, the reference's own from
oracle/_ref, in scratch directories laid out as fp2_link.py lays them out
(input.txt, orion_commit.json, the GKR point file)."""
from __future__ import annotations

import hashlib
import json
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "truepix_b200", "bin")
REF = os.path.join(ROOT, "oracle", "_ref")
LAYOUT_ID = "copy-major-384-const128-pad512-v1"


def ours(name: str) -> str:
    return os.path.join(BIN, name)


def reference(name: str) -> str:
    return os.path.join(REF, name)


def lay_out(d: str, pix: np.ndarray, copies: int, cs: int, point=None, manifest: dict = None):
    """input.txt (one copy per line), the point file, optionally a manifest"""
    rows = np.asarray(pix).reshape(copies, cs)
    with open(os.path.join(d, "input.txt"), "w") as fh:
        fh.write("\n".join(" ".join(str(int(x)) for x in row) for row in rows) + "\n")
    if point is not None:
        with open(os.path.join(d, "gkr_point_prover.txt"), "w") as fh:
            fh.write("%d\n" % len(point) + "".join("%d %d\n" % (int(a), int(b)) for a, b in point))
    if manifest is not None:
        with open(os.path.join(d, "orion_commit.json"), "w") as fh:
            json.dump(manifest, fh)


def manifest(copies: int, cs: int, ci: int, cv: int, root_hex: str, zk: bool = False) -> dict:
    padded = 1 << max(0, (copies - 1).bit_length())
    n = padded * 512
    return dict(protocol="truepix", layout=LAYOUT_ID, zk=zk, copies=copies, padded_copies=padded, copy_size=cs,
                padded_copy_size=512, const_idx=ci, const_val=cv, n=n, lg_n=n.bit_length() - 1,
                masked_root=root_hex, mask_root="")


def env_for(d: str, cs: int, ci: int, cv: int, **extra) -> dict:
    env = dict(os.environ, TRUEPIX_PROTOCOL="truepix", TRUEPIX_COPY_SIZE=str(cs), TRUEPIX_CONST_IDX=str(ci),
               TRUEPIX_CONST_VAL=str(cv), TRUEPIX_GKR_POINT_FILE=os.path.join(d, "gkr_point_prover.txt"))
    for k in ("TRUEPIX_ORION_MODE", "TRUEPIX_ORION_PROOF_FILE", "TRUEPIX_ORION_RESULT_FILE",
              "TRUEPIX_ORION_COMMIT_FILE"):
        env.pop(k, None)
    env.update({k: str(v) for k, v in extra.items()})
    return env


def run(prog: str, d: str, env: dict, *args, timeout: int = 600) -> subprocess.CompletedProcess:
    return subprocess.run([prog] + [str(a) for a in args], cwd=d, env=env, capture_output=True, text=True,
                          timeout=timeout)


def sha256_file(path: str) -> bytes:
    with open(path, "rb") as fh:
        return hashlib.sha256(fh.read()).digest()


def first_error(r: subprocess.CompletedProcess) -> str:
    lines = [ln for ln in r.stderr.splitlines() if ln.strip()]
    return lines[0] if lines else ""
