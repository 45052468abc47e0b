"""Golden traces of the reference's ./fft_gkr program
(TruePix-main/Orion/Orion_nonzk/src/VPD/fft_circuit_GKR.cpp), made by
oracle/_ref/fft_gkr_harness: the reference source compiled in place with
oracle/fft_gkr_ref_harness.cpp, which runs the steps of its main and engage_gkr
one layer function at a time and prints the claim after each (V_output,
addition_layer, mult_layer, intermediate_layer, ifft_gkr), the last sumcheck
tables, the result and the proof size; for lg <= 6 also every circuit layer
(stored here as the SHA-256 of its line). The randomness is the reference's own
(glibc rand() unseeded), so the device program, drawing the same values in the
same order, must reproduce every line. Also the three numbers the reference's
own ./fft_gkr writes (its proof size is compared; the times are not).

Run here (needs the reference checkout and `make -C oracle ref`):
    python tests/golden/gen_fft_gkr_golden.py
"""
from __future__ import annotations

import hashlib
import json
import os
import subprocess
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF_DIR = os.path.join(ROOT, "oracle", "_ref")
LGS = [0, 1, 2, 3, 4, 5, 6, 8, 10, 12]


def split(trace: str) -> dict:
    """trace text -> {"layers": [sha256 hex per layer line], "lines": [the other lines]}"""
    layers, lines = [], []
    for ln in trace.strip().splitlines():
        if ln.startswith("layer "):
            layers.append(hashlib.sha256(ln.strip().encode()).hexdigest())
        elif not ln.startswith("device_ms"):
            lines.append(ln.strip())
    return {"layers": layers, "lines": lines}


def main():
    out = {}
    for lg in LGS:
        tr = subprocess.run([os.path.join(REF_DIR, "fft_gkr_harness"), str(lg)], check=True, capture_output=True,
                            text=True).stdout
        with tempfile.TemporaryDirectory() as d:
            path = os.path.join(d, "log.txt")
            subprocess.run([os.path.join(REF_DIR, "fft_gkr"), str(lg), path], check=True, capture_output=True)
            v_time, proof_size, p_time = open(path).read().split()
        rec = split(tr)
        rec["program_proof_size"] = int(proof_size)
        out[str(lg)] = rec
    with open(os.path.join(HERE, "fft_gkr_golden.json"), "w") as fh:
        json.dump(out, fh, indent=1)
    print("wrote", os.path.join(HERE, "fft_gkr_golden.json"))


if __name__ == "__main__":
    main()
