"""Build the in-tree CUDA libraries for sm_100a with nvcc.

    python -m truepix_b200.build          # builds truepix_b200/lib/*.so

Each library is one nvcc invocation over its .cu sources (static cudart, so
the .so loads on a host without a GPU and travels with the source tree).
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIBDIR = os.path.join(PKG, "lib")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-shared",
         "--expt-relaxed-constexpr", "-I" + os.path.join(ROOT, "include")]

LIBS = {
    "libnative_fp2_gpu.so": ["runtime.cu", "gkr.cu", "gkr_pixels.cu", "gkr_batch.cu", "gkr_session.cu",
                             "native_fp2_abi.cu", "mle_noalloc.cu", "orion.cu", "orion_open.cu", "orion_abi.cu", "ntt.cu", "rs_commit.cu", "virgo.cu", "ntt_abi.cu",
                             "transcript.cu", "sha256_host.cpp", "circuit.cu", "late.cu"],
}


def nvcc() -> str:
    exe = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(exe):
        raise RuntimeError("nvcc not found")
    return exe


def build(verbose: bool = False, ptxas_info: bool = False) -> list[str]:
    os.makedirs(LIBDIR, exist_ok=True)
    out = []
    for name, srcs in LIBS.items():
        target = os.path.join(LIBDIR, name)
        paths = [os.path.join(CSRC, s) for s in srcs]
        deps = paths + [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
        deps.append(os.path.join(ROOT, "include", "native_fp2.h"))
        if os.path.exists(target) and not ptxas_info:
            t = os.path.getmtime(target)
            if all(os.path.getmtime(d) <= t for d in deps if os.path.exists(d)):
                out.append(target)
                continue
        cmd = [nvcc()] + ARCH + FLAGS + (["-Xptxas", "-v"] if ptxas_info else []) + \
            ["-o", target] + paths
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
        out.append(target)
    return out


if __name__ == "__main__":
    for p in build(verbose=True, ptxas_info="-v" in sys.argv):
        print("built", p)
