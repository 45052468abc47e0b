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
                             "transcript.cu", "sha256_host.cpp", "circuit.cu", "late.cu", "open_host.cu", "fft_gkr.cu", "orion_verify.cu"],
}


# Programs over the library (host code), in truepix_b200/bin/: the process
# boundaries the reference's Python front end runs (./fft_gkr and the
# linearPC_multi_* Orion programs), each linked to libnative_fp2_gpu.so.
BINDIR = os.path.join(PKG, "bin")
PROGRAMS = {
    "fft_gkr": ("fft_gkr_main.cpp", []),
    "linearPC_multi_commit": ("orion_cli.cpp", ["-DTP_CLI_PHASE=1"]),
    "linearPC_multi_prove": ("orion_cli.cpp", ["-DTP_CLI_PHASE=2"]),
    "linearPC_multi_open": ("orion_cli.cpp", ["-DTP_CLI_PHASE=3"]),
    "linearPC_multi_commit_zk": ("orion_cli.cpp", ["-DTP_CLI_PHASE=1", "-DTP_CLI_ZK=1"]),
    "linearPC_multi_prove_zk": ("orion_cli.cpp", ["-DTP_CLI_PHASE=2", "-DTP_CLI_ZK=1"]),
    "linearPC_multi_open_zk": ("orion_cli.cpp", ["-DTP_CLI_PHASE=3", "-DTP_CLI_ZK=1"]),
}


def nvcc() -> str:
    exe = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(exe):
        raise RuntimeError("nvcc not found")
    return exe


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(verbose: bool = False, ptxas_info: bool = False, jobs: int | None = None) -> list[str]:
    """Compile every source of each library to an object in parallel (one nvcc
    per source, objects under lib/_build/), then link the shared library."""
    from concurrent.futures import ThreadPoolExecutor
    os.makedirs(LIBDIR, exist_ok=True)
    objdir = os.path.join(LIBDIR, "_build")
    os.makedirs(objdir, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers += [os.path.join(ROOT, "include", f) for f in os.listdir(os.path.join(ROOT, "include"))]
    compile_flags = [f for f in FLAGS if f != "-shared"]
    out = []
    for name, srcs in LIBS.items():
        target = os.path.join(LIBDIR, name)
        objs, todo = [], []
        for s in srcs:
            src = os.path.join(CSRC, s)
            obj = os.path.join(objdir, os.path.splitext(s)[0] + ".o")
            objs.append(obj)
            if ptxas_info or _stale(obj, [src] + headers):
                todo.append([nvcc()] + ARCH + compile_flags + (["-Xptxas", "-v"] if ptxas_info else []) +
                            ["-c", "-o", obj, src])

        def run(cmd):
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.run(cmd, check=True)

        with ThreadPoolExecutor(max_workers=jobs or os.cpu_count() or 4) as ex:
            list(ex.map(run, todo))
        if todo or _stale(target, objs):
            run([nvcc()] + ARCH + ["-shared", "-o", target] + objs)
        out.append(target)
    os.makedirs(BINDIR, exist_ok=True)
    lib = os.path.join(LIBDIR, "libnative_fp2_gpu.so")
    progs = []
    for name, (src, defs) in PROGRAMS.items():
        target = os.path.join(BINDIR, name)
        srcp = os.path.join(CSRC, src)
        if _stale(target, [srcp, lib] + headers):
            progs.append([nvcc()] + ARCH + ["-O2", "-std=c++17", "-I" + os.path.join(ROOT, "include")] + defs +
                         ["-o", target, srcp, "-L" + LIBDIR, "-lnative_fp2_gpu", "-Xlinker", "-rpath",
                          "-Xlinker", "$ORIGIN/../lib"])
        out.append(target)
    with ThreadPoolExecutor(max_workers=jobs or os.cpu_count() or 4) as ex:
        list(ex.map(run, progs))
    return out


if __name__ == "__main__":
    for p in build(verbose=True, ptxas_info="-v" in sys.argv):
        print("built", p)
