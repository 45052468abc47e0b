"""Benchmark: proved 1080p frames/s on one B200.

Workload: seeded 1920x1080x3 uint8 frames; each frame is 16,200 copies of 384
bytes padded to 16,384 x 512 input wires (2^23), proved with TruePix's gray
circuit. A proved frame is what TruePix's prover phase writes for it
(run_truepix_prover.py:218-421, plain prover -z 2): the GKR input layer's NIZK
proof (the IO transcript over the circuit's 2^23 outputs, 14 early and 18 late
VOLE-committed sumcheck rounds, the layer's closing proofs) and the Orion
opening proof (orion_proof.bin) of the frame's input commitment, which is made
in the same run.

One step = one batch of B frames (default 64) through truepix_b200.pipeline:
commits on side streams and IO transcripts on host threads for one batch while
the GKR rounds and openings of the previous batch run on the main stream.

  value         proved frames/s, frames resident in HBM (and in host memory,
                where the IO transcript hashes them); CUDA events on the main
                stream around all steps, the last event recorded after every
                proof of the last step is assembled on the host
  e2e           the same from pinned host frames only: their upload is inside
                the timed region, every proof comes back to host memory
  proof_check   one frame of the timed run against the step-by-step path
                (prove_frames + opening_proof, pinned to the reference's proofs
                and opening files by the GPU tests): byte-identical or the line
                is marked invalid
  breakdown     the single-instance prover (one frame at a time, every stage
                synchronous), batched over plain
  device_core   the device part alone (batched GKR input layer + MLE + Orion
                commit per frame from resident bytes, challenges given): its
                kernels with their time shares and the roofline of the dominant
                ones (the SHA-256 leaf kernel against the integer-ALU pipe, the
                fold kernel against HBM)
  cpu_baseline  the reference implementation's proved frame on one host core
                (oracle/reference_proof.py: the reference's compiled commit,
                native_fp2.cpp and linearPC_multi_prove + fft_gkr programs, its
                Python steps restated)

`--impl reference` runs that reference proved frame on all host cores (one
process per core, one frame per process per step) and prints the same metric.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
from truepix_b200 import native  # noqa: E402

METRIC = ("1080p proved frames/s (whole proof per frame: GKR input-layer NIZK proof with VOLE commitments "
          "+ Orion commitment and opening proof, gray circuit)")
WORKLOAD = "proved_frame_gray_1080p"
UNIT = "frames/s"
H, Wd = 1080, 1920
P61 = (1 << 61) - 1
SEED = 3


def circuit(name="gray"):
    c = np.load(os.path.join(ROOT, "tests", "golden", "circuits.npz"))
    return c[name + "_type"], c[name + "_in0"], c[name + "_in1"]


def rand_fp(rng, n):
    return rng.integers(0, P61, size=n, dtype=np.uint64)


def make_inputs(rng, layout, n_frames):
    frames = [rng.integers(0, 256, size=layout.copies * layout.copy_size, dtype=np.uint8)
              for _ in range(n_frames)]
    nb, ni = layout.n_copy_bits, layout.n_in_bits
    z1 = np.stack([rand_fp(rng, 384), rand_fp(rng, 384)])
    z2 = np.stack([rand_fp(rng, nb), rand_fp(rng, nb)], axis=1)         # [nb, 2]
    point = np.stack([rand_fp(rng, ni + nb), rand_fp(rng, ni + nb)], axis=1)
    chal = np.stack([rand_fp(rng, nb), rand_fp(rng, nb)], axis=1)
    return frames, z1, z2, point, chal


def host_tables(pix, layout):
    """Reference-ABI host inputs for one frame: SoA table and the copy-major vector."""
    C, W, cs = layout.padded_copies, layout.n_wires, layout.copy_size
    vals = np.zeros((C, W), np.uint64)
    vals[:layout.copies, :cs] = pix.reshape(layout.copies, cs)
    vals[:layout.copies, layout.const_idx] = layout.const_val
    return np.ascontiguousarray(vals.T).reshape(-1), vals.reshape(-1)


# --------------------------------------------------------------------------
# CPU side: the reference implementation (oracle/_ref, built from the reference
# sources: native_fp2.cpp and the Orion commit) or the oracle ports when those
# builds are absent.

def frame_elements(pix, layout):
    """The commit input of a frame: element copy * W + wire (img 0, real value)."""
    _, inputs = host_tables(pix, layout)
    out = np.zeros(2 * inputs.size, np.uint64)
    out[1::2] = inputs
    return out


def _cpu_zk_commit(_):
    """The zero-knowledge commit phase (Orion_zk commit_pair of the masked
    polynomial and the mask) of one 1080p frame on one core: (seconds, kind). The
    reference's own sources (oracle/_ref/liborion_zk_ref.so) when built, else the
    oracle's restatement."""
    import ctypes
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from orionlib import ORION_ZK_REF_LIB, OrionOracle, frame_bytes
    from truepix_b200.frame import FrameLayout
    L = FrameLayout.for_frame(H, Wd)
    pix = frame_bytes(SEED, L.copies * L.copy_size)
    if not os.path.exists(ORION_ZK_REF_LIB):
        orc = OrionOracle()
        t0 = time.perf_counter()
        orc.zk_commit(pix, L.copies, L.copy_size, L.n_wires, L.const_idx, L.const_val, L.padded_copies, 12345)
        return time.perf_counter() - t0, "port"
    lib = ctypes.CDLL(ORION_ZK_REF_LIB)
    V = ctypes.c_void_p
    lib.ref_zk_commit.argtypes = [V, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_ulonglong,
                                  V, V, V, V, V]
    coefs = frame_elements(pix, L)
    bufs = [ctypes.create_string_buffer(80) for _ in range(4)]
    t0 = time.perf_counter()
    lib.ref_zk_commit(V(coefs.ctypes.data), L.copies, L.copy_size, L.const_idx, L.const_val, 12345, *bufs, None)
    return time.perf_counter() - t0, "reference"


def _cpu_proved_worker(args):
    """(seconds for n_frames proved frames, stage seconds of the last) of the
    reference implementation on this process's core (oracle/reference_proof.py)"""
    idx, n_frames = args
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import reference_proof
    from truepix_b200.frame import FrameLayout
    os.environ["OMP_NUM_THREADS"] = "1"
    layout = FrameLayout.for_frame(H, Wd)
    rng = np.random.default_rng(SEED + idx)
    pix = rng.integers(0, 256, size=layout.copies * layout.copy_size, dtype=np.uint8)
    count = 4 * layout.n_copy_bits + 7 * layout.n_in_bits + 2
    u = rng.integers(0, P61, size=(count, 2), dtype=np.uint64)
    v = rng.integers(0, P61, size=(count, 2), dtype=np.uint64)
    gt, i0, i1 = circuit()
    t0 = time.perf_counter()
    stages = None
    for k in range(n_frames):
        stages = reference_proof.prove_frame(pix, layout.copies, layout.copy_size, layout.const_idx,
                                             layout.const_val, gt, i0, i1, 1000 + idx * 100 + k, u, v)["times"]
    return time.perf_counter() - t0, stages


REFERENCE_SAMPLE = ("per frame: the reference's commit() of the 2^23 inputs (commit phase); circuit outputs and "
                    "the IO transcript (hashlib, as fiatshamir.py); compute_beta, 14 early rounds and finish in "
                    "the reference's native_fp2.cpp; the VOLE-committed round loop, 18 late rounds and the "
                    "closing proofs restated in Python as the reference prover runs them; the reference's "
                    "linearPC_multi_prove program (recommit, tensor-product opening, EC(y1) self-check with "
                    "its ./fft_gkr) writing orion_proof.bin")


def reference_arm(args, rank, world):
    """The reference implementation's proved frames on all host cores (rank 0
    only): one process per core, each step one frame per process. A proved frame
    takes ~14 s on one core, so at most two timed steps run after one warm-up
    step; the line reports the steps run."""
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import reference_proof
    why = reference_proof.available()
    if why:
        print(json.dumps({"impl": "reference", "unavailable": why}), flush=True)
        return
    import multiprocessing as mp
    workers = max(1, min(os.cpu_count() or 1, 64))
    try:
        import psutil
        workers = max(1, min(workers, int(psutil.virtual_memory().available / 3e9)))
    except Exception:
        pass
    steps = max(1, min(args.steps, 2))
    ctx = mp.get_context("spawn")
    with ctx.Pool(workers) as pool:
        pool.map(_cpu_proved_worker, [(i, 1) for i in range(workers)])     # warm-up step
        t0 = time.perf_counter()
        res = pool.map(_cpu_proved_worker, [(i, steps) for i in range(workers)])
        wall = time.perf_counter() - t0
    frames = workers * steps
    value = frames / wall
    stages = {k: sum(r[1][k] for r in res) / len(res) for k in res[0][1]}
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": steps, "warmup": 1, "ms_per_step": 1e3 * wall / steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64 (Fp2 over 2^61-1)",
        "data": "synthetic",
        "config": {"workload": WORKLOAD, "frame": [H, Wd, 3], "copies": 16200, "wires": 1 << 23,
                   "circuit": "gray.pws", "prover": "plain (-z 2)",
                   "step": f"one proved frame per worker process x {workers} processes",
                   "steps_requested": args.steps, "warmup_requested": args.warmup},
        "stage_seconds_per_frame": stages,
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": workers, "kind": "reference",
                         "sample": f"{steps} timed proved frames per process x {workers} processes after one "
                                   f"warm-up frame each; " + REFERENCE_SAMPLE},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "gpu_launches": 0,
    }
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------------------

class ClockSampler:
    """nvidia-smi samples (50 ms) kept only inside [t_begin, t_end] of the timed region."""

    FIELDS = ("timestamp,clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")
    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.out = ""
        self.t0 = self.t1 = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        time.sleep(0.3)

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        import datetime
        rows = []
        for line in (self.out or "").splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 7 or not parts[1].isdigit():
                continue
            try:
                ts = datetime.datetime.strptime(parts[0], "%Y/%m/%d %H:%M:%S.%f").timestamp()
            except ValueError:
                ts = None
            if ts is not None and self.t0 is not None and not (self.t0 - 0.05 <= ts <= self.t1 + 0.05):
                continue
            rows.append(parts)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = sorted(int(r[1]) for r in rows)
        reasons = sorted({self.NAMES[i] for r in rows for i in range(4) if r[3 + i] == "Active"})
        return {"sm_mhz": sm[len(sm) // 2], "sm_max_mhz": int(rows[0][2]), "reasons": reasons,
                "samples": len(rows)}


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def leaf_int_profile():
    """ALU-pipe instructions per launch of the commits' SHA-256 leaf kernel and the
    pipe's hardware peak per SM per cycle, from the committed ncu summary
    (profiles/leaf_kernel_alu_1080p.json: one 1080p launch)"""
    p = os.path.join(ROOT, "profiles", "leaf_kernel_alu_1080p.json")
    try:
        return json.load(open(p))["leaf_kernel"]
    except (OSError, ValueError, KeyError):
        return None


def int_alu_roof(ms_per_launch, rows_per_launch, sm_mhz, n_sm):
    """the leaf kernel against the integer ALU pipe: ALU warp instructions per
    launch (ncu, scaled by codeword rows) over the live launch duration, against
    the pipe's peak x SMs x the sampled SM clock"""
    prof = leaf_int_profile()
    if not prof or not ms_per_launch or not sm_mhz:
        return None
    inst = prof["alu_warp_inst"] * rows_per_launch / prof["codeword_rows"]
    achieved = inst / (ms_per_launch / 1e3) / 1e9
    peak = prof["alu_peak_warp_inst_per_cycle_per_sm"] * n_sm * sm_mhz * 1e6 / 1e9
    return {"kernel": "leaf_kernel", "bound": "int_alu", "unit": "G ALU warp instructions/s",
            "achieved": achieved, "peak": peak, "frac": achieved / peak,
            "peak_source": "ALU pipe peak_sustained = %d warp instructions per cycle per SM (ncu) x %d SMs x %d MHz "
                           "(SM clock sampled during the run)" % (prof["alu_peak_warp_inst_per_cycle_per_sm"], n_sm,
                                                                  sm_mhz),
            "work_per_launch": {"alu_warp_inst": inst, "compressions": 128 * rows_per_launch,
                                "alu_inst_per_compression": 32 * prof["alu_warp_inst"] / prof["compressions"]},
            "avg_launch_us": 1e3 * ms_per_launch,
            "fmaheavy": {"achieved": prof["fmaheavy_warp_inst"] * rows_per_launch / prof["codeword_rows"] /
                         (ms_per_launch / 1e3) / 1e9,
                         "peak": prof["fmaheavy_peak_warp_inst_per_cycle_per_sm"] * n_sm * sm_mhz * 1e6 / 1e9},
            "traffic": prof["dram_bytes"] * rows_per_launch / prof["codeword_rows"],
            "profile": "profiles/leaf_kernel_int_pipes_1080p.md"}


def profiled_traffic():
    """DRAM bytes (read + write) per launch of each round kernel of the 64-frame
    1080p step, from the committed ncu summary (profiles/gkr_batch_1080p_traffic.json;
    measured at 4 frames per launch and scaled by the frames per launch)."""
    p = os.path.join(ROOT, "profiles", "gkr_batch_1080p_traffic.json")
    if os.path.exists(p):
        try:
            return json.load(open(p))
        except ValueError:
            return None
    return None


COMMIT_TAGS = {9100: "pixel_rows_kernel", 9101: "gather_bytes_kernel", 9102: "gather_kernel",
               9103: "leaf_kernel", 9104: "tree_kernel"}


def kernel_groups(ms, tags, layout, batch=1, cw_len=0, leaves=0):
    """Per kernel kind: launches, total time, algorithmic bytes, folded elements,
    SHA-256 compressions.
    Claim kernels: tag = 1000*(reads bytes) + 100*(fold fused) + log2(copies
    claimed per frame); algorithmic bytes per frame = bytes read once + folded Fp2
    rows written (16 B per element) + table rows read (16 B per element) + beta.
    Commit kernels (tags 9100-9104), per frame: pixel rows = bytes read + 16 B per
    codeword-message element written; leaves = 2 KB read + 32 B written per
    codeword row, 128 compressions per row; tree = 64 B read + 32 B written and 2
    compressions per node; gathers: see ntt/commit notes (one 2 KB row read per
    edge, L2-resident); their algorithmic bytes count every source row read once
    and every target row written once (2 KB each; the depth-0 C graph reads the
    frame's byte matrix, 128 B per row)."""
    rows = layout.const_idx + 1 if layout.const_idx >= 0 else layout.copy_size
    pix_bytes = layout.copies * layout.copy_size
    col_len = layout.padded_copies * layout.n_wires // 128
    groups = {}
    for t, tag in zip(ms, tags):
        comp = 0
        n = 0
        if tag >= 9000:
            name = COMMIT_TAGS.get(tag, "commit_kernel_%d" % tag)
            if name == "pixel_rows_kernel":
                byt, el = pix_bytes + 16 * 128 * col_len + 128 * col_len, 0
            elif name == "leaf_kernel":
                byt, el, comp = 2048 * cw_len + 32 * cw_len, 0, 128 * cw_len
            elif name == "tree_kernel":
                byt, el, comp = 0, 0, 0          # attributed below per frame
            else:
                byt, el = 0, 0
        else:
            pix, fold, lg = tag // 1000, (tag // 100) % 10, tag % 100
            n = 1 << lg                                    # copies claimed
            if pix and not fold:
                name, byt, el = "pix_claim_kernel", pix_bytes + 16 * n, 0
            elif pix and fold:
                name, byt, el = "pix_fold_claim_kernel", pix_bytes + 16 * rows * n + 48 * n, rows * n
            elif fold:
                name, byt, el = "table_round_kernel<fold>", 48 * rows * n + 48 * n, rows * n
            else:
                name, byt, el = "table_round_kernel<claim>", 16 * rows * n + 16 * n, 0
        g = groups.setdefault(name, {"launches": 0, "ms": 0.0, "bytes": 0.0, "folded": 0,
                                     "compressions": 0.0, "by_copies": {}})
        per_launch = batch if tag < 9000 else 1    # a claim launch serves the whole batch
        g["launches"] += 1
        g["ms"] += t
        g["bytes"] += byt * per_launch
        g["folded"] += el * per_launch
        g["compressions"] += comp
        if n:
            bc = g["by_copies"].setdefault(n, [0, 0.0])
            bc[0] += 1
            bc[1] += t
    if "tree_kernel" in groups and leaves:
        g = groups["tree_kernel"]
        frames = g["launches"] / max(1, tree_launches(leaves))
        g["bytes"] = frames * 96 * (leaves - 1)
        g["compressions"] = frames * 2 * (leaves - 1)
    levels = encoder_levels(col_len)
    if "gather_kernel" in groups and levels:
        # every source row read once and every target row written once (2 KB
        # each) over the C graphs of depth >= 1 and all D graphs
        per_frame = 2048 * (sum(n + R for n, R, L, RD in levels[1:]) + sum(L + RD for n, R, L, RD in levels))
        g = groups["gather_kernel"]
        g["bytes"] = per_frame * g["launches"] / (2 * len(levels) - 1)
    if "gather_bytes_kernel" in groups and levels:
        n0, R0 = levels[0][0], levels[0][1]
        g = groups["gather_bytes_kernel"]
        g["bytes"] = g["launches"] * (128 * n0 + 2048 * R0)
    return groups


def encoder_levels(col_len):
    """(n, R, L, RD) per depth of the expander encoder of a column of col_len
    elements (include/linear_code/expanders.h:47-60; the same double arithmetic)."""
    def cw(n):
        if n <= 13:
            return n
        R = int(0.238 * n)
        L = cw(R)
        return n + L + int(n * (1.72 - 1) - L)
    out, n = [], col_len
    while n > 13:
        R = int(0.238 * n)
        L = cw(R)
        out.append((n, R, L, int(n * (1.72 - 1) - L)))
        n = R
    return out


def tree_launches(leaves):
    n, k = leaves, 0
    while n > 1:
        lv = 0
        while lv < 9 and (1 << (lv + 1)) <= n:
            lv += 1
        n >>= lv
        k += 1
    return k


def sha_peak(lib, dev, stream):
    """G compressions/s of the library's SHA-256 code in registers, full device."""
    import torch
    out = torch.zeros(1, dtype=torch.int32, device=dev)
    blocks, iters = 148 * 16, 256
    s = stream.cuda_stream
    with torch.cuda.stream(stream):
        native.check(lib, lib.tp_sha256_peak_dev(blocks, 16, out.data_ptr(), s), "sha peak")
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        native.check(lib, lib.tp_sha256_peak_dev(blocks, iters, out.data_ptr(), s), "sha peak")
        e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    return blocks * 128 * iters * 2 / (ms / 1e3) / 1e9


def ntt_bench(lib, dev, stream, reps=5):
    """Config-2 microbenchmark: forward NTT, inverse NTT and the rate-2^-5 RS
    commit (IFFT + FFT per slice, FRI leaf chains, Merkle tree) at 2^16, 2^20, 2^24."""
    import ctypes
    import torch
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from orionlib import elements
    s = stream.cuda_stream
    out = {}
    for lg in (16, 20, 24):
        n = 1 << lg
        a = torch.from_numpy(elements(lg, n).view(np.int64)).to(dev)
        f = torch.empty_like(a)
        back = torch.empty_like(a)
        cw = torch.empty(2 << (lg + 5), dtype=torch.int64, device=dev)
        tree = torch.empty(32 << (lg - 1), dtype=torch.uint8, device=dev)

        def timed(fn):
            with torch.cuda.stream(stream):
                fn()
                torch.cuda.synchronize()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                for _ in range(reps):
                    fn()
                e1.record(stream)
            torch.cuda.synchronize()
            return e0.elapsed_time(e1) / reps

        t_default = timed(lambda: native.check(lib, lib.tp_fft_dev(a.data_ptr(), n, n, f.data_ptr(), 1, 0, 0, s)))
        digits = (ctypes.c_int * 3)()
        tms = ctypes.c_float()
        passes = lib.tp_ntt_autotune(lg, 1, digits, ctypes.byref(tms))
        native.check(lib, 0 if passes > 0 else -1, "ntt autotune")
        t_f = timed(lambda: native.check(lib, lib.tp_fft_dev(a.data_ptr(), n, n, f.data_ptr(), 1, 0, 0, s)))
        t_i = timed(lambda: native.check(lib, lib.tp_ifft_dev(f.data_ptr(), n, n, back.data_ptr(), 1, 0, 0, s)))
        t_rs = timed(lambda: native.check(lib, lib.tp_rs_commit_dev(a.data_ptr(), lg, cw.data_ptr(),
                                                                      tree.data_ptr(), s)))
        ok = bool(torch.equal(back, a))
        leaves = 1 << (lg - 2)
        comp = leaves * 64 * 2 + (leaves - 1) * 2
        out["2^%d" % lg] = {
            "fft_ms": t_f, "fft_ms_default_split": t_default,
            "autotuned_radix_bits": [int(x) for x in digits[:passes]], "ifft_ms": t_i, "round_trip_exact": ok,
            "fft_elem_per_s": n / (t_f / 1e3), "butterflies_per_s": n / 2 * lg / (t_f / 1e3),
            "fft_hbm_gbs": passes * 32 * n / (t_f / 1e3) / 1e9,
            "rs_commit_ms": t_rs, "rs_codeword_elements": n << 5,
            "rs_sha256_compressions_per_s": comp / (t_rs / 1e3)}
        del a, f, back, cw, tree
        torch.cuda.empty_cache()
    return out


def replica_seed(rank):
    """Replicas only: every rank proves its own frames (seeded by its rank), no
    collective on the data path."""
    return SEED + 101 * rank


def max_over_ranks(ms, world, device):
    """The step time of the whole job: the slowest rank's device time."""
    if world <= 1:
        return float(ms)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(frames_per_rank, max_ms, world):
    """Frames of all ranks over the slowest rank's time (frames/s)."""
    return world * frames_per_rank / (max_ms / 1e3)


def ours_arm(args, rank, world, local_rank):
    import ctypes
    import torch
    import torch.distributed as dist
    from truepix_b200.frame import BatchFrameProver, FrameLayout, GkrInputLayerProver, pack_fp2
    from truepix_b200.orion import FrameCommitter

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    extras = rank == 0 and world == 1
    # ---- the headline: pipelined proved frames (needs the most memory: runs first)
    proved, proved_e2e, pctx = proved_bench(args, rank, world, local_rank)
    check = plain_pf = zk_proved = None
    if rank == 0:
        check = proof_check(pctx)
        if world == 1 and not args.no_plain:
            plain_pf = plain_proved(pctx)
    del pctx
    torch.cuda.empty_cache()
    if extras and not args.skip_zk:
        # TruePix's default: the zero-knowledge prover with commit pairs and two openings per frame
        zres, ze2e, zctx = proved_bench(args, rank, world, local_rank, zk=True, steps=max(2, min(args.steps, 6)),
                                        warmup=2)
        zk_proved = {"frames_per_s": zres["value"], "steps": zres["steps"], "frames_per_step": args.batch,
                     "e2e_frames_per_s": ze2e["value"], "proof_check": proof_check(zctx, zk=True),
                     "what": "the zero-knowledge prover (circuitnizkvec_vole_ZK.py) with the Orion_zk commit pair "
                             "(masked polynomial and mask) and both openings per frame, same pipeline"}
        del zctx
        torch.cuda.empty_cache()
    layout = FrameLayout.for_frame(H, Wd)
    gt, i0, i1 = circuit()
    B = args.batch
    nb = layout.n_copy_bits
    rng = np.random.default_rng(replica_seed(rank))
    frames, z1, z2, point, chal = make_inputs(rng, layout, B)
    pix = [torch.from_numpy(f).to(dev) for f in frames]
    z2_dev = torch.from_numpy(pack_fp2(z2[:, 0], z2[:, 1])).to(dev)
    pt_dev = torch.from_numpy(pack_fp2(point[:, 0], point[:, 1])).to(dev)
    chal_b = np.ascontiguousarray(np.broadcast_to(chal[:, None, :], (nb, B, 2)))
    stream = torch.cuda.Stream(dev)
    lib = native.gkr()
    native.check(lib, lib.tp_orion_set_leaf_chunks(args.leaf_chunks), "leaf chunks")
    bprover = BatchFrameProver([layout] * B, gt, i0, i1, device=local_rank, stream=stream)
    committer = FrameCommitter([layout] * B, device=local_rank, stream=stream, side_streams=args.commit_streams)
    cw_len, leaves = committer.cw_len[0], committer.leaves[0]
    z1s = [z1] * B
    z2s = z2_dev.repeat(B)      # packed [B][nb]
    pts = pt_dev.repeat(B)      # packed [B][9 + nb]

    def run_batch(marks=None):
        """One step. Timed steps: the commits (side streams) start first and run
        under the GKR rounds (step stream), joined at the end. With `marks`
        (the serialised step) the GKR part runs first and `marks` is recorded
        between the two parts."""
        if marks is None and committer.side:
            committer.commit(pix, join=False)
            bprover.prove(pix, z1s, z2s, pts, chal_b)
            committer.join()
            return
        bprover.prove(pix, z1s, z2s, pts, chal_b)
        if marks is not None:
            marks.record(stream)
        committer.commit(pix)

    # ---- one frame at a time (the plain baseline of the GKR part, and of the step)
    plain = GkrInputLayerProver(layout, gt, i0, i1, device=local_rank, stream=stream)
    pcommit = FrameCommitter([layout], device=local_rank, stream=stream)
    n_plain = 0 if args.no_plain else max(8, min(64, B))
    plain_gkr_fps = plain_fps = None
    if n_plain:
        with torch.cuda.stream(stream):
            for i in range(4):
                plain.prove(pix[i % B], z1, z2_dev, pt_dev, chal)
                pcommit.commit([pix[i % B]])
            torch.cuda.synchronize()
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
            ev[0].record(stream)
            for i in range(n_plain):
                plain.prove(pix[i % B], z1, z2_dev, pt_dev, chal)
            ev[1].record(stream)
            for i in range(n_plain):
                plain.prove(pix[i % B], z1, z2_dev, pt_dev, chal)
                pcommit.commit([pix[i % B]])
            ev[2].record(stream)
        torch.cuda.synchronize()
        plain_gkr_fps = n_plain / (ev[0].elapsed_time(ev[1]) / 1e3)
        plain_fps = n_plain / (ev[1].elapsed_time(ev[2]) / 1e3)
    del pcommit
    torch.cuda.empty_cache()

    # ---- compute roof of the SHA-256 leaf kernels
    sha_gcs = sha_peak(lib, dev, stream)

    # ---- batched: the timed region (the first warm-up step measures the round launches' splits)
    from truepix_b200.frame import autotune_rounds, round_tuning
    with torch.cuda.stream(stream):
        for i in range(args.warmup):
            autotune_rounds(i == 0)
            run_batch()
    autotune_rounds(False)
    torch.cuda.synchronize()
    per_step_pairs = nb * 2 + 24 * B + 16
    npairs = args.steps * per_step_pairs
    native.check(lib, lib.tp_timer_enable(npairs), "timer")
    clk = ClockSampler(local_rank)
    clk.start()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    lib.tp_timer_reset()
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    launches = 0
    clk.t0 = time.time()
    with torch.cuda.stream(stream):
        evs[0].record(stream)
        for i in range(args.steps):
            run_batch()
            launches += bprover.launches_last + committer.launches_last
            evs[i + 1].record(stream)
    torch.cuda.synchronize()
    clk.t1 = time.time()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clk.stop()
    tms = (ctypes.c_float * npairs)()
    ttags = (ctypes.c_int * npairs)()
    got = lib.tp_timer_read(tms, ttags, npairs)
    lib.tp_timer_disable()
    ms = evs[0].elapsed_time(evs[-1])
    per_batch = sorted(evs[i].elapsed_time(evs[i + 1]) for i in range(args.steps))
    ms = max_over_ranks(ms, world, dev)
    frames_done = args.steps * B
    value = job_throughput(frames_done, ms, world)

    groups = kernel_groups(list(tms[:max(0, got)]), list(ttags[:max(0, got)]), layout, B,
                           cw_len, leaves)
    peak, peak_kind = peaks()
    traffic = profiled_traffic() or {}

    def summarize(grp, total_ms):
        out = []
        for name, g in sorted(grp.items(), key=lambda kv: -kv[1]["ms"]):
            ach = g["bytes"] / (g["ms"] / 1e3) / 1e9 if g["ms"] > 0 and g["bytes"] else None
            k = {"kernel": name, "launches": g["launches"], "total_ms": g["ms"],
                 "share_of_step": g["ms"] / total_ms, "achieved_gbs": ach}
            if g["compressions"]:
                k["g_compressions_per_s"] = g["compressions"] / (g["ms"] / 1e3) / 1e9
            if g["by_copies"]:
                k["avg_us_by_copies"] = {str(c): round(1e3 * v[1] / v[0], 2)
                                         for c, v in sorted(g["by_copies"].items())}
            out.append(k)
        return out

    n_sm = torch.cuda.get_device_properties(dev).multi_processor_count
    core_mhz = clk.summary()["sm_mhz"] or 1965     # sampled during the timed steps (else the B200's max clock)

    def roof_of(k, grp):
        g = grp[k["kernel"]]
        if k["kernel"] == "leaf_kernel":
            # integer-ALU bound: the hardware ALU pipe is the roof (the HBM and the register-only
            # figures stay beside it)
            # a launch hashes every row over 1 / leaf_chunks of the column pairs
            r = int_alu_roof(g["ms"] / g["launches"], cw_len / args.leaf_chunks, core_mhz, n_sm)
            if r is not None:
                r["hbm"] = {"achieved_gbs": k["achieved_gbs"], "peak_gbs": peak,
                            "frac": k["achieved_gbs"] / peak if k["achieved_gbs"] else None}
                if k.get("g_compressions_per_s"):
                    r["sha256_register_only"] = {"achieved_g_compressions_per_s": k["g_compressions_per_s"],
                                                 "same_code_register_only": sha_gcs}
                return r
        r = {"kernel": k["kernel"], "bound": "hbm", "achieved": k["achieved_gbs"], "peak": peak,
             "unit": "GB/s",
             "frac": k["achieved_gbs"] / peak if k["achieved_gbs"] else None,
             "peak_source": (peak_kind + " hbm_gbs (MEASURED_PEAKS.json)") if peak_kind == "measured"
             else "fallback 6650 GB/s",
             "algorithmic_bytes_per_launch": g["bytes"] / g["launches"],
             "avg_launch_us": 1e3 * g["ms"] / g["launches"], "launches_timed": g["launches"],
             "traffic": traffic.get(k["kernel"])}
        if k.get("g_compressions_per_s"):
            r["compute"] = {"unit": "G SHA-256 compressions/s", "achieved": k["g_compressions_per_s"],
                            "peak": sha_gcs, "frac": k["g_compressions_per_s"] / sha_gcs,
                            "peak_source": "register-only throughput of the same SHA-256 code on "
                                           "this GPU (tp_sha256_peak_dev, measured in this run)"}
        return r

    kernels = summarize(groups, ms)
    roof = roof_of(kernels[0], groups) if kernels else None
    hbm_kernel = next((k for k in kernels if k["kernel"] == "table_round_kernel<fold>"), None)
    roof_fold = roof_of(hbm_kernel, groups) if hbm_kernel else None

    # One more step, outside the timed region, with the commits serialised on the
    # step's stream: per-kernel durations with no other stream's kernels sharing
    # the SMs (the timed step spreads commits over side streams, so its
    # per-kernel durations overlap).
    kernels_iso = roof_iso = None
    gkr_ms = commit_ms = None
    if rank == 0:
        side, committer.side = committer.side, []
        native.check(lib, lib.tp_timer_enable(per_step_pairs), "timer")
        lib.tp_timer_reset()
        with torch.cuda.stream(stream):
            i0e, i1e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            imid = torch.cuda.Event(enable_timing=True)
            i0e.record(stream)
            run_batch(imid)
            i1e.record(stream)
        torch.cuda.synchronize()
        gkr_ms, commit_ms = i0e.elapsed_time(imid), imid.elapsed_time(i1e)
        got_i = lib.tp_timer_read(tms, ttags, npairs)
        lib.tp_timer_disable()
        committer.side = side
        g_iso = kernel_groups(list(tms[:max(0, got_i)]), list(ttags[:max(0, got_i)]), layout, B, cw_len, leaves)
        kernels_iso = summarize(g_iso, i0e.elapsed_time(i1e))
        roof_iso = roof_of(kernels_iso[0], g_iso) if kernels_iso else None

    folded = sum(g["folded"] for g in groups.values())

    res_ok = None
    if rank == 0:
        c, w, b, m = bprover.results(B - 1)
        res_ok = bool(c.any() and w.any() and m != (0, 0) and any(committer.root(B - 1)))

    ntt = e2e = e2e_ref = cpu = uneven = serving = zk = opening = ref_gpu = fs_rounds = programs = None
    # The side measurements run once, at N = 1 (a scaling run holds every GPU
    # while rank 0 works; it only needs the step's value).
    if extras and not args.skip_ntt:
        ntt = ntt_bench(lib, dev, stream)
    if extras and not args.skip_opening:
        opening = opening_bench(args, lib, committer, layout, dev, stream, sha_gcs)
    if extras and not args.skip_zk:
        zk = zk_step(args, bprover, pix, z1s, z2s, pts, chal_b, layout, stream, local_rank)
    if not args.skip_e2e:
        # every rank: the job's e2e is all ranks' frames over the slowest rank's time
        e2e = e2e_batched(args, bprover, committer, frames, z1s, z2s, pts, chal_b, stream, dev, world)
    if extras and not args.skip_e2e:
        e2e_ref = e2e_c_abi(args, lib, frames[0], layout, gt, i0, i1, z1, z2, point, chal)
        ref_gpu = reference_gpu_lib(frames[0], layout, gt, i0, i1, z1, z2, point, chal)
        fs_rounds = transcript_rounds(bprover, pix, z1s, z2s, pts, stream)
        programs = process_boundaries(frames[0], layout)
    if extras and not args.skip_serving:
        del bprover
        committer.rows = committer.trees = None
        torch.cuda.empty_cache()
        uneven, serving = serving_in_own_process(local_rank)
    if rank == 0 and world == 1 and not args.skip_cpu:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import reference_proof
        if reference_proof.available():
            cpu = {"unavailable": reference_proof.available()}
        else:
            import multiprocessing as mp
            with mp.get_context("spawn").Pool(1, maxtasksperchild=1) as pool:
                secs, stages = pool.apply(_cpu_proved_worker, ((0, 1),))
            cpu = {"value": 1.0 / secs, "unit": UNIT, "cores": 1, "kind": "reference",
                   "sample": "1 proved frame of the same workload, one process; " + REFERENCE_SAMPLE,
                   "stage_seconds": stages}
    if rank == 0:
        core = {
            "what": "the device part alone: batched GKR input layer (beta, 14 early rounds, finish, MLE) and the "
                    "Orion commit of every frame from its resident bytes, challenges given, commits on %d side "
                    "streams under the rounds" % len(committer.side),
            "frames_per_s": value, "ms_per_step": ms / args.steps, "steps": args.steps, "frames_per_step": B,
            "fp2_elem_per_s": folded / (ms / 1e3),
            "breakdown": {
                "serialised_step": "GKR part, then the commits, on one stream",
                "gkr_ms_per_step": gkr_ms, "commit_ms_per_step": commit_ms,
                "gkr_frames_per_s": B / (gkr_ms / 1e3) if gkr_ms else None,
                "commit_frames_per_s": B / (commit_ms / 1e3) if commit_ms else None,
                "plain_frames_per_s": plain_fps, "plain_gkr_frames_per_s": plain_gkr_fps,
                "gkr_batched_over_plain": (B / (gkr_ms / 1e3) / plain_gkr_fps) if plain_gkr_fps and gkr_ms
                else None},
            "kernels": kernels_iso or kernels, "roofline_fold_kernel": roof_fold,
            "kernels_timed_region": kernels,
            "kernels_note": "kernels (and the line's roofline) come from one step with the commits serialised "
                            "on the step's stream (CUDA events around every launch), whose shares match the "
                            "serialised ncu launch list; the timed steps overlap them (kernels_timed_region)",
            "e2e_from_pinned_frames": e2e, "outputs_nonzero": res_ok,
            "round_tuning": [{"kind": k, "bucket": b, "ctas_per_sm": m} for k, b, m in round_tuning()],
            "round_tuning_note": "the round autotuner's measured CTA split per (kind: 0 table claim, 1 table fold + "
                                 "claim, 2 byte claim, 3 byte fold + claim; bucket: log2 of pairs x rows), "
                                 "measured in the first warm-up step (tp_batch_autotune)"}
        valid = bool(check and check["ok"])
        line = {
            "metric": METRIC, "value": proved["value"], "unit": UNIT, "n_gpus": world,
            "steps": proved["steps"], "warmup": args.warmup, "ms_per_step": proved["ms"] / proved["steps"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "u64 (Fp2 over 2^61-1)", "data": "synthetic",
            "batched_over_plain": (proved["value"] / world / plain_pf["frames_per_s"]) if plain_pf else None,
            "config": {"workload": WORKLOAD, "frame": [H, Wd, 3],
                       "copies": layout.copies, "padded_copies": layout.padded_copies,
                       "wires": layout.padded_copies * layout.n_wires, "early_rounds": nb, "late_rounds": 18,
                       "circuit": "gray.pws", "prover": "plain (-z 2)", "batch": B,
                       "step": f"one batch of {B} frames through the whole proof (truepix_b200.pipeline)",
                       "orion": {"columns": 128, "codeword_rows": cw_len, "tree_leaves": leaves,
                                 "queried_columns": 1222},
                       "l2": "inputs > L2: B distinct frames (0.4 GB) and their codewords (14.8 GB) per step",
                       "host_threads": os.cpu_count(), "pipeline": proved.get("pipeline"),
                       "parallelism": f"replicas x{world}"},
            "proof_check": check,
            "breakdown": {
                "plain": plain_pf,
                "batched_over_plain": (proved["value"] / world / plain_pf["frames_per_s"]) if plain_pf else None,
                "latency_ms_per_batch": proved["latency_ms_per_batch"],
                "bound": "host: the IO transcript hashes each frame's 64 MiB output vector with SHA-256, a "
                         "sequential chain per frame, on the host cores"},
            "e2e": proved_e2e,
            "roofline": roof_iso or roof,
            "roofline_note": "the dominant device kernel of the step (the commits' SHA-256 leaf chains), timed in "
                             "the device-core measurement below",
            "device_core": core,
            "zk": zk_proved, "zk_device_core": zk,
            "ntt": ntt, "opening": opening, "batched_uneven": uneven, "serving": serving,
            "cpu_baseline": cpu, "e2e_reference_abi": e2e_ref,
            "reference_gpu_library": ref_gpu, "transcript_rounds": fs_rounds, "process_boundaries": programs,
            "gpu_launches": proved["launches"], "clocks": proved["clocks"],
        }
        if not valid:
            line["invalid"] = "proof check failed: the timed proofs differ from the step-by-step path"
        print(json.dumps(line), flush=True)


def proved_inputs(rng, layout, B, zk=False):
    """B seeded frames (pinned host tensors), VOLE correlations per frame"""
    import torch
    from truepix_b200.pipeline import correlations_needed
    count = correlations_needed(layout, zk)
    frames = [torch.from_numpy(rng.integers(0, 256, size=layout.copies * layout.copy_size, dtype=np.uint8))
              .pin_memory() for _ in range(B)]
    corr = [(rng.integers(0, P61, size=(count, 2), dtype=np.uint64),
             rng.integers(0, P61, size=(count, 2), dtype=np.uint64)) for _ in range(B)]
    return frames, corr


def proved_bench(args, rank, world, local_rank, zk=False, steps=None, warmup=None):
    """The headline: proved frames/s of the pipelined prover (truepix_b200.pipeline),
    frames resident in HBM, then (`e2e`) from pinned host frames. CUDA events on
    the pipeline's main stream; the end event is recorded once every proof of the
    last step is assembled on the host. Max over ranks."""
    import torch
    import torch.distributed as dist
    from truepix_b200.frame import FrameLayout
    from truepix_b200.pipeline import ProofPipeline
    dev = torch.device("cuda", local_rank)
    layout = FrameLayout.for_frame(H, Wd)
    gt, i0, i1 = circuit()
    B = args.batch
    K = steps or args.steps
    Wm = warmup or args.warmup
    rng = np.random.default_rng(replica_seed(rank) + 100)
    frames, corr = proved_inputs(rng, layout, B, zk)
    frames_dev = [f.to(dev) for f in frames]
    pipe = ProofPipeline(layout, gt, i0, i1, batch=B, device=local_rank, zk=zk, commit_streams=args.commit_streams)

    def batches(k, resident, base):
        for b in range(k):
            yield dict(frames_host=frames, frames_dev=frames_dev if resident else None,
                       pids=[base + b * B + f for f in range(B)], correlations=corr,
                       mask_seeds=[base + b * B + f for f in range(B)] if zk else None)

    out = {}
    for mode in ("resident", "host"):
        for _ in pipe.run(batches(Wm, mode == "resident", 1 << 20)):
            pass
        torch.cuda.synchronize(dev)
        if world > 1:
            dist.barrier()
        clk = ClockSampler(local_rank)
        if mode == "resident":
            clk.start()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize(dev)
        clk.t0 = time.time()
        pipe.launches_last = 0
        e0.record(pipe.stream)
        last = None
        marks = []
        t0 = time.perf_counter()
        for proofs in pipe.run(batches(K, mode == "resident", 0)):
            last = proofs
            marks.append(time.perf_counter() - t0)
        e1.record(pipe.stream)
        torch.cuda.synchronize(dev)
        clk.t1 = time.time()
        launches = pipe.launches_last
        if mode == "resident":
            clk.stop()
        if world > 1:
            dist.barrier()
        ms = max_over_ranks(e0.elapsed_time(e1), world, dev)
        value = job_throughput(K * B, ms, world)
        gaps = sorted(b - a for a, b in zip([0.0] + marks[:-1], marks))
        res = {"value": value, "ms": ms, "launches": launches, "steps": K,
               "latency_ms_per_batch": {"p50": 1e3 * gaps[len(gaps) // 2],
                                        "p99": 1e3 * gaps[min(len(gaps) - 1, int(0.99 * len(gaps)))]}}
        if mode == "resident":
            res["clocks"] = clk.summary()
            res["last"] = last
        out[mode] = res
    frame_bytes = layout.copies * layout.copy_size
    cw, qc, lv = pipe.cw_len, pipe.qc, pipe.leaves
    # host -> device per step: frames (e2e only), z2, transcript and VOLE states, correlations, the opening's
    # r0 / r1 / queried indices / node lists; device -> host: roots, the GKR proof values and final states,
    # per opened polynomial the combined codeword, its root, the answer, the queried columns and the nodes
    n_poly = 2 if zk else 1
    small_h2d = B * (16 * layout.n_copy_bits + 120 + 160 + 2 * 16 * pipe.count)
    open_h2d = B * n_poly * (16 * 128 + 16 * (pipe.N // 128) + 8 * qc + 4 * qc * 17)
    d2h = B * (32 * n_poly + 16 * (5 * layout.n_copy_bits + 8 * layout.n_in_bits + 20 + layout.n_in_bits +
                                   layout.n_copy_bits + 1) + 120 + 160) + \
        B * n_poly * (16 * cw + 32 + 16 + 16 * 128 * qc + 2 * 32 * qc * 17)
    res_e2e = {"value": out["host"]["value"], "unit": UNIT, "h2d_bytes_per_step": B * frame_bytes + small_h2d + open_h2d,
               "d2h_bytes_per_step": d2h, "steps": K, "frames_per_step": B,
               "timer": "CUDA events on the main stream, the end event after the last proofs are assembled",
               "path": "pinned host frames uploaded on a copy stream inside the timed region; every proof "
                       "(GKR proof values, opening file bytes) assembled in host memory"}
    # the pipeline's shape: device slots, IO hashing groups and lookahead, opening groups, host threads
    out["resident"]["pipeline"] = {"slots": len(pipe.slots), "io_group": pipe.io_group, "io_ahead": pipe.io_ahead,
                                   "open_group": pipe.open_group, "io_threads": pipe.io_pool._max_workers,
                                   "host_threads": pipe.pool._max_workers}
    pipe.close()
    last = out["resident"].pop("last")
    del pipe, frames_dev
    torch.cuda.empty_cache()
    return out["resident"], res_e2e, (frames, corr, last, layout, gt, i0, i1)


def proof_check(ctx, zk=False):
    """One frame of the timed run against the step-by-step path (commit,
    prove_frames, opening_proof; pinned to the reference prover's proofs and to
    the reference program's opening files by the GPU tests)."""
    import torch
    from truepix_b200.opening import opening_proof
    from truepix_b200.orion import FrameCommitter
    from truepix_b200.prover import manifests_of, prove_frames
    frames, corr, last, layout, gt, i0, i1 = ctx
    f = len(last) - 1
    p = last[f]
    pix = frames[f].cuda()
    fc = FrameCommitter([layout], zk=zk)
    fc.commit([pix], mask_seeds=[p.pid] if zk else None)
    torch.cuda.synchronize()
    [m] = manifests_of(fc)
    [t] = prove_frames([pix], layout, gt, i0, i1, [p.pid], [corr[f]], [m], zk=zk)
    pt = [(int(x[0]), int(x[1])) if not hasattr(x, "real") else (int(x.real), int(x.imag))
          for x in t.final_input_point]
    ok = p.manifest == m and p.proof_bytes() == t.proof_bytes()
    if zk:
        ok = ok and p.opening["masked"] == opening_proof(fc, 0, pt, "masked") and \
            p.opening["mask"] == opening_proof(fc, 0, pt, "mask")
    else:
        ok = ok and p.opening == opening_proof(fc, 0, pt)
    del fc
    torch.cuda.empty_cache()
    return {"ok": bool(ok), "frame": "the last frame of the last timed step",
            "against": "truepix_b200.prover.prove_frames + truepix_b200.opening.opening_proof on the same frame, "
                       "pid and correlations (the step-by-step path the GPU tests pin to the reference)",
            "proof_bytes": len(p.proof_bytes()),
            "opening_bytes": sum(map(len, p.opening.values())) if zk else len(p.opening)}


def plain_proved(ctx, n=6):
    """The single-instance prover: one frame at a time, every stage synchronous
    (commit, IO transcript, GKR rounds and closing proofs, opening) on the same
    device code, no batching and no overlap. Wall clock."""
    import torch
    from truepix_b200.opening import opening_proof
    from truepix_b200.orion import FrameCommitter
    from truepix_b200.prover import manifests_of, prove_frames
    frames, corr, _, layout, gt, i0, i1 = ctx
    fc = FrameCommitter([layout])

    def one(f):
        pix = frames[f % len(frames)].cuda()
        fc.commit([pix])
        torch.cuda.synchronize()
        [t] = prove_frames([pix], layout, gt, i0, i1, [f], [corr[f % len(corr)]], manifests_of(fc), zk=False)
        pt = [(int(x[0]), int(x[1])) if not hasattr(x, "real") else (int(x.real), int(x.imag))
              for x in t.final_input_point]
        opening_proof(fc, 0, pt)

    one(0)
    t0 = time.perf_counter()
    for f in range(n):
        one(f)
    secs = (time.perf_counter() - t0) / n
    del fc
    torch.cuda.empty_cache()
    return {"frames_per_s": 1.0 / secs, "ms_per_frame": 1e3 * secs, "frames": n,
            "what": "one frame at a time through the same device code, each stage synchronous: commit "
                    "(FrameCommitter), prove_frames (IO transcript, VOLE rounds, closing proofs), opening_proof"}


def zk_step(args, bprover, pix, z1s, z2s, pts, chal_b, layout, stream, local_rank):
    """The step with TruePix's default zero-knowledge commit: the batched GKR
    input layer plus, per frame, the commit pair of the masked polynomial and the
    mask (Orion_zk commit_pair, two encodes and two trees), the pairs on side
    streams under the rounds as in the timed steps. Device time, CUDA events."""
    import torch
    from truepix_b200.orion import FrameCommitter
    B = bprover.B
    zc = FrameCommitter([layout] * B, device=local_rank, stream=stream, side_streams=args.commit_streams, zk=True)
    seeds = [0x5EED0000 + f for f in range(B)]

    def one():
        zc.commit(pix, join=False, mask_seeds=seeds)
        bprover.prove(pix, z1s, z2s, pts, chal_b)
        zc.join()

    steps = max(2, min(args.steps, 5))
    with torch.cuda.stream(stream):
        for _ in range(2):
            one()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            one()
        e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    ok = any(zc.root(B - 1)) and any(zc.mask_root(B - 1)) and zc.root(B - 1) != zc.mask_root(B - 1)
    out = {"frames_per_s": B / (ms / 1e3), "ms_per_step": ms, "steps": steps, "frames_per_step": B,
           "commit_pairs_per_step": B, "roots_nonzero": bool(ok),
           "what": "batched GKR input layer + ZK commit pair per frame (masked polynomial and mask, "
                   "tp_orion_commit_zk_pixels_dev) from resident bytes, pairs on %d side streams"
                   % len(zc.side)}
    del zc
    torch.cuda.empty_cache()
    if not args.skip_cpu:
        try:
            import multiprocessing as mp
            with mp.get_context("spawn").Pool(1, maxtasksperchild=1) as pool:
                secs, kind = pool.apply(_cpu_zk_commit, (0,))
            out["cpu_zk_commit"] = {"seconds_per_frame": secs, "cores": 1, "kind": kind,
                                    "sample": "one 1080p frame: Orion_zk commit_pair (masked polynomial "
                                              "and mask from a seed), one process"}
        except OSError as e:
            out["cpu_zk_commit"] = {"unavailable": str(e)}
    return out


def _cpu_opening(job):
    """The reference's own code for one opening-side row on one core (oracle/_ref,
    one fresh process per call): seconds of its work (ref_last_seconds), or None
    when the reference build is absent."""
    import ctypes
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from orionlib import ORION_REF_LIB, elements, virgo_inputs
    if not os.path.exists(ORION_REF_LIB):
        return None
    lib = ctypes.CDLL(ORION_REF_LIB)
    V = ctypes.c_void_p
    lib.ref_last_seconds.restype = ctypes.c_double
    kind, size = job
    if kind == "combine":
        lib.ref_combine.argtypes = [V, ctypes.c_longlong, V, V, V, V, V]
        lib.ref_encode_len.argtypes = [ctypes.c_longlong]
        lib.ref_encode_len.restype = ctypes.c_longlong
        src = elements(1, size)
        r0, r1 = elements(2, 128), elements(3, size // 128)
        comb = np.zeros(2 * lib.ref_encode_len(size // 128), np.uint64)
        ans = np.zeros(2, np.uint64)
        lib.ref_combine(V(src.ctypes.data), size, V(r0.ctypes.data), V(r1.ctypes.data), V(comb.ctypes.data),
                        ctypes.create_string_buffer(32), V(ans.ctypes.data))
    elif kind == "virgo":
        lib.ref_virgo_update.argtypes = [ctypes.c_int, V, V, V, ctypes.c_int, V, ctypes.c_int, V, V, V, V]
        vma, addv, ams, r = virgo_inputs(size, 4)
        outs = [np.zeros(4 * size, np.uint64) for _ in range(3)]
        ret = np.zeros(6, np.uint64)
        lib.ref_virgo_update(1, V(vma.ctypes.data), V(addv.ctypes.data), V(ams.ctypes.data), size,
                             V(r.ctypes.data), 1, *[V(o.ctypes.data) for o in outs], V(ret.ctypes.data))
    elif kind == "vinit":
        from orionlib import virgo_layer
        phase, lg, lu = size
        L = virgo_layer(71, lg, lu)
        lib.ref_virgo_init.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int] + [V] * 17
        outs = [np.zeros(4 << lu, np.uint64) for _ in range(3)]
        vp = lambda a: V(a.ctypes.data)
        lib.ref_virgo_init(phase, lg, lu, vp(L["ty"]), vp(L["u"]), vp(L["v"]), vp(L["comb_ptr"]), vp(L["comb_src"]),
                           vp(L["comb_w"]), vp(L["values"]), vp(L["r0"]), vp(L["r1"]), vp(L["alpha"]),
                           vp(L["beta"]), vp(L["vma0"]), vp(L["prev_r"]), vp(L["r_u"]), *[vp(o) for o in outs])
    else:
        lib.ref_fri_step.argtypes = [V, ctypes.c_int, V, V, V]
        w = elements(5, (1 << size) * 64)
        nxt = np.zeros(w.size // 2, np.uint64)
        lib.ref_fri_step(V(w.ctypes.data), size, V(elements(6, 1).ctypes.data), V(nxt.ctypes.data),
                         ctypes.create_string_buffer(32))
    return lib.ref_last_seconds()


def opening_bench(args, lib, committer, layout, dev, stream, sha_gcs, reps=5):
    """The opening-side rows on the device, each against its roofline, with the
    reference's CPU code for the same work timed beside it: the tensor-product
    passes over a resident 1080p codeword (combine, its Merkle tree, answer,
    queried columns), one Virgo sumcheck update and one FRI commit-phase step."""
    import torch
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from orionlib import elements, virgo_inputs
    peak, peak_kind = peaks()
    s = stream.cuda_stream
    N = layout.padded_copies * layout.n_wires
    cw, leaves = committer.cw_len[0], committer.leaves[0]
    rows = committer.rows[0]
    dt = lambda a: torch.from_numpy(a.view(np.int64)).to(dev)
    r0, r1 = dt(elements(2, 128)), dt(elements(3, N // 128))
    comb = torch.empty(2 * cw, dtype=torch.int64, device=dev)
    ctree = torch.empty(64 * leaves, dtype=torch.uint8, device=dev)
    ans = torch.empty(2, dtype=torch.int64, device=dev)
    q = torch.from_numpy(np.random.default_rng(7).integers(0, cw, size=1222, dtype=np.int64)).to(dev)
    qout = torch.empty(2 * 128 * 1222, dtype=torch.int64, device=dev)

    def timed(fn):
        with torch.cuda.stream(stream):
            fn()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(reps):
                fn()
            e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    def roof(bytes_, ms):
        gbs = bytes_ / (ms / 1e3) / 1e9
        return {"bound": "hbm", "achieved": gbs, "peak": peak, "unit": "GB/s", "frac": gbs / peak,
                "peak_source": peak_kind + " hbm_gbs" if peak_kind == "measured" else "fallback"}

    out = {}
    ms = timed(lambda: native.check(lib, lib.tp_orion_combine_dev(rows.data_ptr(), N, r0.data_ptr(),
                                                                  comb.data_ptr(), None, s), "combine"))
    out["combine"] = {"ms": ms, "rows": cw, "roofline": roof(cw * (2048 + 16), ms)}
    ms_t = timed(lambda: native.check(lib, lib.tp_orion_combine_dev(rows.data_ptr(), N, r0.data_ptr(),
                                                                    comb.data_ptr(), ctree.data_ptr(), s), "combine"))
    comp = 2 * leaves + 2 * (leaves - 1)
    out["combine_with_tree"] = {"ms": ms_t, "tree_ms": ms_t - ms, "leaves": leaves,
                                "g_compressions_per_s": comp / ((ms_t - ms) / 1e3) / 1e9,
                                "sha_peak_g_compressions_per_s": sha_gcs}
    ms = timed(lambda: native.check(lib, lib.tp_orion_answer_dev(comb.data_ptr(), N // 128, r1.data_ptr(),
                                                                 ans.data_ptr(), s), "answer"))
    out["answer"] = {"ms": ms, "roofline": roof(32 * (N // 128), ms)}
    t0 = time.perf_counter()
    for _ in range(reps):
        native.check(lib, lib.tp_orion_query_columns_dev(rows.data_ptr(), N, q.data_ptr(), 1222, qout.data_ptr(),
                                                         s), "query")
    out["query_1222_columns"] = {"ms": 1e3 * (time.perf_counter() - t0) / reps,
                                 "timer": "host wall clock (the call synchronises to check indices)"}
    del comb, ctree, qout

    n_v = 1 << 22
    vma, addv, ams, r = (dt(a) for a in virgo_inputs(n_v, 4))
    vouts = [torch.empty(4 * n_v // 2, dtype=torch.int64, device=dev) for _ in range(3)]
    ret = torch.empty(6, dtype=torch.int64, device=dev)
    rr = [int(x) for x in r.cpu().numpy().view(np.uint64)]
    ms = timed(lambda: native.check(lib, lib.tp_virgo_sumcheck_update_dev(
        vma.data_ptr(), addv.data_ptr(), ams.data_ptr(), n_v, rr[1], rr[0], 1, vouts[0].data_ptr(),
        vouts[1].data_ptr(), vouts[2].data_ptr(), ret.data_ptr(), s), "virgo"))
    out["virgo_update"] = {"ms": ms, "total_uv": n_v, "roofline": roof((192 + 96) * (n_v // 2), ms)}
    del vma, addv, ams, vouts

    # Virgo layer inits: 2^20 gates of every kind over 2^20 values
    from orionlib import virgo_layer
    import ctypes
    lgv = 20
    L = virgo_layer(71, lgv, lgv)
    vp = lambda a: ctypes.c_void_p(a.ctypes.data)
    h = lib.tp_virgo_layer_create(lgv, lgv, vp(L["ty"]), vp(L["u"]), vp(L["v"]), vp(L["comb_ptr"]),
                                  vp(L["comb_src"]), vp(L["comb_w"]))
    if not h:
        native.check(lib, -1, "virgo layer")
    vals = dt(L["values"])
    vouts = [torch.empty(4 << lgv, dtype=torch.int64, device=dev) for _ in range(3)]
    vma0 = dt(L["vma0"])
    ms1 = timed(lambda: native.check(lib, lib.tp_virgo_phase1_init_dev(
        h, vals.data_ptr(), vp(L["r0"]), vp(L["r1"]), vp(L["alpha"]), vp(L["beta"]),
        *[o.data_ptr() for o in vouts], s), "virgo phase1 init"))
    ms2 = timed(lambda: native.check(lib, lib.tp_virgo_phase2_init_dev(
        h, vals.data_ptr(), vp(L["r0"]), vp(L["r1"]), vp(L["alpha"]), vp(L["beta"]), vma0.data_ptr(),
        vp(L["prev_r"]), vp(L["r_u"]), *[o.data_ptr() for o in vouts], s), "virgo phase2 init"))
    lib.tp_virgo_layer_destroy(h)
    out["virgo_inits"] = {"phase1_ms": ms1, "phase2_ms": ms2, "gates": 1 << lgv, "values": 1 << lgv,
                          "what": "sumcheck_phase1_init / phase2_init of a seeded layer with every gate kind "
                                  "(tests/orionlib.py virgo_layer), tables written to HBM"}
    del vals, vouts, vma0

    lm = 18
    w = dt(elements(5, (1 << lm) * 64))
    nxt = torch.empty(w.numel() // 2, dtype=torch.int64, device=dev)
    ftree = torch.empty(64 * (1 << (lm - 2)), dtype=torch.uint8, device=dev)
    fr = [int(x) for x in elements(6, 1)]
    ms = timed(lambda: native.check(lib, lib.tp_fri_commit_step_dev(w.data_ptr(), lm, fr[1], fr[0], nxt.data_ptr(),
                                                                    ftree.data_ptr(), s), "fri step"))
    n_leaves = 1 << (lm - 2)
    comp = n_leaves * 128 + 2 * (n_leaves - 1)
    out["fri_step"] = {"ms": ms, "log_m": lm, "witness_elements": (1 << lm) * 64,
                       "g_compressions_per_s": comp / (ms / 1e3) / 1e9, "sha_peak_g_compressions_per_s": sha_gcs}
    del w, nxt, ftree
    torch.cuda.empty_cache()

    if not args.skip_cpu:
        import multiprocessing as mp
        jobs = [("combine", N), ("virgo", n_v), ("fri", lm), ("vinit", (1, lgv, lgv)), ("vinit", (2, lgv, lgv))]
        with mp.get_context("spawn").Pool(1, maxtasksperchild=1) as pool:
            secs = pool.map(_cpu_opening, jobs, chunksize=1)
        for (kind, _), sec, key in zip(jobs[:3], secs[:3], ("combine_with_tree", "virgo_update", "fri_step")):
            if sec is not None:
                out[key]["cpu_reference_ms"] = 1e3 * sec
                out[key]["speedup_vs_cpu_reference"] = 1e3 * sec / out[key]["ms"]
        if secs[3] is not None and secs[4] is not None:
            vi = out["virgo_inits"]
            vi["cpu_reference_phase1_ms"], vi["cpu_reference_phase2_ms"] = 1e3 * secs[3], 1e3 * secs[4]
            vi["speedup_vs_cpu_reference"] = (secs[3] + secs[4]) * 1e3 / (vi["phase1_ms"] + vi["phase2_ms"])
        out["cpu_note"] = ("reference sources (oracle/_ref/liborion_ref.so) on one core, same sizes: "
                           "combine + leaves + tree of a 2^23-element commit, phase-1 update of 2^22 "
                           "entries, FRI step of 2^18 x 64 elements, phase-1 / phase-2 inits of the 2^20-gate "
                           "layer")
    return out


def e2e_batched(args, bprover, committer, frames, z1s, z2s, pts, chal_b, stream, dev, world=1):
    """The batched path from pinned host frames: H2D of every frame's bytes, a D2H
    of all claims after every round with a synchronise, the commits, D2H of wires,
    MLEs and commitment roots."""
    import torch
    B = bprover.B
    host = [torch.from_numpy(f).pin_memory() for f in frames]
    dpix = [torch.empty_like(h, device=dev) for h in host]
    R = bprover.max_rounds
    claims_h = torch.zeros(B * 8, dtype=torch.int64).pin_memory()
    wires_h = torch.zeros_like(bprover.wires, device="cpu").pin_memory()
    mle_h = torch.zeros_like(bprover.mle, device="cpu").pin_memory()
    roots_h = torch.zeros(B * 32, dtype=torch.uint8).pin_memory()
    roots_d = torch.zeros(B * 32, dtype=torch.uint8, device=dev)

    def hook(k):
        claims_h.copy_(bprover.claims[k * B * 8:(k + 1) * B * 8], non_blocking=True)
        stream.synchronize()

    copy = torch.cuda.Stream(dev)
    landed = [torch.cuda.Event() for _ in range(B)]

    def one():
        # frames go up on a copy stream one by one; each frame's commit starts when
        # its own bytes have landed, the batched rounds when all have
        copy.wait_stream(stream)
        with torch.cuda.stream(copy):
            for d, h, ev in zip(dpix, host, landed):
                d.copy_(h, non_blocking=True)
                ev.record(copy)
        with torch.cuda.stream(stream):
            committer.commit(dpix, join=False, ready=landed)      # commits run under the rounds
            stream.wait_event(landed[-1])
            bprover.prove(dpix, z1s, z2s, pts, chal_b, round_hook=hook)
            committer.join()
            for f in range(B):
                roots_d[32 * f:32 * f + 32].copy_(committer.trees[f][32:64])
            wires_h.copy_(bprover.wires, non_blocking=True)
            mle_h.copy_(bprover.mle, non_blocking=True)
            roots_h.copy_(roots_d, non_blocking=True)
        stream.synchronize()

    one()
    steps = max(2, min(args.steps, 5))
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(steps):
        one()
    wall = time.perf_counter() - t0
    if world > 1:
        wall = max_over_ranks(1e3 * wall, world, dev) / 1e3
    h2d = sum(f.nbytes for f in frames)
    d2h = R * B * 64 + bprover.wires.numel() * 8 + bprover.mle.numel() * 8 + 32 * B
    return {"value": world * steps * B / wall, "unit": UNIT, "h2d_bytes_per_step": h2d,
            "d2h_bytes_per_step": d2h, "steps": steps, "frames_per_step": B,
            "timer": "host wall clock", "path": "tp_batch_* + tp_orion_commit_pixels_dev from "
            "pinned host frames (copied frame by frame on a copy stream; each commit starts when its "
            "frame has landed), claims read back every round, roots at the end"}


def e2e_c_abi(args, lib, pix, layout, gt, i0, i1, z1, z2, point, chal):
    """Same metric through the reference-facing C ABI with pinned host buffers."""
    import ctypes
    import torch
    C, W, nb = layout.padded_copies, layout.n_wires, layout.n_copy_bits
    table, inputs = host_tables(pix, layout)

    def pinned(a):
        t = torch.from_numpy(a.view(np.int64) if a.dtype == np.uint64 else a).pin_memory()
        return t

    t_re = pinned(table)
    t_im = pinned(np.zeros_like(table))
    t_in = pinned(inputs)
    b_re = torch.zeros(C, dtype=torch.int64).pin_memory()
    b_im = torch.zeros(C, dtype=torch.int64).pin_memory()
    w_re = torch.zeros(W, dtype=torch.int64).pin_memory()
    w_im = torch.zeros(W, dtype=torch.int64).pin_memory()
    out8 = torch.zeros(8, dtype=torch.int64).pin_memory()
    u = ctypes.POINTER(ctypes.c_uint64)
    P = lambda t: ctypes.cast(t.data_ptr(), u)
    arr = lambda a: a.ctypes.data_as(u)
    gti, i0i, i1i = (np.ascontiguousarray(x, np.int32) for x in (gt, i0, i1))
    ip = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))
    z1r, z1i = np.ascontiguousarray(z1[0]), np.ascontiguousarray(z1[1])
    z2r, z2i = np.ascontiguousarray(z2[:, 0]), np.ascontiguousarray(z2[:, 1])
    pr, pim = np.ascontiguousarray(point[:, 0]), np.ascontiguousarray(point[:, 1])
    mr, mi = ctypes.c_uint64(), ctypes.c_uint64()
    br1, bi1 = ctypes.c_uint64(), ctypes.c_uint64()
    elems = pinned(frame_elements(pix, layout))            # commit input, {img, real}
    n_el = C * W
    leaves = lib.tp_orion_tree_leaves(n_el)
    tree_h = torch.zeros(64 * leaves, dtype=torch.uint8).pin_memory()

    def one():
        lib.native_fp2_compute_beta(arr(z2r), arr(z2i), nb, 1, 0, P(b_re), P(b_im))
        h = lib.native_fp2_early_create(gti.size, ip(gti), ip(i0i), ip(i1i), arr(z1r), arr(z1i),
                                        C, W, P(t_re), P(t_im), P(b_re), P(b_im))
        assert h, lib.tp_last_error()
        for k in range(nb):
            assert lib.native_fp2_early_claim(h, P(out8)) == 0
            assert lib.native_fp2_early_fold(h, int(chal[k][0]), int(chal[k][1])) == 0
        assert lib.native_fp2_early_finish(h, P(w_re), P(w_im), ctypes.byref(br1),
                                           ctypes.byref(bi1)) == 0
        lib.native_fp2_early_destroy(h)
        lib.native_fp2_mle_eval_base(P(t_in), arr(pr), arr(pim), pr.size, ctypes.byref(mr),
                                     ctypes.byref(mi))
        assert lib.tp_last_error_code() == 0, lib.tp_last_error()
        assert lib.tp_orion_commit(elems.data_ptr(), n_el, tree_h.data_ptr(), None) == 0, \
            lib.tp_last_error()

    for _ in range(max(1, min(args.warmup, 3))):
        one()
    steps = max(3, min(args.steps, 10))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(steps):
        one()
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    h2d = 16 * W * C + 16 * C + 8 * W * C + 16 * (nb + point.shape[0] + z1.shape[1]) + 16 * n_el
    d2h = 16 * C + 64 * nb + 16 * (W + 1) + 16 + 64 * leaves
    return {"value": steps / wall, "unit": UNIT, "h2d_bytes_per_step": h2d,
            "d2h_bytes_per_step": d2h, "steps": steps, "timer": "host wall clock (synchronous API)",
            "path": "native_fp2_compute_beta/early_create/claim/fold/finish/mle_eval_base + "
                    "tp_orion_commit (the whole tree back), pinned host buffers"}


def reference_gpu_lib(frame, layout, gt, i0, i1, z1, z2, point, chal, reps=3):
    """The GKR part of one 1080p frame (compute_beta, early_create, 14 x claim +
    fold, finish, mle_eval_base) through the 14-symbol C ABI with host buffers,
    for the reference's own CUDA library (native_fp2.cu built for sm_100a,
    oracle/_ref/libnative_fp2_ref_gpu.so) and for ours, same inputs, same calls;
    outputs compared bit for bit. Host wall clock, synchronous API."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from fp2lib import GPU_LIB, REF_GPU_LIB, Fp2Lib, run_session
    if not os.path.exists(REF_GPU_LIB):
        return {"unavailable": "oracle/_ref/libnative_fp2_ref_gpu.so not built"}
    C, W, nb = layout.padded_copies, layout.n_wires, layout.n_copy_bits
    table, inputs = host_tables(frame, layout)
    zero = np.zeros_like(table)
    gti, i0i, i1i = (np.ascontiguousarray(x, np.int32) for x in (gt, i0, i1))
    z1r, z1i = np.ascontiguousarray(z1[0]), np.ascontiguousarray(z1[1])
    z2r, z2i = np.ascontiguousarray(z2[:, 0]), np.ascontiguousarray(z2[:, 1])
    pr, pim = np.ascontiguousarray(point[:, 0]), np.ascontiguousarray(point[:, 1])
    out, res, loop = {}, {}, {}
    for name, path in (("reference", REF_GPU_LIB), ("ours", GPU_LIB)):
        lib = Fp2Lib(path)
        lib.init()
        if lib.cuda_available() != 1:
            return {"unavailable": name + " library sees no CUDA device"}

        def one():
            bre, bim = lib.compute_beta(z2r, z2i, (1, 0))
            sess = run_session(lib, gti, i0i, i1i, z1r, z1i, C, W, table, zero, bre, bim, chal)
            return sess[:4], lib.mle_eval_base(inputs, pr, pim)

        res[name] = one()
        t0 = time.perf_counter()
        for _ in range(reps):
            one()
        out[name + "_frames_per_s"] = reps / (time.perf_counter() - t0)
        # the round loop alone on the resident session: the tables are on the
        # device after early_create (untimed); nb x (claim, fold), each call
        # returning when its kernels are done (both libraries' API is synchronous)
        bre, bim = lib.compute_beta(z2r, z2i, (1, 0))
        best = None
        for _ in range(reps):
            h = lib.early_create(gti, i0i, i1i, z1r, z1i, C, W, table, zero, bre, bim)
            t0 = time.perf_counter()
            for k in range(nb):
                lib.early_claim(h)
                lib.early_fold(h, chal[k])
            dt = time.perf_counter() - t0
            lib.early_destroy(h)
            best = dt if best is None else min(best, dt)
        loop[name] = 1e3 * best
    a, b = res["reference"], res["ours"]
    out["identical_outputs"] = bool(np.array_equal(a[0][0], b[0][0]) and np.array_equal(a[0][1], b[0][1])
                                    and np.array_equal(a[0][2], b[0][2]) and a[0][3] == b[0][3] and a[1] == b[1])
    out["ours_over_reference"] = out["ours_frames_per_s"] / out["reference_frames_per_s"]
    out["round_loop_ms"] = {"reference": loop["reference"], "ours": loop["ours"],
                            "reference_over_ours": loop["reference"] / loop["ours"],
                            "what": "%d x (claim, fold) on the session resident on the device (best of %d), "
                                    "host wall clock around the calls" % (nb, reps)}
    out["what"] = ("GKR input layer of one 1080p frame through the native_fp2 C ABI (host buffers, %d rounds): "
                   "the reference's native_fp2.cu (its build.sh recipe, -arch=sm_100a) vs ours" % nb)
    return out


def process_boundaries(frame, layout):
    """The Orion programs TruePix runs as subprocesses, on one 1080p frame: the
    reference's linearPC_multi_{commit,prove,open} (built from its sources in
    oracle/_ref, with its own ./fft_gkr) and ours (truepix_b200/bin), each a fresh
    process in a scratch directory with input.txt and the point file; wall clock
    per process, manifest roots and orion_proof.bin bytes compared."""
    import shutil
    import tempfile
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from clilib import env_for, lay_out, ours, reference, run, sha256_file
    if not os.path.exists(reference("linearPC_multi_prove")) or not os.path.exists(reference("linearPC_multi_open")):
        return {"unavailable": "oracle/_ref reference programs not built"}
    copies, cs, ci, cv = layout.copies, layout.copy_size, layout.const_idx, layout.const_val
    rng = np.random.default_rng(SEED + 7)
    point = rng.integers(0, P61, size=(layout.n_in_bits + layout.n_copy_bits, 2), dtype=np.uint64)
    out = {"workload": "one 1080p frame (%d copies of %d bytes), gray layout; fresh process per phase" % (copies, cs)}
    files = {}
    for who, prog, fft in (("reference", reference, reference("fft_gkr")), ("ours", ours, ours("fft_gkr"))):
        d = tempfile.mkdtemp(prefix="tp_programs_")
        try:
            lay_out(d, frame, copies, cs, [(int(a), int(b)) for a, b in point])
            os.symlink(fft, os.path.join(d, "fft_gkr"))
            env = env_for(d, cs, ci, cv, TRUEPIX_ORION_RESULT_FILE=os.path.join(d, "result.json"))
            t = {}
            for phase in ("commit", "prove", "open"):
                t0 = time.perf_counter()
                r = run(prog("linearPC_multi_" + phase), d, env, copies, 0, timeout=1800)
                t[phase + "_s"] = time.perf_counter() - t0
                if r.returncode != 0 or "check pass" not in r.stdout and phase != "commit":
                    return {"unavailable": "%s %s failed: %s" % (who, phase, (r.stdout + r.stderr)[-300:])}
            files[who] = (json.load(open(os.path.join(d, "orion_commit.json")))["masked_root"],
                          sha256_file(os.path.join(d, "orion_proof.bin")),
                          json.load(open(os.path.join(d, "result.json"))))
            out[who] = t
        finally:
            shutil.rmtree(d, ignore_errors=True)
    out["same_root_proof_and_result"] = files["reference"] == files["ours"]
    out["reference_over_ours"] = {k: out["reference"][k] / out["ours"][k] for k in out["ours"]}
    return out


def _serving_job(device):
    import torch
    torch.cuda.set_device(device)
    uneven = batched_uneven()
    uneven["graph_early_rounds"] = uneven_graph()
    return uneven, serving_sweep()


def serving_in_own_process(device):
    """Configs 4 and 5 in a fresh process on the same GPU: their latencies then do
    not depend on what this process left in the device's pools and caches (the
    step's batch, the committers, other libraries loaded for the comparisons)."""
    import multiprocessing as mp
    with mp.get_context("spawn").Pool(1, maxtasksperchild=1) as pool:
        return pool.apply(_serving_job, (device,))


def release(srv):
    """Free a server's device memory before the next measurement (outside it)."""
    import gc
    import torch
    srv.close()
    gc.collect()
    torch.cuda.synchronize()
    torch.cuda.empty_cache()


def transcript_rounds(bprover, pix, z1s, z2s, pts, stream, reps=3):
    """The batched GKR input layer of the step's 64 frames with a Fiat-Shamir
    transcript per frame (the reference's binary format, tp_fs_*): (host) every
    round the claims come back to the host, each frame's host transcript puts
    them and draws the fold challenge; (device) the transcripts live on the
    device and the same happens there (tp_fs_*_dev, tp_batch_fold_dev). Host
    wall clock per batch; both give the same challenges."""
    import ctypes
    import torch
    lib = bprover.lib
    B, R = bprover.B, bprover.max_rounds
    nbytes = lib.tp_fs_state_bytes()
    states = []
    for f in range(B):
        st = ctypes.create_string_buffer(nbytes)
        lib.tp_fs_init(st, b"truepix")
        v = np.array([f], np.uint64)
        lib.tp_fs_put_u64s(st, v.ctypes.data, 1)
        states.append(st)
    init = b"".join(st.raw for st in states)
    chal = np.zeros((R, B, 2), np.uint64)
    claims_h = torch.zeros(B * 8, dtype=torch.int64).pin_memory()
    re, im = ctypes.c_uint64(), ctypes.c_uint64()
    hs = []

    def hook(k):
        claims_h.copy_(bprover.claims[k * B * 8:(k + 1) * B * 8], non_blocking=True)
        stream.synchronize()
        cl = claims_h.numpy().view(np.uint64).reshape(B, 4, 2)
        label = ("sc-0-%d" % k).encode()
        for f in range(B):
            r, i = np.ascontiguousarray(cl[f, :, 0]), np.ascontiguousarray(cl[f, :, 1])
            lib.tp_fs_put_fp2s(hs[f], r.ctypes.data, i.ctypes.data, 4)
            lib.tp_fs_rand_ext(hs[f], label, ctypes.byref(re), ctypes.byref(im))
            chal[k, f] = (re.value, im.value)

    d_states = torch.empty(B * nbytes, dtype=torch.uint8, device=bprover.dev)
    init_t = torch.from_numpy(np.frombuffer(init, np.uint8).copy())

    def host_run():
        hs[:] = [ctypes.create_string_buffer(init[f * nbytes:(f + 1) * nbytes], nbytes) for f in range(B)]
        with torch.cuda.stream(stream):
            bprover.prove(pix, z1s, z2s, pts, chal, round_hook=hook)
        stream.synchronize()

    def dev_run():
        with torch.cuda.stream(stream):
            d_states.copy_(init_t, non_blocking=True)
            bprover.prove(pix, z1s, z2s, pts, None, transcripts=d_states)
        stream.synchronize()

    count = 4 * R
    vole = dict(states=torch.empty(B * lib.tp_vole_state_bytes(), dtype=torch.uint8, device=bprover.dev),
                u=torch.randint(0, P61, (B * count * 2,), dtype=torch.int64, device=bprover.dev),
                v=torch.randint(0, P61, (B * count * 2,), dtype=torch.int64, device=bprover.dev), count=count)
    vs = ctypes.create_string_buffer(lib.tp_vole_state_bytes())
    lib.tp_vole_state_init(vs, 0, None)
    vole_init = torch.from_numpy(np.frombuffer(vs.raw * B, np.uint8).copy())

    def vole_run():
        with torch.cuda.stream(stream):
            d_states.copy_(init_t, non_blocking=True)
            vole["states"].copy_(vole_init, non_blocking=True)
            bprover.prove(pix, z1s, z2s, pts, None, transcripts=d_states, vole=vole)
        stream.synchronize()

    out = {}
    for name, fn in (("host_transcripts", host_run), ("device_transcripts", dev_run),
                     ("device_vole_rounds", vole_run)):
        fn()
        t0 = time.perf_counter()
        for _ in range(reps):
            fn()
        out[name + "_frames_per_s"] = reps * B / (time.perf_counter() - t0)
    dev_run()
    got = bprover.device_challenges.cpu().numpy().view(np.uint64).reshape(R, B, 2)
    out["same_challenges"] = bool(np.array_equal(got, chal))
    out["what"] = ("batched GKR input layer of %d 1080p frames (%d rounds, beta, MLE) with one Fiat-Shamir "
                   "transcript per frame: claims read back and challenges drawn on the host every round, vs "
                   "put and drawn on the device; and the reference prover's VOLE-committed round on the device "
                   "(interpolation, commitments, equality proof, challenge); host wall clock" % (B, R))
    return out


def pinned_frame(a):
    """A frame as the serving loop takes it from a decoder: pinned host memory
    (copied straight to the device, no staging copy on the host)."""
    import torch
    return torch.from_numpy(a).pin_memory()


def serving_circuits():
    from truepix_b200.serving import Circuit
    c = np.load(os.path.join(ROOT, "tests", "golden", "circuits.npz"))
    g = lambda n: (c[n + "_type"], c[n + "_in0"], c[n + "_in1"])
    return {"gray": Circuit("gray", *g("gray"), 384, 384, 128),
            "mask": Circuit("mask", *g("mask"), 384, -1, 0),
            "crop": Circuit("crop", *g("Crop"), 385, -1, 0)}


def _correlations(rng, circuit, h, w):
    from truepix_b200.pipeline import correlations_needed
    from truepix_b200.serving import layout_for
    count = correlations_needed(layout_for(circuit, h, w))
    return (rng.integers(0, P61, size=(count, 2), dtype=np.uint64),
            rng.integers(0, P61, size=(count, 2), dtype=np.uint64))


def batched_uneven(seed=4):
    """64 crop-then-gray frames of uneven size proven together: sources 240p to
    1080p (16:9), crop fractions x1 < x2, y1 < y2 uniform in [0, 1] (seeded); the
    cropped region goes through the gray circuit (2^14 .. 2^23 input wires). All 64
    queued at once into the serving loop: one claim launch and one VOLE-round
    launch per tick for every frame in its early rounds, each at its own round;
    every frame leaves with its whole proof."""
    from truepix_b200.serving import ProofServer, Request, latency_stats
    rng = np.random.default_rng(seed)
    gray = serving_circuits()["gray"]
    heights = [240, 360, 480, 720, 1080]
    reqs = []
    for i in range(64):
        h = int(rng.choice(heights))
        w = (h * 16 + 8) // 9
        x = np.sort(rng.random(2))
        y = np.sort(rng.random(2))
        cw, ch = max(1, int(round((x[1] - x[0]) * w))), max(1, int(round((y[1] - y[0]) * h)))
        reqs.append(Request(i, gray, ch, cw, pinned_frame(rng.integers(0, 256, size=ch * cw * 3, dtype=np.uint8)),
                            pid=9000 + i, correlations=_correlations(rng, gray, ch, cw), arrival=0.0))
    srv = ProofServer(slots=64, hbm_budget=80e9, max_height=1080, max_width=1920)
    srv.run(reqs, realtime=False)                  # warm-up: every size's expander graphs, pools
    t0 = srv.ticks
    res = srv.run(reqs, realtime=False)
    st = latency_stats(res)
    ticks = srv.ticks - t0
    release(srv)
    wires = sorted(1 << (9 + int(np.log2(max(2, 1 << int(np.ceil(np.log2(max(2, -(-r.height * r.width * 3 // 384)))))))))
                   for r in reqs)
    return {"workload": "64 crop-then-gray frames, sources 240p-1080p, seeded crops", "frames": len(res),
            "frames_per_s": st.get("frames_per_s"), "p50_ms": st.get("p50_ms"), "p99_ms": st.get("p99_ms"),
            "input_wires_min": wires[0], "input_wires_max": wires[-1], "ticks": ticks,
            "what": "whole proofs (proof container + Orion opening file) of 64 uneven frames, continuous batch "
                    "of 64 slots on device transcripts"}


def uneven_graph(seed=4, reps=10):
    """The early rounds of the same 64 uneven crop-then-gray frames as one CUDA
    graph per batch (tp_batch_vole_rounds_graph): per round one claim launch per
    source kind for every frame still in its rounds, one VOLE-committed round on
    the frames' device transcripts (frames past their last round skip it) and the
    folds by the drawn challenges; then the finish, beta and MLE. Captured on the
    first call, replayed after (transcripts and VOLE states reset before each
    replay, inside the timed region); CUDA events on the batch's stream."""
    import ctypes
    import torch
    from truepix_b200.frame import BatchFrameProver, pack_fp2
    from truepix_b200.pipeline import correlations_needed
    from truepix_b200.serving import layout_for
    rng = np.random.default_rng(seed)
    gray = serving_circuits()["gray"]
    heights = [240, 360, 480, 720, 1080]
    dev = torch.device("cuda", torch.cuda.current_device())
    layouts, frames = [], []
    for i in range(64):                 # the draws of batched_uneven: same crops, same bytes
        h = int(rng.choice(heights))
        w = (h * 16 + 8) // 9
        x = np.sort(rng.random(2))
        y = np.sort(rng.random(2))
        cw, ch = max(1, int(round((x[1] - x[0]) * w))), max(1, int(round((y[1] - y[0]) * h)))
        L = layout_for(gray, ch, cw)
        t = torch.zeros(L.copies * L.copy_size, dtype=torch.uint8, device=dev)
        t[:ch * cw * 3] = torch.from_numpy(rng.integers(0, 256, size=ch * cw * 3, dtype=np.uint8)).to(dev)
        _correlations(rng, gray, ch, cw)
        layouts.append(L)
        frames.append(t)
    B = len(layouts)
    gt, i0, i1 = (np.ascontiguousarray(a, np.int32) for a in (gray.gate_type, gray.in0, gray.in1))
    zg = [np.stack([rng.integers(0, P61, size=gt.size, dtype=np.uint64),
                    rng.integers(0, P61, size=gt.size, dtype=np.uint64)]) for _ in range(B)]
    z2d, ptd = {}, {}
    for C in sorted({L.padded_copies for L in layouts}):
        n = sum(1 for L in layouts if L.padded_copies == C)
        nb = int(np.log2(C))
        z2d[C] = torch.from_numpy(pack_fp2(rng.integers(0, P61, size=n * nb, dtype=np.uint64),
                                           rng.integers(0, P61, size=n * nb, dtype=np.uint64))).to(dev)
        ptd[C] = torch.zeros(2 * n * (9 + nb), dtype=torch.int64, device=dev)
    stream = torch.cuda.Stream(dev)
    bp = BatchFrameProver(layouts, gt, i0, i1, stream=stream)
    lib = bp.lib
    count = max(correlations_needed(L) for L in layouts)
    st0 = []
    for f in range(B):
        st = ctypes.create_string_buffer(lib.tp_fs_state_bytes())
        lib.tp_fs_init(st, b"truepix")
        lib.tp_fs_put_u64s(st, np.array([f], np.uint64).ctypes.data, 1)
        st0.append(st.raw)
    vs = ctypes.create_string_buffer(lib.tp_vole_state_bytes())
    lib.tp_vole_state_init(vs, 0, None)
    init_st = torch.from_numpy(np.frombuffer(b"".join(st0), np.uint8).copy()).to(dev)
    init_vs = torch.from_numpy(np.frombuffer(vs.raw * B, np.uint8).copy()).to(dev)
    d_st, d_vs = init_st.clone(), init_vs.clone()
    vole = dict(states=d_vs, u=torch.from_numpy(rng.integers(0, P61, size=B * count * 2, dtype=np.uint64).view(
        np.int64)).to(dev), v=torch.from_numpy(rng.integers(0, P61, size=B * count * 2, dtype=np.uint64).view(
            np.int64)).to(dev), count=count)

    def once():
        with torch.cuda.stream(stream):
            d_st.copy_(init_st, non_blocking=True)
            d_vs.copy_(init_vs, non_blocking=True)
            bp.prove(frames, zg, z2d, ptd, None, transcripts=d_st, vole=vole, graph=True)

    for _ in range(3):
        once()
    stream.synchronize()
    l0 = lib.tp_batch_launches(bp.handle)
    r0 = lib.tp_batch_graph_replays(bp.handle)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        once()
    e1.record(stream)
    stream.synchronize()
    ms = e0.elapsed_time(e1) / reps
    rounds = sorted({L.n_copy_bits for L in layouts})
    return {"frames_per_s": B / (ms / 1e3), "ms_per_batch": ms, "reps": reps,
            "graph_replays": lib.tp_batch_graph_replays(bp.handle) - r0,
            "kernels_per_replay": (lib.tp_batch_launches(bp.handle) - l0) / reps,
            "rounds_min": rounds[0], "rounds_max": rounds[-1],
            "what": "the early rounds (VOLE-committed, device transcripts) of the same 64 uneven frames as one "
                    "CUDA graph per batch, replayed; plus beta and MLE"}


def serving_sweep(rates=(100, 250, 500, 1000), n_req=192, seed=5):
    """Poisson arrivals of gray / crop / mask proofs of 360p .. 2160p frames at rate
    lambda (frames/s), real time, admission by HBM footprint (60 GB budget); frames
    in pinned host memory; every request leaves with its whole proof."""
    from truepix_b200.serving import ProofServer, Request, latency_stats
    cs = serving_circuits()
    sizes = [(360, 640), (480, 854), (720, 1280), (1080, 1920), (1440, 2560), (2160, 3840)]
    rng = np.random.default_rng(seed)
    frames = {hw: [pinned_frame(rng.integers(0, 256, size=hw[0] * hw[1] * 3, dtype=np.uint8)) for _ in range(2)]
              for hw in sizes}
    srv = ProofServer(slots=64, hbm_budget=60e9)
    out = []
    runs = []
    corr = {}
    for lam in rates:
        t = 0.0
        reqs = []
        for i in range(n_req):
            t += rng.exponential(1.0 / lam)
            hw = sizes[int(rng.integers(len(sizes)))]
            op = ["gray", "crop", "mask"][int(rng.integers(3))]
            if (op, hw) not in corr:
                corr[(op, hw)] = _correlations(rng, cs[op], hw[0], hw[1])
            reqs.append(Request(i, cs[op], hw[0], hw[1], frames[hw][i % 2], pid=77 + i, correlations=corr[(op, hw)],
                                arrival=t))
        runs.append((lam, reqs))
    # warm-up: one rate's requests all at once (every size's graphs, the pools
    # grown to a full batch's footprint)
    import dataclasses
    srv.run([dataclasses.replace(r) for r in runs[-1][1]], realtime=False)
    for lam, reqs in runs:
        res = srv.run(reqs, realtime=True)
        st = latency_stats(res)
        st["lambda_per_s"] = lam
        out.append(st)
    release(srv)
    return {"workload": "Poisson requests, ops gray/crop/mask uniform, 360p-2160p uniform, %d per rate, "
                        "frames in pinned host memory, whole proofs" % n_req,
            "slots": 64, "hbm_budget_gb": 60, "by_rate": out}


def profile_case(name):
    """A short fixed workload for `ncu` captures (no timing, no JSON line):
    orion = one 1080p Orion commit from bytes, one RS commit of 2^20 elements and
    one 2^24-point forward NTT, through include/orion_gpu.h; proved = two batches of
    16 1080p frames through the pipelined whole proof after two warm-up batches
    (the profiler API brackets the measured two: ncu --profile-from-start off);
    refgpu = one 1080p frame's GKR session through the native_fp2 C ABI, the
    reference's CUDA library, then ours."""
    import torch
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from orionlib import elements
    from truepix_b200.frame import FrameLayout
    if name == "refgpu":
        # one 1080p frame's GKR session through the native_fp2 C ABI: the
        # reference's CUDA library, then ours (kernel-against-kernel launch lists)
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        from fp2lib import GPU_LIB, REF_GPU_LIB, Fp2Lib, run_session
        L = FrameLayout.for_frame(H, Wd)
        gt, i0, i1 = circuit()
        frames, z1, z2, _, chal = make_inputs(np.random.default_rng(SEED), L, 1)
        table, _ = host_tables(frames[0], L)
        zero = np.zeros_like(table)
        g = [np.ascontiguousarray(x, np.int32) for x in (gt, i0, i1)]
        for path in (REF_GPU_LIB, GPU_LIB):
            lib = Fp2Lib(path)
            lib.init()
            bre, bim = lib.compute_beta(np.ascontiguousarray(z2[:, 0]), np.ascontiguousarray(z2[:, 1]), (1, 0))
            run_session(lib, *g, np.ascontiguousarray(z1[0]), np.ascontiguousarray(z1[1]), L.padded_copies,
                        L.n_wires, table, zero, bre, bim, chal)
        torch.cuda.synchronize()
        return
    if name == "proved":
        # two batches of 16 1080p frames through the pipelined whole proof (truepix_b200.pipeline)
        from truepix_b200.frame import FrameLayout
        from truepix_b200.pipeline import ProofPipeline
        L = FrameLayout.for_frame(H, Wd)
        gt, i0, i1 = circuit()
        frames, corr = proved_inputs(np.random.default_rng(SEED), L, 16)
        pipe = ProofPipeline(L, gt, i0, i1, batch=16)
        batch = dict(frames_host=frames, pids=list(range(16)), correlations=corr)
        for _ in pipe.run([batch, batch]):          # the round autotuner and the graph capture
            pass
        torch.cuda.synchronize()
        torch.cuda.profiler.start()                 # ncu --profile-from-start off: the steady state only
        for _ in pipe.run([batch, batch]):
            pass
        torch.cuda.synchronize()
        torch.cuda.profiler.stop()
        pipe.close()
        return
    assert name == "orion", name
    lib = native.gkr()
    dev = torch.device("cuda", 0)
    s = torch.cuda.current_stream().cuda_stream
    L = FrameLayout.for_frame(H, Wd)
    n = L.padded_copies * L.n_wires
    cw_len, leaves = lib.tp_orion_codeword_len(n // 128), lib.tp_orion_tree_leaves(n)
    rng = np.random.default_rng(SEED)
    pix = torch.from_numpy(rng.integers(0, 256, size=L.copies * L.copy_size, dtype=np.uint8)).to(dev)
    rows = torch.empty(2 * 128 * cw_len, dtype=torch.int64, device=dev)
    tree = torch.empty(64 * leaves, dtype=torch.uint8, device=dev)
    native.check(lib, lib.tp_orion_commit_pixels_dev(pix.data_ptr(), L.copies, L.padded_copies, L.copy_size,
                                                     L.n_wires, L.const_idx, L.const_val, rows.data_ptr(),
                                                     tree.data_ptr(), s), "commit")
    lg = 20
    a = torch.from_numpy(elements(2, 1 << lg).view(np.int64)).to(dev)
    cw = torch.empty(2 << (lg + 5), dtype=torch.int64, device=dev)
    rt = torch.empty(32 << (lg - 1), dtype=torch.uint8, device=dev)
    native.check(lib, lib.tp_rs_commit_dev(a.data_ptr(), lg, cw.data_ptr(), rt.data_ptr(), s), "rs commit")
    m = 1 << 24
    b = torch.from_numpy(elements(1, m).view(np.int64)).to(dev)
    out = torch.empty_like(b)
    native.check(lib, lib.tp_fft_dev(b.data_ptr(), m, m, out.data_ptr(), 1, 0, 0, s), "fft")
    torch.cuda.synchronize()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--batch", type=int, default=64)
    ap.add_argument("--no-plain", action="store_true", help="skip the single-frame measurement")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--skip-e2e", action="store_true")
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--skip-ntt", action="store_true")
    ap.add_argument("--skip-serving", action="store_true")
    ap.add_argument("--skip-zk", action="store_true")
    ap.add_argument("--skip-opening", action="store_true")
    ap.add_argument("--leaf-chunks", type=int, default=1,
                    help="launches the commits' SHA-256 leaf chains are split into (tp_orion_set_leaf_chunks)")
    ap.add_argument("--commit-streams", type=int, default=8,
                    help="streams the step's commits are spread over (0: the step's stream)")
    ap.add_argument("--profile-case", choices=["orion", "proved", "refgpu"],
                    help="run a fixed short workload for ncu and exit")
    args = ap.parse_args()
    if args.profile_case:
        profile_case(args.profile_case)
        return
    args.warmup = max(3, args.warmup)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        reference_arm(args, rank, world)
        return
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        ours_arm(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
