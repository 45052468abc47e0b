"""Benchmark: proved 1080p frames/s on one B200 (GKR input layer of the gray circuit).

Workload: seeded 1920x1080x3 uint8 frames; each frame is 16,200 copies of 384
bytes padded to 16,384 x 512 input wires (2^23) and is proven by the
device-resident path (truepix_b200.frame): beta over the 14 copy challenges, 14
early sumcheck rounds (claim + fold; rounds 0 and 1 read the frame's bytes),
finish, and the MLE of the 2^23-entry input vector at the final point.

One step = one batch of B frames (default 64) proven together, one kernel
launch per round for the whole batch (BatchFrameProver). Inputs stay in HBM:
B distinct frames (400 MB of bytes) and their folded tables (~4.8 GB) are far
larger than the 126 MB L2, so no flush is needed.

  value         frames/s over all ranks, device time (CUDA events), batched
  plain         frames/s of single-frame proofs (one session per frame), same
                device timing -- the batched/plain ratio is reported
  e2e           the batched path from pinned host frames: H2D of the bytes, and
                every round a D2H of all claims with a synchronise (the host
                needs them for its transcript) inside the timed region
  e2e_reference_abi  one frame through the reference C ABI (native_fp2_*) with
                pinned host SoA tables
  roofline      the claim kernel with the largest share: algorithmic bytes (per
                launch kind, see kernel_groups) / its event-timed duration,
                against MEASURED_PEAKS.json
  cpu_baseline  the reference CPU library (built from the reference's source)
                proving one frame of the same workload on one host core

`--impl reference` times that reference CPU library on all host cores instead
(one frame per worker process per step) and prints the same metric.
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

METRIC = "1080p proved frames/s (GKR input layer, gray circuit)"
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
# CPU side: reference library (oracle/_ref, built from the reference source) or
# the oracle port when that build is absent.

def cpu_lib():
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from fp2lib import Fp2Lib, REF_LIB, ORACLE_LIB
    if os.path.exists(REF_LIB):
        return Fp2Lib(REF_LIB, "native_fp2_"), "reference"
    if not os.path.exists(ORACLE_LIB):
        subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "all"])
    return Fp2Lib(ORACLE_LIB, "oracle_fp2_"), "port"


def cpu_prove_frame(lib, gt, i0, i1, z1, z2, point, chal, table, inputs, layout):
    from fp2lib import run_session
    C, W = layout.padded_copies, layout.n_wires
    bre, bim = lib.compute_beta(np.ascontiguousarray(z2[:, 0]), np.ascontiguousarray(z2[:, 1]),
                                (1, 0))
    run_session(lib, gt, i0, i1, z1[0], z1[1], C, W, table, np.zeros_like(table), bre, bim, chal)
    lib.mle_eval_base(inputs, np.ascontiguousarray(point[:, 0]), np.ascontiguousarray(point[:, 1]))


def _cpu_worker(args):
    idx, n_frames = args
    from truepix_b200.frame import FrameLayout
    layout = FrameLayout.for_frame(H, Wd)
    rng = np.random.default_rng(SEED + idx)
    frames, z1, z2, point, chal = make_inputs(rng, layout, 1)
    table, inputs = host_tables(frames[0], layout)
    lib, kind = cpu_lib()
    gt, i0, i1 = circuit()
    t0 = time.perf_counter()
    for _ in range(n_frames):
        cpu_prove_frame(lib, gt, i0, i1, z1, z2, point, chal, table, inputs, layout)
    return time.perf_counter() - t0, kind


def reference_arm(args, rank, world):
    """The reference CPU implementation on all host cores (rank 0 only)."""
    if rank != 0:
        return
    import multiprocessing as mp
    workers = max(1, min(os.cpu_count() or 1, 64))
    ctx = mp.get_context("spawn")
    with ctx.Pool(workers) as pool:
        for _ in range(args.warmup and 1):      # one warm-up frame per worker
            pool.map(_cpu_worker, [(i, 1) for i in range(workers)])
        t0 = time.perf_counter()
        res = pool.map(_cpu_worker, [(i, args.steps) for i in range(workers)])
        wall = time.perf_counter() - t0
    kind = res[0][1]
    frames = workers * args.steps
    value = frames / wall
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * wall / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64 (Fp2)",
        "data": "synthetic",
        "config": {"workload": "gkr_input_layer_gray_1080p", "frame": [H, Wd, 3],
                   "copies": 16200, "wires": 1 << 23, "circuit": "gray.pws"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": workers, "kind": kind,
                         "sample": f"{args.steps} frames per worker process x {workers} processes"},
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


def kernel_groups(ms, tags, layout, batch=1):
    """Per claim-kernel kind: launches, total time, algorithmic bytes, folded elements.
    tag = 1000*(reads bytes) + 100*(fold fused) + log2(copies claimed per frame).
    Algorithmic bytes per frame: bytes read once + folded Fp2 rows written (16 B
    per element) + table rows read (16 B per element) + beta."""
    rows = layout.const_idx + 1 if layout.const_idx >= 0 else layout.copy_size
    pix_bytes = layout.copies * layout.copy_size
    groups = {}
    for t, tag in zip(ms, tags):
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
                                     "by_copies": {}})
        g["launches"] += 1
        g["ms"] += t
        g["bytes"] += byt * batch
        g["folded"] += el * batch
        bc = g["by_copies"].setdefault(n, [0, 0.0])
        bc[0] += 1
        bc[1] += t
    return groups


def ours_arm(args, rank, world, local_rank):
    import ctypes
    import torch
    import torch.distributed as dist
    from truepix_b200 import native
    from truepix_b200.frame import BatchFrameProver, FrameLayout, GkrInputLayerProver, pack_fp2

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    layout = FrameLayout.for_frame(H, Wd)
    gt, i0, i1 = circuit()
    B = args.batch
    nb = layout.n_copy_bits
    rng = np.random.default_rng(SEED + 101 * rank)
    frames, z1, z2, point, chal = make_inputs(rng, layout, B)
    pix = [torch.from_numpy(f).to(dev) for f in frames]
    z2_dev = torch.from_numpy(pack_fp2(z2[:, 0], z2[:, 1])).to(dev)
    pt_dev = torch.from_numpy(pack_fp2(point[:, 0], point[:, 1])).to(dev)
    chal_b = np.ascontiguousarray(np.broadcast_to(chal[:, None, :], (nb, B, 2)))
    stream = torch.cuda.Stream(dev)
    lib = native.gkr()
    bprover = BatchFrameProver([layout] * B, gt, i0, i1, device=local_rank, stream=stream)
    z1s = [z1] * B
    z2s = z2_dev.repeat(B)      # packed [B][nb]
    pts = pt_dev.repeat(B)      # packed [B][9 + nb]

    def run_batch(hook=None):
        bprover.prove(pix, z1s, z2s, pts, chal_b, round_hook=hook)

    # ---- plain single-frame proofs (the baseline of the batched/plain ratio)
    plain = GkrInputLayerProver(layout, gt, i0, i1, device=local_rank, stream=stream)
    n_plain = 0 if args.no_plain else max(10, min(200, 4 * B))
    plain_fps = None
    if n_plain:
        with torch.cuda.stream(stream):
            for i in range(5):
                plain.prove(pix[i % B], z1, z2_dev, pt_dev, chal)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for i in range(n_plain):
                plain.prove(pix[i % B], z1, z2_dev, pt_dev, chal)
            e1.record(stream)
        torch.cuda.synchronize()
        plain_fps = n_plain / (e0.elapsed_time(e1) / 1e3)

    # ---- batched: the timed region
    with torch.cuda.stream(stream):
        for i in range(args.warmup):
            run_batch()
    torch.cuda.synchronize()
    native.check(lib, lib.tp_timer_enable(args.steps * nb * 2 + 16), "timer")
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
            launches += bprover.launches_last
            evs[i + 1].record(stream)
    torch.cuda.synchronize()
    clk.t1 = time.time()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clk.stop()
    npairs = args.steps * nb * 2 + 16
    tms = (ctypes.c_float * npairs)()
    ttags = (ctypes.c_int * npairs)()
    got = lib.tp_timer_read(tms, ttags, npairs)
    lib.tp_timer_disable()
    ms = evs[0].elapsed_time(evs[-1])
    per_batch = sorted(evs[i].elapsed_time(evs[i + 1]) for i in range(args.steps))
    t = torch.tensor([ms], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms = float(t.item())
    frames_done = args.steps * B
    value = world * frames_done / (ms / 1e3)

    groups = kernel_groups(list(tms[:max(0, got)]), list(ttags[:max(0, got)]), layout, B)
    peak, peak_kind = peaks()
    kernels = []
    for name, g in sorted(groups.items(), key=lambda kv: -kv[1]["ms"]):
        ach = g["bytes"] / (g["ms"] / 1e3) / 1e9 if g["ms"] > 0 else None
        kernels.append({"kernel": name, "launches": g["launches"], "total_ms": g["ms"],
                        "share_of_step": g["ms"] / ms, "achieved_gbs": ach,
                        "avg_us_by_copies": {str(k): round(1e3 * v[1] / v[0], 2)
                                             for k, v in sorted(g["by_copies"].items())}})
    roof = None
    traffic = profiled_traffic()
    if kernels:
        top = kernels[0]
        g = groups[top["kernel"]]
        roof = {"kernel": top["kernel"], "bound": "hbm", "achieved": top["achieved_gbs"],
                "peak": peak, "unit": "GB/s",
                "frac": top["achieved_gbs"] / peak if top["achieved_gbs"] else None,
                "peak_source": (peak_kind + " hbm_gbs (MEASURED_PEAKS.json)") if peak_kind == "measured"
                else "fallback 6650 GB/s",
                "algorithmic_bytes_per_launch": g["bytes"] / g["launches"],
                "avg_launch_us": 1e3 * g["ms"] / g["launches"], "launches_timed": g["launches"],
                "traffic": (traffic or {}).get(top["kernel"]),
                "all_claim_kernels": kernels}
    folded = sum(g["folded"] for g in groups.values())

    res_ok = None
    if rank == 0:
        c, w, b, m = bprover.results(B - 1)
        res_ok = bool(c.any() and w.any() and m != (0, 0))

    e2e = e2e_ref = cpu = None
    if rank == 0 and not args.skip_e2e:
        e2e = e2e_batched(args, bprover, frames, z1s, z2s, pts, chal_b, stream, dev)
        e2e_ref = e2e_c_abi(args, lib, frames[0], layout, gt, i0, i1, z1, z2, point, chal)
    if rank == 0 and world == 1 and not args.skip_cpu:
        secs, kind = _cpu_worker((0, 1))
        cpu = {"value": 1.0 / secs, "unit": UNIT, "cores": 1, "kind": kind,
               "sample": "1 frame of the same workload (compute_beta + 14 early rounds + finish "
                         "+ MLE over 2^23 inputs), library calls only, one process"}
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "u64 (Fp2 over 2^61-1)", "data": "synthetic",
            "config": {"workload": "gkr_input_layer_gray_1080p", "frame": [H, Wd, 3],
                       "copies": layout.copies, "padded_copies": layout.padded_copies,
                       "wires": layout.padded_copies * layout.n_wires, "rounds": nb,
                       "circuit": "gray.pws", "batch": B, "step": f"one batch of {B} frames",
                       "path": "bytes -> batched rounds (tp_batch_*)",
                       "l2": "inputs > L2: B distinct frames (0.4 GB) and their folded "
                             "tables (~4.8 GB) per step",
                       "parallelism": f"replicas x{world}"},
            "plain": {"value": plain_fps, "unit": UNIT, "frames": n_plain,
                      "what": "single-frame sessions back to back, same device timing"},
            "batched_over_plain": (value / world / plain_fps) if plain_fps else None,
            "fp2_elem_per_s": folded / (ms / 1e3),
            "latency_ms_per_batch": {"p50": per_batch[len(per_batch) // 2],
                                     "p99": per_batch[min(len(per_batch) - 1,
                                                          int(0.99 * len(per_batch)))]},
            "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "e2e_reference_abi": e2e_ref,
            "gpu_launches": launches, "clocks": clk.summary(), "outputs_nonzero": res_ok,
        }
        print(json.dumps(line), flush=True)


def e2e_batched(args, bprover, frames, z1s, z2s, pts, chal_b, stream, dev):
    """The batched path from pinned host frames: H2D of every frame's bytes, a D2H
    of all claims after every round with a synchronise, D2H of wires and MLEs."""
    import torch
    B = bprover.B
    host = [torch.from_numpy(f).pin_memory() for f in frames]
    dpix = [torch.empty_like(h, device=dev) for h in host]
    R = bprover.max_rounds
    claims_h = torch.zeros(B * 8, dtype=torch.int64).pin_memory()
    wires_h = torch.zeros_like(bprover.wires, device="cpu").pin_memory()
    mle_h = torch.zeros_like(bprover.mle, device="cpu").pin_memory()

    def hook(k):
        claims_h.copy_(bprover.claims[k * B * 8:(k + 1) * B * 8], non_blocking=True)
        stream.synchronize()

    def one():
        with torch.cuda.stream(stream):
            for d, h in zip(dpix, host):
                d.copy_(h, non_blocking=True)
            bprover.prove(dpix, z1s, z2s, pts, chal_b, round_hook=hook)
            wires_h.copy_(bprover.wires, non_blocking=True)
            mle_h.copy_(bprover.mle, non_blocking=True)
        stream.synchronize()

    one()
    steps = max(2, min(args.steps, 8))
    t0 = time.perf_counter()
    for _ in range(steps):
        one()
    wall = time.perf_counter() - t0
    h2d = sum(f.nbytes for f in frames)
    d2h = R * B * 64 + bprover.wires.numel() * 8 + bprover.mle.numel() * 8
    return {"value": steps * B / wall, "unit": UNIT, "h2d_bytes_per_step": h2d,
            "d2h_bytes_per_step": d2h, "steps": steps, "frames_per_step": B,
            "timer": "host wall clock", "path": "tp_batch_* from pinned host frames, "
            "claims read back every round"}


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

    for _ in range(max(1, min(args.warmup, 3))):
        one()
    steps = max(3, min(args.steps, 20))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(steps):
        one()
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    h2d = 16 * W * C + 16 * C + 8 * W * C + 16 * (nb + point.shape[0] + z1.shape[1])
    d2h = 16 * C + 64 * nb + 16 * (W + 1) + 16
    return {"value": steps / wall, "unit": UNIT, "h2d_bytes_per_step": h2d,
            "d2h_bytes_per_step": d2h, "steps": steps, "timer": "host wall clock (synchronous API)",
            "path": "native_fp2_compute_beta/early_create/claim/fold/finish/mle_eval_base, "
                    "pinned host buffers"}


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
    args = ap.parse_args()
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
