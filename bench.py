"""Benchmark: proved 1080p frames/s on one B200 (GKR input layer of the gray circuit).

Workload (one "step" = one frame): a seeded 1920x1080x3 uint8 frame, 16,200
copies of 384 bytes padded to 16,384 x 512 input wires (2^23), proven by the
device-resident path in truepix_b200.frame: table build from the pixels, beta
over the 14 copy challenges, 14 early sumcheck rounds (claim + fold), finish,
and the MLE of the 2^23-entry input vector at the final point. Inputs stay in
HBM (every frame's table, 128 MiB, and input vector, 64 MiB, exceed the 126 MB
L2, so no flush is needed).

  value      frames/s over all ranks, device time (CUDA events), inputs resident
  e2e        frames/s through the reference C ABI (native_fp2_*) with pinned
             host buffers: H2D of the tables and D2H of every claim inside
  roofline   the fused fold+claim kernel: algorithmic bytes (48 B per folded
             element) / its event-timed duration, against MEASURED_PEAKS.json
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
    """DRAM bytes per fold+claim launch of the 1080p round 1, from the committed
    ncu summary (profiles/claim_kernel_fold_1080p.json), scaled like `achieved`."""
    p = os.path.join(ROOT, "profiles", "claim_kernel_fold_1080p.json")
    if os.path.exists(p):
        try:
            return json.load(open(p))
        except ValueError:
            return None
    return None


def kernel_groups(ms, tags, layout):
    """Per claim-kernel kind: launches, total time and algorithmic bytes.
    tag = 1000*(reads pixels) + 100*(fold fused) + log2(copies claimed)."""
    rows = layout.const_idx + 1 if layout.const_idx >= 0 else layout.copy_size
    pix_bytes = layout.copies * layout.copy_size
    groups = {}
    for t, tag in zip(ms, tags):
        pix, fold, lg = tag // 1000, (tag // 100) % 10, tag % 100
        n = 1 << lg                                    # copies claimed
        if pix and not fold:
            name, byt = "claim_pixels_kernel", pix_bytes + 16 * n
        elif pix and fold:
            name, byt = "fold_claim_pixels_kernel", pix_bytes + 16 * rows * n + 48 * n
        elif fold:
            name, byt = "claim_kernel<FOLD_CLAIM>", 48 * rows * n + 48 * n
        else:
            name, byt = "claim_kernel<CLAIM>", 16 * rows * n + 16 * n
        g = groups.setdefault(name, {"launches": 0, "ms": 0.0, "bytes": 0.0, "by_copies": {}})
        g["launches"] += 1
        g["ms"] += t
        g["bytes"] += byt
        bc = g["by_copies"].setdefault(n, [0, 0.0])
        bc[0] += 1
        bc[1] += t
    return groups


def ours_arm(args, rank, world, local_rank):
    import ctypes
    import torch
    import torch.distributed as dist
    from truepix_b200 import native
    from truepix_b200.frame import FrameLayout, GkrInputLayerProver, pack_fp2

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    layout = FrameLayout.for_frame(H, Wd)
    gt, i0, i1 = circuit()
    rng = np.random.default_rng(SEED + 101 * rank)
    n_frames = 4
    frames, z1, z2, point, chal = make_inputs(rng, layout, n_frames)
    pix = [torch.from_numpy(f).to(dev) for f in frames]
    z2_dev = torch.from_numpy(pack_fp2(z2[:, 0], z2[:, 1])).to(dev)
    pt_dev = torch.from_numpy(pack_fp2(point[:, 0], point[:, 1])).to(dev)
    stream = torch.cuda.Stream(dev)
    prover = GkrInputLayerProver(layout, gt, i0, i1, device=local_rank, stream=stream)
    lib = native.gkr()
    nb = layout.n_copy_bits

    with torch.cuda.stream(stream):
        for i in range(args.warmup):
            prover.prove(pix[i % n_frames], z1, z2_dev, pt_dev, chal)
    torch.cuda.synchronize()
    native.check(lib, lib.tp_timer_enable(args.steps * nb + 16), "timer")
    clk = ClockSampler(local_rank)
    clk.start()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    lib.tp_timer_reset()
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    launches = 0
    clk.t0 = time.time()
    with torch.cuda.stream(stream):
        start.record(stream)
        for i in range(args.steps):
            prover.prove(pix[i % n_frames], z1, z2_dev, pt_dev, chal)
            launches += prover.launches_last
        end.record(stream)
    torch.cuda.synchronize()
    clk.t1 = time.time()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clk.stop()
    npairs = args.steps * nb + 16
    tms = (ctypes.c_float * npairs)()
    ttags = (ctypes.c_int * npairs)()
    got = lib.tp_timer_read(tms, ttags, npairs)
    lib.tp_timer_disable()
    ms = start.elapsed_time(end)
    t = torch.tensor([ms], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms = float(t.item())
    value = world * args.steps / (ms / 1e3)

    groups = kernel_groups(list(tms[:max(0, got)]), list(ttags[:max(0, got)]), layout)
    peak, peak_kind = peaks()
    kernels = []
    for name, g in sorted(groups.items(), key=lambda kv: -kv[1]["ms"]):
        ach = g["bytes"] / (g["ms"] / 1e3) / 1e9 if g["ms"] > 0 else None
        kernels.append({"kernel": name, "launches": g["launches"], "total_ms": g["ms"],
                        "share_of_step": g["ms"] / ms, "achieved_gbs": ach,
                        "avg_us_by_copies": {str(k): round(1e3 * v[1] / v[0], 2)
                                             for k, v in sorted(g["by_copies"].items())}})
    top = kernels[0] if kernels else None
    traffic = profiled_traffic()
    roof = None
    if top:
        g = groups[top["kernel"]]
        roof = {"kernel": top["kernel"], "bound": "hbm", "achieved": top["achieved_gbs"],
                "peak": peak, "unit": "GB/s",
                "frac": top["achieved_gbs"] / peak if top["achieved_gbs"] else None,
                "peak_source": peak_kind + " (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured"
                else "fallback 6650 GB/s",
                "algorithmic_bytes_per_launch": g["bytes"] / g["launches"],
                "avg_launch_us": 1e3 * g["ms"] / g["launches"], "launches_timed": g["launches"],
                "traffic": (traffic or {}).get(top["kernel"]),
                "all_claim_kernels": kernels}

    res_ok = None
    if rank == 0:
        c, w, b, m = prover.results()
        res_ok = bool(c.any() and w.any() and m != (0, 0))

    e2e = None
    cpu = None
    if rank == 0 and not args.skip_e2e:
        e2e = e2e_c_abi(args, lib, frames[0], layout, gt, i0, i1, z1, z2, point, chal)
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
                       "circuit": "gray.pws", "path": "pixels (tp_early_create_pixels)",
                       "l2": "inputs > L2: 4 distinct frames cycled; the folded table of "
                             "round 1 (47 MiB) is rewritten every frame",
                       "parallelism": f"replicas x{world}"},
            "roofline": roof, "cpu_baseline": cpu, "e2e": e2e,
            "gpu_launches": launches, "clocks": clk.summary(), "outputs_nonzero": res_ok,
        }
        print(json.dumps(line), flush=True)


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
    steps = max(3, min(args.steps // 100, 20))
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
    ap.add_argument("--steps", type=int, default=3000)
    ap.add_argument("--warmup", type=int, default=50)
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
