"""Serving loop: continuous batching of frame proofs on one GPU.

Requests (an operation's circuit, a frame of some resolution, a seed for its
transcript values) arrive over time. The server keeps up to `slots` proofs in
flight in one tp_batch: every tick runs ONE claim launch per source kind for all
frames in their early sumcheck rounds, whatever round each is in, reads the
claims back (the host transcript needs them), and folds each frame by its own
challenge. A frame whose early rounds are over is finished alone
(tp_batch_finish_frame), its input MLE evaluated from its bytes, and its Orion
commitment queued on one of several commit streams, so commits overlap each
other and the rounds of the frames still in flight; its slot is free for the next request at once. Requests
are admitted while a slot is free and the frame's HBM footprint fits the budget.

The frame layout and the per-round work are those of truepix_b200.frame and
truepix_b200.orion (TruePix-main/libTruePix/layerprover.py:144-290 drives the
same early rounds one frame at a time). Challenges, z1, z2 and the MLE point
are derived from each request's seed; a request's results do not depend on what
else is in flight (tests/test_gpu_serving.py checks this).
"""
from __future__ import annotations

import ctypes
import math
import time
from dataclasses import dataclass

import numpy as np

from . import native
from .frame import FrameLayout, pack_fp2

P61 = (1 << 61) - 1


@dataclass
class Circuit:
    """One layer's gate table and the frame layout it reads (copy_size inputs per
    copy, constant wire, 512 wires per copy)."""
    name: str
    gate_type: np.ndarray
    in0: np.ndarray
    in1: np.ndarray
    copy_size: int = 384
    const_idx: int = 384
    const_val: int = 128


@dataclass
class Request:
    rid: int
    circuit: Circuit
    height: int
    width: int
    # uint8, height * width * 3 bytes on the host: a numpy array (copied through
    # a pinned staging buffer) or a pinned torch tensor (copied straight to the
    # device; keep it unchanged until the request's Result is returned)
    pixels: object
    seed: int
    arrival: float = 0.0          # seconds after the start of the run


@dataclass
class Result:
    rid: int
    claims: np.ndarray            # [rounds, 8] u64
    wires: np.ndarray             # [512, 2] u64
    beta: tuple
    mle: tuple
    root: bytes
    arrival: float = 0.0
    done: float = 0.0

    @property
    def latency(self) -> float:
        return self.done - self.arrival


def transcript_values(seed: int, n_gates: int, n_copy_bits: int, n_in_bits: int):
    """z1 [2, n_gates], z2 [n_copy_bits, 2], point [n_in_bits + n_copy_bits, 2],
    challenges [n_copy_bits, 2]: canonical, from the request's seed (they stand in
    for the Fiat-Shamir transcript, which stays on the host)."""
    rng = np.random.default_rng(seed)
    f = lambda *shape: rng.integers(0, P61, size=shape, dtype=np.uint64)
    return f(2, n_gates), f(n_copy_bits, 2), f(n_in_bits + n_copy_bits, 2), f(n_copy_bits, 2)


def layout_for(c: Circuit, height: int, width: int) -> FrameLayout:
    copies = math.ceil(height * width * 3 / c.copy_size)
    return FrameLayout(copies=copies, copy_size=c.copy_size, n_wires=512, const_idx=c.const_idx,
                       const_val=c.const_val)


class _Job:
    """One request in flight: its layout, transcript values, and views into the
    slot's persistent device buffers."""

    def __init__(self, srv, req: Request, slot: int):
        self.req, self.slot = req, slot
        c = req.circuit
        self.L = L = layout_for(c, req.height, req.width)
        if L.copies * L.copy_size > srv.max_bytes or L.padded_copies > srv.max_copies:
            raise ValueError("request %d: frame larger than the server's maximum" % req.rid)
        nb, ni = L.n_copy_bits, L.n_in_bits
        self.z1, z2, point, self.chal = transcript_values(req.seed, c.gate_type.size, nb, ni)
        b = srv.slot_bufs[slot]
        self.pix = b["pix"][:L.copies * L.copy_size]
        self.beta = b["beta"][:2 * L.padded_copies]
        self.z2 = b["z2"][:2 * nb]
        self.point = b["point"][:2 * (ni + nb)]
        self.wires, self.mle = b["wires"], b["mle"]
        self.out_h = b["out_h"]      # pinned: wires, beta, MLE, root after the commit
        # transcript values through the slot's pinned buffer (a pageable source
        # would synchronise the stream); the slot's previous job is long done
        zh = b["z_h"].numpy()
        zh[:2 * nb] = pack_fp2(z2[:, 0], z2[:, 1])
        zh[2 * nb:2 * nb + 2 * (ni + nb)] = pack_fp2(point[:, 0], point[:, 1])
        srv.upload(self.pix, req.pixels, L.copies * L.copy_size, after=lambda: (
            self.z2.copy_(b["z_h"][:2 * nb], non_blocking=True),
            self.point.copy_(b["z_h"][2 * nb:2 * nb + 2 * (ni + nb)], non_blocking=True)))
        self.round = 0
        self.host_claims = []          # what the host transcript read, round by round
        self.done_event = None
        self.commit_buf = None
        self.footprint = srv.footprint(L)

    def rounds(self) -> int:
        return self.L.n_copy_bits


class ProofServer:
    """Continuous batching of frame proofs (see the module docstring).

    Device memory is allocated once: per slot the frame's bytes, beta and the
    small transcript / result vectors (sized for max_height x max_width); the
    slot's folded tables stay in the library's pool for the next frame; and
    `commit_buffers` codeword + tree buffers that commits take in turn (a commit
    waits for a free one). A served frame's codeword is recycled once its root
    is read, so Result carries the root; a prover that opens the commitment
    later keeps the codeword instead (truepix_b200.orion.FrameCommitter)."""

    def __init__(self, slots: int = 64, hbm_budget: float = 40e9, device: int = 0, max_height: int = 2160,
                 max_width: int = 3840, commit_buffers: int = 16, leaf_chunks: int = 4):
        """leaf_chunks: the commits' SHA-256 leaf chains run as that many shorter
        launches (tp_orion_set_leaf_chunks, process-wide), so SMs free up sooner
        for the rounds the loop waits on every tick."""
        import torch
        self.torch = torch
        self.lib = native.gkr()
        native.check(self.lib, self.lib.tp_orion_set_leaf_chunks(leaf_chunks), "leaf chunks")
        self.dev = torch.device("cuda", device)
        # the rounds' stream has the higher priority: its small claim and fold
        # kernels (on which the host waits every tick) go ahead of queued commits
        self.stream = torch.cuda.Stream(self.dev, priority=-1)
        self.upload_stream = torch.cuda.Stream(self.dev)
        # commits go round-robin over a few streams so that one frame's
        # latency-bound commit phases overlap another's SHA-256 leaves
        self.commit_streams = [torch.cuda.Stream(self.dev) for _ in range(max(1, commit_buffers))]
        self.commit_next = 0
        self.slots = slots
        self.budget = hbm_budget
        self.batch = self.lib.tp_batch_create(slots, self.stream.cuda_stream)
        if not self.batch:
            native.check(self.lib, -1, "batch_create")
        self.max_bytes = max_height * max_width * 3 + 512
        self.max_copies = 1 << math.ceil(math.log2(max(2, -(-max_height * max_width * 3 // 384))))
        nbmax = int(math.log2(self.max_copies))
        i64, dev = torch.int64, self.dev
        self.slot_bufs = [{"pix": torch.zeros(self.max_bytes, dtype=torch.uint8, device=dev),
                           "beta": torch.empty(2 * self.max_copies, dtype=i64, device=dev),
                           "z2": torch.empty(2 * nbmax, dtype=i64, device=dev),
                           "point": torch.empty(2 * (9 + nbmax), dtype=i64, device=dev),
                           "wires": torch.zeros(2 * 513, dtype=i64, device=dev),
                           "mle": torch.zeros(2, dtype=i64, device=dev),
                           "z_h": torch.zeros(2 * (9 + 2 * nbmax), dtype=i64).pin_memory(),
                           "out_h": torch.zeros(2 * 513 + 2 + 4, dtype=i64).pin_memory()}
                          for _ in range(slots)]
        col = self.max_copies * 512 // 128
        cw_max = self.lib.tp_orion_codeword_len(col)
        leaves_max = self.lib.tp_orion_tree_leaves(col * 128)
        self.commit_free = [(torch.empty(2 * 128 * cw_max, dtype=i64, device=dev),
                             torch.empty(64 * leaves_max, dtype=torch.uint8, device=dev))
                            for _ in range(commit_buffers)]
        # pinned staging buffers for numpy frames (a few uploads may be in flight)
        self.staging = [torch.empty(self.max_bytes, dtype=torch.uint8).pin_memory() for _ in range(3)]
        self.staging_ev = [None] * len(self.staging)
        self.staging_next = 0
        self.free = list(range(slots))[::-1]
        self.active: dict = {}          # slot -> _Job
        self.committing: list = []      # jobs whose commit is queued, oldest first
        self.used = 0.0
        self.d_claims = torch.zeros(8 * slots, dtype=i64, device=dev)
        self.h_claims = torch.zeros(8 * slots, dtype=i64).pin_memory()
        self.chal = np.zeros((slots, 2), np.uint64)
        self.ticks = 0
        self.launches = 0
        self._t0 = time.perf_counter()
        self._out = []

    def close(self):
        """Release the batch and the server's device buffers now (freeing device
        memory synchronises the device, so a server that is dropped inside
        another one's run would stall it)."""
        if getattr(self, "batch", None):
            self.torch.cuda.synchronize(self.dev)
            self.lib.tp_batch_destroy(self.batch)
            self.batch = None
        self.slot_bufs = self.commit_free = self.staging = []
        self.active, self.committing = {}, []

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def footprint(L: FrameLayout) -> float:
        """HBM held by one proof in flight: folded tables (rows x C/2 + rows x C/4),
        beta, the frame's bytes, the codeword (cw_len x 2 KB) and its tree."""
        rows = L.const_idx + 1 if L.const_idx >= 0 else L.copy_size
        C = L.padded_copies
        col = C * L.n_wires // 128
        cw = col * 1.72 + 64
        leaves = 1 << math.ceil(math.log2(2 * col))
        return 16 * rows * (C // 2 + C // 4) + 32 * C + L.copies * L.copy_size + 2048 * cw + 64 * leaves

    def upload(self, d_pix, pixels, n: int, after=None):
        """Frame bytes to the slot's device buffer (zero-padded to the layout's
        copies x copy_size) on the upload stream: a pinned torch tensor directly,
        a numpy array through a pinned staging buffer. `after()` queues more
        copies behind it. The rounds' stream waits for the upload, the host only
        for a staging buffer's previous copy (DMA, never kernels)."""
        torch = self.torch
        with torch.cuda.stream(self.upload_stream):
            if isinstance(pixels, torch.Tensor):
                if not pixels.is_pinned():
                    raise ValueError("tensor frames must be in pinned host memory")
                src = pixels.reshape(-1)
                m = min(n, src.numel())
                d_pix[:m].copy_(src[:m], non_blocking=True)
                if m < n:
                    d_pix[m:n].zero_()
            else:
                k = self.staging_next
                self.staging_next = (k + 1) % len(self.staging)
                if self.staging_ev[k] is not None:
                    self.staging_ev[k].synchronize()
                h = self.staging[k].numpy()
                m = min(n, pixels.size)
                h[:m] = pixels.reshape(-1)[:m]
                h[m:n] = 0
                d_pix.copy_(self.staging[k][:n], non_blocking=True)
                self.staging_ev[k] = torch.cuda.Event()
                self.staging_ev[k].record(self.upload_stream)
            if after is not None:
                after()
            ev = torch.cuda.Event()
            ev.record(self.upload_stream)
        self.stream.wait_event(ev)

    def _start(self, req: Request):
        lib, s = self.lib, self.stream.cuda_stream
        slot = self.free.pop()
        with self.torch.cuda.stream(self.stream):
            job = _Job(self, req, slot)
        L, c = job.L, req.circuit
        native.check(lib, lib.tp_compute_beta_dev(job.z2.data_ptr(), L.n_copy_bits, 1, 0,
                                                  job.beta.data_ptr(), s), "beta")
        z1r = np.ascontiguousarray(job.z1[0])
        z1i = np.ascontiguousarray(job.z1[1])
        gt = np.ascontiguousarray(c.gate_type, np.int32)
        i0 = np.ascontiguousarray(c.in0, np.int32)
        i1 = np.ascontiguousarray(c.in1, np.int32)
        native.check(lib, lib.tp_batch_set_pixels(
            self.batch, slot, gt.size, gt.ctypes.data, i0.ctypes.data, i1.ctypes.data,
            z1r.ctypes.data, z1i.ctypes.data, job.pix.data_ptr(), L.copies, L.padded_copies,
            L.copy_size, L.n_wires, L.const_idx, L.const_val, job.beta.data_ptr()), "set_pixels")
        self.active[slot] = job
        self.used += job.footprint

    def _finish(self, job: _Job):
        torch, lib, s = self.torch, self.lib, self.stream.cuda_stream
        L = job.L
        wp = job.wires.data_ptr()
        native.check(lib, lib.tp_batch_finish_frame(self.batch, job.slot, wp, wp + 16 * L.n_wires),
                     "finish_frame")
        native.check(lib, lib.tp_mle_eval_pixels(job.pix.data_ptr(), L.copies, L.padded_copies,
                                                 L.copy_size, L.n_wires, L.const_idx, L.const_val,
                                                 job.point.data_ptr(), job.mle.data_ptr(), s), "mle")
        while not self.commit_free:                 # back-pressure: wait for the oldest commit
            self._collect(block_first=True)
        job.commit_buf = rows, tree = self.commit_free.pop()
        cs = self.commit_streams[self.commit_next]
        self.commit_next = (self.commit_next + 1) % len(self.commit_streams)
        ev = torch.cuda.Event()
        ev.record(self.stream)
        cs.wait_event(ev)
        native.check(lib, lib.tp_orion_commit_pixels_dev(
            job.pix.data_ptr(), L.copies, L.padded_copies, L.copy_size, L.n_wires, L.const_idx,
            L.const_val, rows.data_ptr(), tree.data_ptr(), cs.cuda_stream), "commit")
        self.launches += lib.tp_orion_last_launches() + 3
        # results to the slot's pinned buffer behind the commit (read by _collect)
        with torch.cuda.stream(cs):
            job.out_h[:2 * 513].copy_(job.wires, non_blocking=True)
            job.out_h[2 * 513:2 * 513 + 2].copy_(job.mle, non_blocking=True)
            job.out_h[2 * 513 + 2:].copy_(tree[32:64].view(torch.int64), non_blocking=True)
        job.done_event = torch.cuda.Event()
        job.done_event.record(cs)
        del self.active[job.slot]
        self.committing.append(job)

    def _collect(self, block: bool = False, block_first: bool = False):
        """Results of the commits that are done (all of them when block; at least
        the oldest when block_first); their slots and commit buffers return."""
        keep = []
        for q, job in enumerate(self.committing):
            if block or (block_first and q == 0):
                job.done_event.synchronize()
            if job.done_event.query():
                c = np.stack(job.host_claims)
                out = job.out_h.numpy().view(np.uint64)
                w = out[:2 * 513].reshape(513, 2)
                m = out[2 * 513:2 * 513 + 2]
                root = out[2 * 513 + 2:].tobytes()
                self._out.append(Result(job.req.rid, c, w[:job.L.n_wires].copy(),
                                        (int(w[job.L.n_wires, 0]), int(w[job.L.n_wires, 1])),
                                        (int(m[0]), int(m[1])), root, job.req.arrival,
                                        time.perf_counter() - self._t0))
                self.used -= job.footprint
                self.commit_free.append(job.commit_buf)
                self.free.append(job.slot)
            else:
                keep.append(job)
        self.committing = keep

    def tick(self):
        """One round for every frame in flight: claim (one launch per source kind),
        claims to the host, fold each frame by its own challenge."""
        lib, torch = self.lib, self.torch
        if not self.active:
            return
        l0 = lib.tp_batch_launches(self.batch)
        native.check(lib, lib.tp_batch_claim(self.batch, self.d_claims.data_ptr()), "batch_claim")
        with torch.cuda.stream(self.stream):
            self.h_claims.copy_(self.d_claims, non_blocking=True)
        self.stream.synchronize()                   # the host transcript reads the claims
        hc = self.h_claims.numpy().view(np.uint64).reshape(self.slots, 8)
        self.chal[:] = 0
        for slot, job in self.active.items():
            job.host_claims.append(hc[slot].copy())  # absorbed into the frame's transcript
            self.chal[slot] = job.chal[job.round]
            job.round += 1
        native.check(lib, lib.tp_batch_fold(
            self.batch, self.chal.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))), "batch_fold")
        for job in [j for j in self.active.values() if j.round == j.rounds()]:
            self._finish(job)
        self.launches += lib.tp_batch_launches(self.batch) - l0
        self.ticks += 1

    def run(self, requests, realtime: bool = True):
        """Serve `requests` (sorted by arrival). realtime: a request enters the
        queue when the wall clock reaches its arrival time; otherwise arrivals are
        in ticks (arrival = tick index). Returns the results in completion order."""
        reqs = sorted(requests, key=lambda r: r.arrival)
        queue = []
        self._out = []
        i = 0
        self._t0 = t0 = time.perf_counter()
        while i < len(reqs) or queue or self.active or self.committing:
            now = time.perf_counter() - t0 if realtime else float(self.ticks)
            while i < len(reqs) and reqs[i].arrival <= now:
                queue.append(reqs[i])
                i += 1
            while queue and self.free:
                L = layout_for(queue[0].circuit, queue[0].height, queue[0].width)
                if (self.active or self.committing) and self.used + self.footprint(L) > self.budget:
                    break
                req = queue.pop(0)
                if not realtime:
                    req.arrival = time.perf_counter() - t0
                self._start(req)
            if self.active:
                self.tick()
            elif not queue and i < len(reqs):
                if realtime:
                    time.sleep(max(0.0, min(0.001, reqs[i].arrival - now)))
                else:
                    self.ticks += 1
            self._collect(block=not self.active and not queue and i >= len(reqs),
                          block_first=not self.active and bool(queue))
        return self._out


def latency_stats(results):
    lat = sorted(r.latency for r in results)
    if not lat:
        return {}
    pick = lambda q: lat[min(len(lat) - 1, int(q * len(lat)))]
    span = max(r.done for r in results) - min(r.arrival for r in results)
    return {"p50_ms": 1e3 * pick(0.5), "p99_ms": 1e3 * pick(0.99), "mean_ms": 1e3 * sum(lat) / len(lat),
            "frames": len(lat), "frames_per_s": len(lat) / span if span > 0 else None}
