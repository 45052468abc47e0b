"""Serving loop: continuous batching of whole frame proofs on one GPU.

Requests (an operation's circuit, a frame of some resolution, the prover's pid
and VOLE correlations) arrive over time; each leaves with the proof the
reference's prover phase writes for its frame (run_truepix_prover.py:218-421,
plain prover): the GKR input layer's proof container and the Orion opening file
(truepix_b200.pipeline.FrameProof). A request moves through these stages, each
frame on its own, frames of different circuits and sizes side by side:

  admit     a free slot and room in the HBM budget: the frame's bytes go up on
            the upload stream, its Orion commit runs on one of the commit
            streams, its IO transcript (the circuit's output vector computed on
            the host from the bytes and hashed as it is made,
            tp_fs_put_circuit_outputs_pixels) on a host thread, which then binds
            the commit's root and draws z1, z2
  rounds    the frame joins the running batch (tp_batch_set_pixels) with its
            transcript and VOLE state uploaded to its slot; every tick is one
            claim launch for all frames in their early rounds, ONE VOLE-committed
            round launch in which each slot runs its own round on its own
            transcript (tp_vole_round_slots_dev: the label "sc-0-<round>" is made
            on the device, the challenge stays there) and one fold by those
            device challenges (tp_batch_fold_dev): the host never waits on a tick
  late      the frame's finish, then its late rounds and closing proofs
            (tp_late_rounds_dev) on the late stream, the proof values to pinned
            host memory
  open      on a host thread the opening's eq tables, queried columns and node
            lists; on the open stream the combined codeword, its tree, the
            answer, the queried columns and the gathered nodes over the frame's
            codeword in HBM; on a host thread the file's bytes

Admission is by HBM footprint (tables, codeword, tree, opening buffers). Every
value of a request depends only on its own inputs: a proof is the same alone
and in any mix (tests/test_gpu_serving.py), and the same as
truepix_b200.prover.prove_frames + truepix_b200.opening.opening_proof give.
"""
from __future__ import annotations

import concurrent.futures
import ctypes
import math
import os
import struct
import time
from dataclasses import dataclass

import numpy as np

from . import native
from .frame import FrameLayout, pack_fp2
from .opening import COLUMN_SIZE, opening_bytes, query_count
from .pipeline import CircuitOutputs, FrameProof, correlations_needed
from .prover import LayerTranscript, commit_binding, commit_manifest

P61 = (1 << 61) - 1
_I32P = ctypes.POINTER(ctypes.c_int)


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
    # uint8, height * width * 3 bytes on the host: a numpy array or a pinned torch
    # tensor (copied straight to the device; keep it unchanged until the request's
    # Result is returned)
    pixels: object
    pid: int
    correlations: tuple           # (u, v) uint64 [count, 2], count >= correlations_needed(layout)
    arrival: float = 0.0          # seconds after the start of the run


@dataclass
class Result:
    rid: int
    proof: FrameProof
    arrival: float = 0.0
    done: float = 0.0

    @property
    def latency(self) -> float:
        return self.done - self.arrival


def layout_for(c: Circuit, height: int, width: int) -> FrameLayout:
    copies = math.ceil(height * width * 3 / c.copy_size)
    return FrameLayout(copies=copies, copy_size=c.copy_size, n_wires=512, const_idx=c.const_idx,
                       const_val=c.const_val)


class _Job:
    """One request in flight: its layout, stage, slot and per-request buffers."""

    def __init__(self, req: Request, slot: int, L: FrameLayout, footprint: float):
        self.req, self.slot, self.L, self.footprint = req, slot, L, footprint
        self.stage = "io"
        self.round = 0
        self.future = None
        self.event = None


class ProofServer:
    """Continuous batching of whole frame proofs (see the module docstring).

    Slots hold a frame's bytes, beta, transcript, VOLE state, correlations and
    round outputs in device memory allocated once, and its codeword, tree and
    opening buffers (device and pinned staging) made at the slot's first use: all
    sized for max_height x max_width (a 2160p slot holds ~1 GB of HBM), so a
    running server allocates nothing per request."""

    def __init__(self, slots: int = 32, hbm_budget: float = 60e9, device: int = 0, max_height: int = 2160,
                 max_width: int = 3840, host_threads: int = 0, commit_streams: int = 8, leaf_chunks: int = 4,
                 fp2_type=None):
        """leaf_chunks: the commits' SHA-256 leaf chains run as that many shorter
        launches (tp_orion_set_leaf_chunks, process-wide), so SMs free up sooner for
        the ticks' small kernels."""
        import torch
        self.torch = torch
        self.lib = lib = native.gkr()
        native.check(lib, lib.tp_orion_set_leaf_chunks(leaf_chunks), "leaf chunks")
        self.dev = dev = torch.device("cuda", device)
        self.fp2_type = fp2_type
        # the ticks' stream has the higher priority: its small kernels go ahead of queued commits
        self.stream = torch.cuda.Stream(dev, priority=-1)
        self.upload_stream = torch.cuda.Stream(dev)
        self.late_stream = torch.cuda.Stream(dev)
        self.open_stream = torch.cuda.Stream(dev)
        self.commit_streams = [torch.cuda.Stream(dev) for _ in range(max(1, commit_streams))]
        self.commit_next = 0
        self.slots = slots
        self.budget = hbm_budget
        self.batch = lib.tp_batch_create(slots, self.stream.cuda_stream)
        if not self.batch:
            native.check(lib, -1, "batch_create")
        self.max_bytes = max_height * max_width * 3 + 512
        self.max_copies = 1 << math.ceil(math.log2(max(2, -(-max_height * max_width * 3 // 384))))
        self.nbmax = nbmax = int(math.log2(self.max_copies))
        self.count = correlations_needed(FrameLayout(copies=self.max_copies), False)
        n = 9
        self.n = n
        i64, u8 = torch.int64, torch.uint8
        S, C = slots, self.count
        nst, nvs = lib.tp_fs_state_bytes(), lib.tp_vole_state_bytes()
        self.nst, self.nvs = nst, nvs
        self.d = dict(pix=[torch.zeros(self.max_bytes, dtype=u8, device=dev) for _ in range(S)],
                      beta=[torch.empty(2 * self.max_copies, dtype=i64, device=dev) for _ in range(S)],
                      z2=torch.zeros(2 * S * nbmax, dtype=i64, device=dev),
                      zg=torch.zeros(2 * S * 1024, dtype=i64, device=dev),
                      states=torch.zeros(S * nst, dtype=u8, device=dev),
                      vs=torch.zeros(S * nvs, dtype=u8, device=dev),
                      meta=torch.full((2 * S,), -1, dtype=torch.int32, device=dev),
                      u=torch.zeros(2 * S * C, dtype=i64, device=dev),
                      v=torch.zeros(2 * S * C, dtype=i64, device=dev),
                      claims=torch.zeros(8 * S, dtype=i64, device=dev),
                      chal=torch.zeros(2 * S, dtype=i64, device=dev),
                      chal_hist=torch.zeros(2 * S * nbmax, dtype=i64, device=dev),
                      proof=torch.zeros(10 * S * nbmax, dtype=i64, device=dev),
                      wires=torch.zeros(2 * S * 512, dtype=i64, device=dev),
                      fin_beta=torch.zeros(2 * S, dtype=i64, device=dev),
                      coefs=torch.zeros(2 * S * 6 * n, dtype=i64, device=dev),
                      line=torch.zeros(2 * S * (n + 1), dtype=i64, device=dev),
                      chal_out=torch.zeros(2 * S * 2 * n, dtype=i64, device=dev),
                      late=torch.zeros(2 * S * 8 * n, dtype=i64, device=dev),
                      closing=torch.zeros(2 * S * (n + 10), dtype=i64, device=dev),
                      point=torch.zeros(2 * S * (n + nbmax), dtype=i64, device=dev),
                      tag=torch.zeros(2 * S, dtype=i64, device=dev))
        # pinned host mirrors, one region per slot (rewritten only when the slot is reused)
        self.h = dict(z2=torch.zeros(2 * S * nbmax, dtype=i64).pin_memory(),
                      zg=torch.zeros(2 * S * 1024, dtype=i64).pin_memory(),
                      states=torch.zeros(S * nst, dtype=u8).pin_memory(),
                      vs=torch.zeros(S * nvs, dtype=u8).pin_memory(),
                      meta=torch.zeros(2 * S, dtype=torch.int32).pin_memory(),
                      u=torch.zeros(2 * S * C, dtype=i64).pin_memory(),
                      v=torch.zeros(2 * S * C, dtype=i64).pin_memory(),
                      roots=torch.zeros((S, 32), dtype=u8).pin_memory(),
                      proof=torch.zeros(10 * S * nbmax, dtype=i64).pin_memory(),
                      late=torch.zeros(2 * S * 8 * n, dtype=i64).pin_memory(),
                      closing=torch.zeros(2 * S * (n + 10), dtype=i64).pin_memory(),
                      point=torch.zeros(2 * S * (n + nbmax), dtype=i64).pin_memory(),
                      tag=torch.zeros(2 * S, dtype=i64).pin_memory(),
                      states_out=torch.zeros(S * nst, dtype=u8).pin_memory(),
                      vs_out=torch.zeros(S * nvs, dtype=u8).pin_memory())
        vs0 = ctypes.create_string_buffer(nvs)
        native.check(lib, lib.tp_vole_state_init(vs0, 0, None), "tp_vole_state_init")
        self.vs0 = np.frombuffer(vs0.raw, np.uint8).copy()
        self.pool = concurrent.futures.ThreadPoolExecutor(host_threads or os.cpu_count() or 4)
        self.free = list(range(slots))[::-1]
        self.slot_mem = [None] * slots      # codeword, tree and opening buffers, made at a slot's first use
        # ticks in flight: a new tick is queued only when at most max_ticks_ahead are not done, so
        # the ticks' stream never runs far ahead of the device (uploads queued on it stay prompt)
        self.tick_events = []
        self.max_ticks_ahead = 2
        self.jobs: list = []
        self.used = 0.0
        self.ticks = 0
        self.launches = 0
        self._t0 = time.perf_counter()
        self._out = []

    def close(self):
        """Finish the host threads and release the batch and the device buffers."""
        if getattr(self, "batch", None):
            self.pool.shutdown(wait=True)
            self.torch.cuda.synchronize(self.dev)
            self.lib.tp_batch_destroy(self.batch)
            self.batch = None
        self.d = self.h = {}
        self.jobs = []

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- sizes ------------------------------------------------------------------
    def footprint(self, L: FrameLayout) -> float:
        """HBM one proof in flight holds: folded tables (rows x C/2 + rows x C/4),
        its codeword (cw_len x 2 KB) and tree, and its opening buffers (combined
        codeword and tree, queried columns, gathered nodes, eq tables)."""
        rows = L.const_idx + 1 if L.const_idx >= 0 else L.copy_size
        C = L.padded_copies
        N = C * L.n_wires
        cw = self.lib.tp_orion_codeword_len(N // COLUMN_SIZE)
        leaves = self.lib.tp_orion_tree_leaves(N)
        qc = query_count()
        opening = 16 * cw + 64 * leaves + 16 * COLUMN_SIZE * qc + 2 * 32 * qc * 24 + 16 * (N // COLUMN_SIZE)
        return 16 * rows * (C // 2 + C // 4) + 2048 * cw + 64 * leaves + opening

    def _slot_mem(self, s: int) -> dict:
        """slot s's codeword, tree and opening buffers (device) and the opening's
        pinned staging, sized for the server's largest frame"""
        if self.slot_mem[s] is None:
            torch, lib, dev = self.torch, self.lib, self.dev
            N = self.max_copies * 512
            cw, lv, qc = lib.tp_orion_codeword_len(N // COLUMN_SIZE), lib.tp_orion_tree_leaves(N), query_count()
            nodes = qc * int(math.log2(lv))
            i64, u8 = torch.int64, torch.uint8
            dv = lambda n, t: torch.empty(n, dtype=t, device=dev)
            pn = lambda n, t: torch.empty(n, dtype=t, pin_memory=True)
            self.slot_mem[s] = dict(
                rows=dv(2 * COLUMN_SIZE * cw, i64), tree=dv(64 * lv, u8), comb=dv(2 * cw, i64), ctree=dv(64 * lv, u8),
                ans=dv(2, i64), cols=dv(2 * COLUMN_SIZE * qc, i64), nodes=dv(64 * nodes, u8),
                r0=dv(2 * COLUMN_SIZE, i64), r1=dv(2 * (N // COLUMN_SIZE), i64), q=dv(qc, i64),
                idx=dv(nodes, torch.int32),
                h_r0=pn(2 * COLUMN_SIZE, i64), h_r1=pn(2 * (N // COLUMN_SIZE), i64), h_q=pn(qc, i64),
                h_idx=pn(nodes, torch.int32), h_comb=pn(2 * cw, i64), h_ans=pn(2, i64),
                h_cols=pn(2 * COLUMN_SIZE * qc, i64), h_root=pn(32, u8), h_nodes=pn(64 * nodes, u8))
        return self.slot_mem[s]

    # ---- stages -----------------------------------------------------------------
    def _admit(self, req: Request):
        torch, lib = self.torch, self.lib
        c = req.circuit
        L = layout_for(c, req.height, req.width)
        if L.copies * L.copy_size > self.max_bytes or L.padded_copies > self.max_copies:
            raise ValueError("request %d: frame larger than the server's maximum" % req.rid)
        need = correlations_needed(L)
        if len(req.correlations[0]) < need or len(req.correlations[1]) < need:
            raise IndexError("request %d: %d VOLE correlations needed" % (req.rid, need))
        job = _Job(req, self.free.pop(), L, self.footprint(L))
        self.used += job.footprint
        s = job.slot
        nbytes = L.copies * L.copy_size
        if torch.is_tensor(req.pixels):
            if not req.pixels.is_pinned():
                raise ValueError("tensor frames must be in pinned host memory")
            host_t = req.pixels.reshape(-1)
        else:
            host_t = torch.from_numpy(np.ascontiguousarray(req.pixels, np.uint8).reshape(-1))
        # a frame whose bytes end inside its last copy is zero-padded to whole copies (the
        # layout's unused wires): on the device by the upload, on the host by the IO
        # transcript, which reads the frame's own bytes only
        have = min(host_t.numel(), nbytes)
        job.host = host_t.numpy()[:have]
        job.pix = self.d["pix"][s][:nbytes]
        with torch.cuda.stream(self.upload_stream):
            job.pix[:have].copy_(host_t[:have], non_blocking=True)
            if have < nbytes:
                job.pix[have:].zero_()
            job.uploaded = torch.cuda.Event()
            job.uploaded.record(self.upload_stream)
        job.host_t = host_t     # kept alive until the copy is done
        # the commit, on a commit stream, once the bytes are up; its root back to pinned memory
        N = L.padded_copies * L.n_wires
        job.N, job.cw_len, job.leaves = N, lib.tp_orion_codeword_len(N // COLUMN_SIZE), lib.tp_orion_tree_leaves(N)
        cs = self.commit_streams[self.commit_next]
        self.commit_next = (self.commit_next + 1) % len(self.commit_streams)
        job.mem = mem = self._slot_mem(s)
        with torch.cuda.stream(cs):
            cs.wait_event(job.uploaded)
            job.rows = mem["rows"][:2 * COLUMN_SIZE * job.cw_len]
            job.tree = mem["tree"][:64 * job.leaves]
            native.check(lib, lib.tp_orion_commit_pixels_dev(
                job.pix.data_ptr(), L.copies, L.padded_copies, L.copy_size, L.n_wires, L.const_idx, L.const_val,
                job.rows.data_ptr(), job.tree.data_ptr(), cs.cuda_stream), "commit")
            self.launches += lib.tp_orion_last_launches()
            self.h["roots"][s].copy_(job.tree[32:64], non_blocking=True)
            job.committed = torch.cuda.Event()
            job.committed.record(cs)
        job.tr = LayerTranscript(req.pid, self.fp2_type)
        job.future = self.pool.submit(self._io, job)
        self.jobs.append(job)

    def _io(self, job: _Job):
        """host thread: the IO transcript, the binding of the commit's root, z1 and z2"""
        lib, L, c, t = self.lib, job.L, job.req.circuit, job.tr
        gt, i0, i1 = (np.ascontiguousarray(a, np.int32) for a in (c.gate_type, c.in0, c.in1))
        t.fs.put(t.pid)
        t.fs.put(None, True)
        t.fs.put(["private_input_omitted", int(L.padded_copies * L.n_wires)], True)
        t.fs.io.append(CircuitOutputs(job.host, L, gt, i0, i1, self.dev))
        st = (ctypes.c_void_p * 1)(ctypes.addressof(t.fs._st))
        px = (ctypes.c_void_p * 1)(job.host.ctypes.data)
        native.check(lib, lib.tp_fs_put_circuit_outputs_pixels(
            st, px, job.host.size, 1, L.copies, L.padded_copies, L.copy_size, L.n_wires, L.const_idx, L.const_val,
            gt.size,
            gt.ctypes.data_as(_I32P), i0.ctypes.data_as(_I32P), i1.ctypes.data_as(_I32P)),
            "tp_fs_put_circuit_outputs_pixels")
        job.committed.synchronize()
        root = self.h["roots"][job.slot].numpy().tobytes()
        hx = "%016x%016x%016x%016x" % tuple(np.frombuffer(root, np.uint64)[[1, 0, 3, 2]])
        t.manifest = commit_manifest(L, hx, "", False)
        job.root = root
        t.fs.put(commit_binding(t.manifest))
        pair = lambda x: (int(x.real), int(x.imag)) if hasattr(x, "real") else (int(x[0]), int(x[1]))
        job.z1 = [pair(t.fs.rand_ext("z1-%d" % i)) for i in range((gt.size - 1).bit_length())]
        job.z2 = [pair(t.fs.rand_ext("z2-%d" % i)) for i in range(L.n_copy_bits)]
        # gate weights eq(z1, g) on the host
        k = len(job.z1)
        tab = np.empty(2 << k, np.uint64)
        z = np.ascontiguousarray(job.z1, np.uint64).reshape(-1)
        native.check(lib, lib.tp_eq_table_host(z.ctypes.data, k, tab.ctypes.data), "eq table")
        job.zg = tab.reshape(-1, 2)[:gt.size].copy()

    def _join_rounds(self, job: _Job):
        """the frame joins the running batch: beta, its gate form and bytes, its
        transcript, VOLE state, correlations and round counter uploaded to its slot"""
        torch, lib, L, s = self.torch, self.lib, job.L, job.slot
        c = job.req.circuit
        nb, S = L.n_copy_bits, self.slots
        h, d = self.h, self.d
        st = self.stream
        h["z2"].numpy().view(np.uint64).reshape(S, self.nbmax, 2)[s, :nb] = np.asarray(job.z2, np.uint64)
        nst, nvs, C = self.nst, self.nvs, self.count
        h["states"].numpy()[s * nst:(s + 1) * nst] = np.frombuffer(job.tr.fs.state(), np.uint8)
        h["vs"].numpy()[s * nvs:(s + 1) * nvs] = self.vs0
        u, v = job.req.correlations
        m = min(len(u), C)
        hu = h["u"].numpy().view(np.uint64).reshape(S, C, 2)
        hv = h["v"].numpy().view(np.uint64).reshape(S, C, 2)
        hu[s, :m] = np.asarray(u, np.uint64)[:m]
        hv[s, :m] = np.asarray(v, np.uint64)[:m]
        hu[s, m:] = 0
        hv[s, m:] = 0
        h["meta"].numpy()[2 * s:2 * s + 2] = (0, nb)
        G = c.gate_type.size
        h["zg"].numpy().view(np.uint64).reshape(S, 1024, 2)[s, :G] = job.zg
        sl = lambda t, k: t[k * s:k * (s + 1)]
        with torch.cuda.stream(st):
            st.wait_event(job.uploaded)
            sl(d["z2"], 2 * self.nbmax).copy_(sl(h["z2"], 2 * self.nbmax), non_blocking=True)
            sl(d["states"], nst).copy_(sl(h["states"], nst), non_blocking=True)
            sl(d["vs"], nvs).copy_(sl(h["vs"], nvs), non_blocking=True)
            sl(d["u"], 2 * C).copy_(sl(h["u"], 2 * C), non_blocking=True)
            sl(d["v"], 2 * C).copy_(sl(h["v"], 2 * C), non_blocking=True)
            sl(d["meta"], 2).copy_(sl(h["meta"], 2), non_blocking=True)
            sl(d["zg"], 2048).copy_(sl(h["zg"], 2048), non_blocking=True)
        z2p = d["z2"].data_ptr() + 16 * self.nbmax * s
        beta = d["beta"][s]
        native.check(lib, lib.tp_compute_beta_dev(z2p, nb, 1, 0, beta.data_ptr(), st.cuda_stream), "beta")
        gt, i0, i1 = (np.ascontiguousarray(a, np.int32) for a in (c.gate_type, c.in0, c.in1))
        zr, zi = np.ascontiguousarray(job.zg[:, 0]), np.ascontiguousarray(job.zg[:, 1])
        native.check(lib, lib.tp_batch_set_pixels(
            self.batch, s, gt.size, gt.ctypes.data, i0.ctypes.data, i1.ctypes.data, zr.ctypes.data, zi.ctypes.data,
            job.pix.data_ptr(), L.copies, L.padded_copies, L.copy_size, L.n_wires, L.const_idx, L.const_val,
            beta.data_ptr()), "set_pixels")
        job.stage = "rounds"
        job.round = 0

    def _tick(self):
        """one round of every frame in its early rounds: claims (one launch per
        source kind), the VOLE-committed rounds of all slots (one launch), folds by
        the device challenges"""
        lib, d, st = self.lib, self.d, self.stream.cuda_stream
        l0 = lib.tp_batch_launches(self.batch)
        native.check(lib, lib.tp_batch_claim(self.batch, d["claims"].data_ptr()), "batch_claim")
        native.check(lib, lib.tp_vole_round_slots_dev(
            d["states"].data_ptr(), d["vs"].data_ptr(), self.slots, d["meta"].data_ptr(), d["claims"].data_ptr(),
            d["u"].data_ptr(), d["v"].data_ptr(), self.count, 0, d["chal"].data_ptr(), d["chal_hist"].data_ptr(),
            d["proof"].data_ptr(), self.nbmax, st), "vole round slots")
        native.check(lib, lib.tp_batch_fold_dev(self.batch, d["chal"].data_ptr()), "batch_fold_dev")
        self.launches += lib.tp_batch_launches(self.batch) - l0 + 1
        self.ticks += 1
        ev = self.torch.cuda.Event()
        ev.record(self.stream)
        self.tick_events.append(ev)
        for job in self.jobs:
            if job.stage == "rounds":
                job.round += 1
                if job.round == job.L.n_copy_bits:
                    self._late(job)

    def _late(self, job: _Job):
        """finish, then the late rounds and closing proofs on the late stream"""
        torch, lib, d, h, L, s = self.torch, self.lib, self.d, self.h, job.L, job.slot
        n, nb, S, C = self.n, L.n_copy_bits, self.slots, self.count
        wires = d["wires"].data_ptr() + 16 * 512 * s
        fin_beta = d["fin_beta"].data_ptr() + 16 * s
        native.check(lib, lib.tp_batch_finish_frame(self.batch, s, wires, fin_beta), "finish_frame")
        ev = torch.cuda.Event()
        ev.record(self.stream)
        ls = self.late_stream
        ls.wait_event(ev)
        c = job.req.circuit
        gt, i0, i1 = (np.ascontiguousarray(a, np.int32) for a in (c.gate_type, c.in0, c.in1))
        at = lambda t, k: t.data_ptr() + k * s
        native.check(lib, lib.tp_late_rounds_dev(
            1, n, gt.size, gt.ctypes.data_as(_I32P), i0.ctypes.data_as(_I32P), i1.ctypes.data_as(_I32P), wires,
            fin_beta, at(d["zg"], 16 * 1024), 1, None, at(d["states"], self.nst), at(d["vs"], self.nvs),
            at(d["u"], 16 * C), at(d["v"], 16 * C), C, 0, nb, at(d["coefs"], 16 * 6 * n),
            at(d["line"], 16 * (n + 1)), at(d["chal_out"], 16 * 2 * n), at(d["late"], 16 * 8 * n),
            at(d["z2"], 16 * self.nbmax), at(d["chal_hist"], 16 * self.nbmax), 0, 1,
            at(d["closing"], 16 * (n + 10)), at(d["point"], 16 * (n + self.nbmax)), at(d["tag"], 16), 0,
            ls.cuda_stream), "tp_late_rounds_dev")
        self.launches += 2
        sl = lambda t, k: t[k * s:k * (s + 1)]
        with torch.cuda.stream(ls):
            sl(h["proof"], 10 * self.nbmax).copy_(sl(d["proof"], 10 * self.nbmax), non_blocking=True)
            sl(h["late"], 16 * n).copy_(sl(d["late"], 16 * n), non_blocking=True)
            sl(h["closing"], 2 * (n + 10)).copy_(sl(d["closing"], 2 * (n + 10)), non_blocking=True)
            sl(h["point"], 2 * (n + self.nbmax)).copy_(sl(d["point"], 2 * (n + self.nbmax)), non_blocking=True)
            sl(h["tag"], 2).copy_(sl(d["tag"], 2), non_blocking=True)
            sl(h["states_out"], self.nst).copy_(sl(d["states"], self.nst), non_blocking=True)
            sl(h["vs_out"], self.nvs).copy_(sl(d["vs"], self.nvs), non_blocking=True)
            job.event = torch.cuda.Event()
            job.event.record(ls)
        job.stage = "late"

    def _record(self, job: _Job):
        """the proof values the device put, into the frame's proof container"""
        h, L, s, n = self.h, job.L, job.slot, self.n
        nb = L.n_copy_bits
        if struct.unpack_from("<I", h["vs_out"].numpy().tobytes(), s * self.nvs + 12)[0]:
            raise IndexError("request %d: VOLE correlations ran out" % job.req.rid)
        early = h["proof"].numpy().view(np.uint64).reshape(self.slots, self.nbmax, 5, 2)[s, :nb]
        late = h["late"].numpy().view(np.uint64).reshape(self.slots, 2 * n, 4, 2)[s]
        closing = h["closing"].numpy().view(np.uint64).reshape(self.slots, n + 10, 2)[s]
        point = h["point"].numpy().view(np.uint64).reshape(self.slots, n + self.nbmax, 2)[s, :n + nb]
        tag = h["tag"].numpy().view(np.uint64).reshape(self.slots, 2)[s]
        t = job.tr
        t.record(early, late, closing, point, tag, zk=False)
        t.fs.set_state(h["states_out"].numpy()[s * self.nst:(s + 1) * self.nst].tobytes())
        job.point = [(int(a), int(b)) for a, b in point]

    def _open_host(self, job: _Job):
        """host thread: the proof record, the opening's eq tables, queried columns and node list"""
        self._record(job)
        lib, N = self.lib, job.N
        pt = job.point
        lg = len(pt)
        c0, c1 = pt[lg - 7:], pt[:lg - 7]
        r0 = np.empty((COLUMN_SIZE, 2), np.uint64)
        r1 = np.empty((N // COLUMN_SIZE, 2), np.uint64)
        z0 = np.ascontiguousarray(c0, np.uint64).reshape(-1)
        z1 = np.ascontiguousarray(c1, np.uint64).reshape(-1)
        native.check(lib, lib.tp_eq_table_host(z0.ctypes.data, len(c0), r0.ctypes.data), "eq table")
        native.check(lib, lib.tp_eq_table_host(z1.ctypes.data, len(c1), r1.ctypes.data), "eq table")
        qc = query_count()
        q = np.empty(qc, np.int64)
        native.check(lib, lib.tp_orion_open_queries(job.root, N, 1, r0.ctypes.data, len(r0), r1.ctypes.data, len(r1),
                                                    job.cw_len, -1, qc, q.ctypes.data), "tp_orion_open_queries")
        if q.min() < 0 or q.max() >= job.cw_len:
            raise IndexError("queried column outside the codeword")
        m = job.mem
        cap = m["h_idx"].numel()
        idx = m["h_idx"].numpy()
        nn = lib.tp_orion_path_nodes(job.leaves, q.ctypes.data, qc, idx.ctypes.data, cap)
        native.check(lib, 0 if nn >= 0 else -1, "tp_orion_path_nodes")
        job.q, job.nn = q, nn
        m["h_q"].numpy()[:qc] = q
        # (img, real): the codeword's element order
        m["h_r0"].numpy().view(np.uint64).reshape(-1, 2)[:len(r0)] = r0[:, ::-1]
        m["h_r1"].numpy().view(np.uint64).reshape(-1, 2)[:len(r1)] = r1[:, ::-1]

    def _open_device(self, job: _Job):
        """the opening's passes over the frame's codeword on the open stream, in the
        slot's buffers"""
        torch, lib = self.torch, self.lib
        os_ = self.open_stream
        sp = os_.cuda_stream
        m = job.mem
        qc, nn, N = len(job.q), job.nn, job.N
        nr1 = 2 * (N // COLUMN_SIZE)
        with torch.cuda.stream(os_):
            os_.wait_event(job.committed)
            os_.wait_event(job.event)
            m["r0"].copy_(m["h_r0"], non_blocking=True)
            m["r1"][:nr1].copy_(m["h_r1"][:nr1], non_blocking=True)
            m["q"][:qc].copy_(m["h_q"][:qc], non_blocking=True)
            m["idx"][:nn].copy_(m["h_idx"][:nn], non_blocking=True)
            rows = job.rows.data_ptr()
            comb, ctree, cols, nodes = m["comb"], m["ctree"], m["cols"], m["nodes"]
            native.check(lib, lib.tp_orion_combine_dev(rows, N, m["r0"].data_ptr(), comb.data_ptr(), ctree.data_ptr(),
                                                       sp), "combine")
            native.check(lib, lib.tp_orion_answer_dev(comb.data_ptr(), N // COLUMN_SIZE, m["r1"].data_ptr(),
                                                      m["ans"].data_ptr(), sp), "answer")
            native.check(lib, lib.tp_orion_query_columns_async_dev(rows, N, m["q"].data_ptr(), qc, cols.data_ptr(),
                                                                   None, sp), "query columns")
            native.check(lib, lib.tp_orion_gather_nodes_dev(job.tree.data_ptr(), 2 * job.leaves, m["idx"].data_ptr(),
                                                            nn, nodes.data_ptr(), sp), "gather")
            native.check(lib, lib.tp_orion_gather_nodes_dev(ctree.data_ptr(), 2 * job.leaves, m["idx"].data_ptr(), nn,
                                                            nodes.data_ptr() + 32 * nn, sp), "gather")
            self.launches += 6 + -(-int(math.log2(job.leaves)) // 9)
            cw = 2 * job.cw_len
            m["h_comb"][:cw].copy_(comb[:cw], non_blocking=True)
            m["h_ans"].copy_(m["ans"], non_blocking=True)
            m["h_cols"].copy_(cols, non_blocking=True)
            m["h_root"].copy_(ctree[32:64], non_blocking=True)
            m["h_nodes"][:64 * nn].copy_(nodes[:64 * nn], non_blocking=True)
            job.event = torch.cuda.Event()
            job.event.record(os_)
        job.stage = "open_dev"

    def _assemble(self, job: _Job) -> FrameProof:
        job.event.synchronize()
        m, N, nn = job.mem, job.N, job.nn
        nodes = m["h_nodes"].numpy()[:64 * nn].reshape(-1, 32)
        idx = m["h_idx"].numpy()[:nn]
        data = opening_bytes(N, N // COLUMN_SIZE, job.cw_len, m["h_ans"].numpy().view(np.uint64), job.root,
                             m["h_root"].numpy().tobytes(), job.q, m["h_cols"].numpy().view(np.uint64),
                             m["h_comb"].numpy()[:2 * job.cw_len].view(np.uint64).reshape(-1, 2), (idx, nodes[:nn]),
                             (idx, nodes[nn:2 * nn]), use_group1=1)
        t = job.tr
        return FrameProof(t.pid, t, t.manifest, data)

    # ---- the loop -----------------------------------------------------------------
    def _advance(self) -> bool:
        """move every job whose stage is done; True when anything moved"""
        moved = False
        keep = []
        for job in self.jobs:
            if job.stage == "io" and job.future.done():
                job.future.result()
                self._join_rounds(job)
                moved = True
            elif job.stage == "late" and job.event.query():
                job.future = self.pool.submit(self._open_host, job)
                job.stage = "open_host"
                moved = True
            elif job.stage == "open_host" and job.future.done():
                job.future.result()
                self._open_device(job)
                moved = True
            elif job.stage == "open_dev" and job.event.query():
                job.future = self.pool.submit(self._assemble, job)
                job.stage = "assemble"
                moved = True
            elif job.stage == "assemble" and job.future.done():
                proof = job.future.result()
                self._out.append(Result(job.req.rid, proof, job.req.arrival, time.perf_counter() - self._t0))
                self.used -= job.footprint
                self.free.append(job.slot)
                job.rows = job.tree = job.mem = None
                moved = True
                continue
            keep.append(job)
        self.jobs = keep
        return moved

    def run(self, requests, realtime: bool = True):
        """Serve `requests`. realtime: a request enters the queue when the wall
        clock reaches its arrival time; otherwise all are queued at once (in
        arrival order). Returns the results in completion order."""
        import sys
        reqs = sorted(requests, key=lambda r: r.arrival)
        queue = []
        self._out = []
        i = 0
        # the loop thread hands work to host threads that hold the interpreter lock in
        # short stretches (numpy assembly, transcript puts): a short switch interval
        # lets it take the lock back soon
        switch = sys.getswitchinterval()
        sys.setswitchinterval(2e-4)
        try:
            return self._run(reqs, queue, i, realtime)
        finally:
            sys.setswitchinterval(switch)

    def _run(self, reqs, queue, i, realtime):
        self._t0 = t0 = time.perf_counter()
        while i < len(reqs) or queue or self.jobs:
            now = time.perf_counter() - t0
            while i < len(reqs) and (not realtime or reqs[i].arrival <= now):
                queue.append(reqs[i])
                i += 1
            while queue and self.free:
                L = layout_for(queue[0].circuit, queue[0].height, queue[0].width)
                if self.jobs and self.used + self.footprint(L) > self.budget:
                    break
                req = queue.pop(0)
                if not realtime:
                    req.arrival = time.perf_counter() - t0
                self._admit(req)
            moved = self._advance()
            self.tick_events = [e for e in self.tick_events if not e.query()]
            if len(self.tick_events) < self.max_ticks_ahead and any(j.stage == "rounds" for j in self.jobs):
                self._tick()
                moved = True
            if not moved:
                time.sleep(0.0002)
        return self._out


def latency_stats(results):
    lat = sorted(r.latency for r in results)
    if not lat:
        return {}
    pick = lambda q: lat[min(len(lat) - 1, int(q * len(lat)))]
    span = max(r.done for r in results) - min(r.arrival for r in results)
    return {"p50_ms": 1e3 * pick(0.5), "p99_ms": 1e3 * pick(0.99), "mean_ms": 1e3 * sum(lat) / len(lat),
            "frames": len(lat), "frames_per_s": len(lat) / span if span > 0 else None}
