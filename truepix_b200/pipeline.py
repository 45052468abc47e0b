"""Whole proofs of many frames, pipelined: for every frame the proof the
reference's prover phase writes (TruePix-main/run_truepix_prover.py:218-421):
the GKR input layer's NIZK proof of CircuitProverNIZK.run
(libTruePix/circuitnizkvec_vole.py:265-500; with zk=True the zero-knowledge
prover, circuitnizkvec_vole_ZK.py:293-520) and the Orion opening proof of the
frame's committed input (linearPC_multi_prove's orion_proof.bin,
Orion_nonzk/src/VPD/linearPC.cpp:426-640, src/truepix/orion_proof.cpp:67-95), for
batches of frames of one layout and circuit.

Stages of a batch, and where they run:

  commit    device, side streams: the Orion commitment of every frame from its
            bytes (truepix_b200.orion.FrameCommitter); codewords and trees stay
            in HBM for the opening, the roots come back to pinned memory
  IO        host threads (a pool of their own): each frame's transcript puts
            its pid, the IO values and the circuit's output vector, computed from
            the frame's bytes and hashed as it is made, 16 frames per task in the
            lanes of the multi-buffer SHA-256 (tp_fs_put_circuit_outputs_pixels;
            the first batch of a run in pairs, for latency); this runs io_ahead
            batches ahead of the commits. Then, once a frame's root is back, the
            commitment binding and the GKR point's draws z1, z2
  GKR       device, main stream: gate weights and beta, the VOLE-committed
            early rounds, late rounds and closing proofs of all frames, each
            frame's transcript and VOLE state resident on the device
            (truepix_b200.frame.BatchFrameProver.prove / prove_late); the
            first batch's rounds run launch by launch with the round autotuner
            on, every later batch replays them as one CUDA graph
  opening   host threads: the point's eq tables and the Orion transcript's
            queried columns and Merkle node lists; device: the combined codeword,
            its tree and the answer, the queried columns and the Merkle nodes
            gathered over the HBM-resident codeword and trees; host threads:
            the opening file's bytes

Batches overlap: while the device commits batch b on the side streams, the main
stream proves and opens batch b - 1, the host threads assemble batch b - 2's
proofs (handed out once batch b - 1 is proved) and hash the IO of batches
b .. b + io_ahead.
Every value is the reference's: truepix_b200.prover.prove_frames and
truepix_b200.opening.opening_proof produce the same proofs one step at a time
and are pinned to proofs and files made by the reference itself.
"""
from __future__ import annotations

import collections
import concurrent.futures
import ctypes
import math
import os
import struct
import threading

import numpy as np

from . import native
from .fiatshamir import P61
from .opening import COLUMN_SIZE, opening_bytes, query_count
from .prover import LayerTranscript, commit_binding, commit_manifest

_I32P = ctypes.POINTER(ctypes.c_int)


def correlations_needed(layout, zk: bool = False) -> int:
    """VOLE correlations one frame's proof consumes: four per early round, three
    per late round, and the closing proofs' n + 2 commitments (three more for
    the zero-knowledge prover's masks)."""
    n = layout.n_in_bits
    return 4 * layout.n_copy_bits + 6 * n + n + 2 + (3 if zk else 0)


class CircuitOutputs:
    """A frame's circuit output vector as the proof container holds it (the io
    value circuitnizkvec_vole.py:351-355 puts), kept as the frame's bytes and
    evaluated on the device when the container is serialised."""

    def __init__(self, pixels_host: np.ndarray, layout, gt, i0, i1, device):
        self.pixels, self.layout, self.gates, self.device = pixels_host, layout, (gt, i0, i1), device

    def values(self) -> np.ndarray:
        import torch
        from .frame import circuit_outputs
        L = self.layout
        full = np.zeros(L.copies * L.copy_size, np.uint8)        # a short last copy is zero-padded
        n = min(full.size, self.pixels.size)
        full[:n] = np.asarray(self.pixels).reshape(-1)[:n]
        pix = torch.from_numpy(full).to(self.device)
        out = circuit_outputs(pix, self.layout, *self.gates)
        torch.cuda.synchronize(self.device)
        return out.cpu().numpy().view(np.uint64)


class FrameProof:
    """One frame's proof: `transcript` (truepix_b200.prover.LayerTranscript; its
    proof_bytes() is the reference prover's proof container), the commitment
    `manifest`, and `opening`: the orion_proof.bin bytes (zero-knowledge: a dict
    with the masked polynomial's and the mask's files)."""
    __slots__ = ("pid", "transcript", "manifest", "opening")

    def __init__(self, pid, transcript, manifest, opening):
        self.pid, self.transcript, self.manifest, self.opening = pid, transcript, manifest, opening

    def proof_bytes(self) -> bytes:
        t = self.transcript
        io = t.fs.io
        saved = list(io)
        io.clear()
        io.extend(v.values() if isinstance(v, CircuitOutputs) else v for v in saved)
        try:
            return t.proof_bytes()
        finally:
            io.clear()
            io.extend(saved)


class _Pending:
    """A batch taken from the input whose IO hashing is under way: its frames'
    host views, transcripts and hashing futures (one per group of frames)."""
    batch: dict
    host_t: list
    frames_host: list
    tr: list
    groups: list
    hashed: list


class _Slot:
    """Device and pinned host buffers of one batch in flight."""

    def __init__(self, pipe):
        import torch
        self.torch = torch
        from .orion import FrameCommitter
        p = pipe
        self.committer = FrameCommitter([p.layout] * p.B, device=p.dev.index, stream=p.stream,
                                        side_streams=p.commit_streams, zk=p.zk)
        n_trees = 2 if p.zk else 1
        self.roots = torch.empty((n_trees, p.B, 32), dtype=torch.uint8).pin_memory()
        self.root_events = []
        self.io = []
        self.assembly = []
        # opening buffers per frame and polynomial (device) and their pinned copies
        cw, qc, lv = p.cw_len, p.qc, p.leaves
        self.max_nodes = qc * int(math.log2(lv))
        self.open_dev = [[dict(comb=torch.empty(2 * cw, dtype=torch.int64, device=p.dev),
                               ctree=torch.empty(64 * lv, dtype=torch.uint8, device=p.dev),
                               ans=torch.empty(2, dtype=torch.int64, device=p.dev),
                               cols=torch.empty(2 * COLUMN_SIZE * qc, dtype=torch.int64, device=p.dev),
                               nodes_com=torch.empty(32 * self.max_nodes, dtype=torch.uint8, device=p.dev),
                               nodes_comb=torch.empty(32 * self.max_nodes, dtype=torch.uint8, device=p.dev),
                               r0=torch.empty(2 * COLUMN_SIZE, dtype=torch.int64, device=p.dev),
                               r1=torch.empty(2 * (p.N // COLUMN_SIZE), dtype=torch.int64, device=p.dev),
                               q=torch.empty(qc, dtype=torch.int64, device=p.dev),
                               idx=torch.empty(self.max_nodes, dtype=torch.int32, device=p.dev))
                          for _ in range(n_trees)] for _ in range(p.B)]
        self.open_host = [[dict(comb=torch.empty(2 * cw, dtype=torch.int64).pin_memory(),
                                ctree_root=torch.empty(32, dtype=torch.uint8).pin_memory(),
                                ans=torch.empty(2, dtype=torch.int64).pin_memory(),
                                cols=torch.empty(2 * COLUMN_SIZE * qc, dtype=torch.int64).pin_memory(),
                                nodes_com=torch.empty(32 * self.max_nodes, dtype=torch.uint8).pin_memory(),
                                nodes_comb=torch.empty(32 * self.max_nodes, dtype=torch.uint8).pin_memory(),
                                r0=torch.empty(2 * COLUMN_SIZE, dtype=torch.int64).pin_memory(),
                                r1=torch.empty(2 * (p.N // COLUMN_SIZE), dtype=torch.int64).pin_memory(),
                                q=torch.empty(qc, dtype=torch.int64).pin_memory(),
                                idx=torch.empty(self.max_nodes, dtype=torch.int32).pin_memory())
                           for _ in range(n_trees)] for _ in range(p.B)]
        self.opened = torch.cuda.Event()
        # the GKR's inputs and results in pinned memory: per slot, since a batch's
        # results are read (opener thread) while the next batch's GKR is launched
        B, nb, n, i64 = p.B, p.nb, p.n, torch.int64
        nst, nvs = p.lib.tp_fs_state_bytes(), p.lib.tp_vole_state_bytes()
        self.h_in = dict(z2=torch.empty(2 * B * nb, dtype=i64).pin_memory(),
                         states=torch.empty(B * nst, dtype=torch.uint8).pin_memory(),
                         vs=torch.empty(B * nvs, dtype=torch.uint8).pin_memory(),
                         u=torch.empty(2 * B * p.count, dtype=i64).pin_memory(),
                         v=torch.empty(2 * B * p.count, dtype=i64).pin_memory())
        ncl = n + (15 if p.zk else 10)
        self.h_out = dict(early=torch.empty(nb * B * 10, dtype=i64).pin_memory(),
                          late=torch.empty(B * 2 * n * 4 * 2, dtype=i64).pin_memory(),
                          closing=torch.empty(B * ncl * 2, dtype=i64).pin_memory(),
                          point=torch.empty(B * (n + nb) * 2, dtype=i64).pin_memory(),
                          tag=torch.empty(B * 2, dtype=i64).pin_memory(),
                          states=torch.empty(B * nst, dtype=torch.uint8).pin_memory(),
                          vs=torch.empty(B * nvs, dtype=torch.uint8).pin_memory())
        self.inputs_sent = torch.cuda.Event()   # h_in copied to the device: free to refill
        self.gkr_done = torch.cuda.Event()


class ProofPipeline:
    """Proves batches of `batch` frames of one `layout` (truepix_b200.frame.FrameLayout)
    and circuit (gate tables) end to end; see the module docstring.

    run(batches) takes an iterable of batches, each a dict with
      frames_host  uint8 numpy arrays (layout.copies * layout.copy_size bytes),
                   pinned (torch) or plain: the IO transcript hashes them
      frames_dev   uint8 device tensors of the same bytes (optional: else they
                   are copied to the device on the upload stream)
      pids         the prover process ids the transcripts put first
      correlations per frame (u, v) uint64 [count, 2], count >=
                   correlations_needed(layout, zk) (the reference's VOLE prover
                   file, truepix_b200.prover.read_vole_prover_file)
      mask_seeds   zk only: one 64-bit mask seed per frame
      manifests    optional: the commitment manifests the transcripts bind
                   (truepix_b200.prover.commit_manifest); by default each frame's
                   manifest is made from its device commit's roots
    and yields, per batch, the list of FrameProof. io_group frames are hashed per
    IO task (0: 16 where the host has the multi-buffer SHA-256, else 2), on
    io_threads threads (0: one per CPU but four), io_ahead batches ahead of the
    commits; host_threads run the bindings, openings (open_group per task, their
    transcripts hashed in lockstep: 16 use the multi-buffer SHA-256's lanes, at a
    longer latency per task than the default 2) and assembly. `slots` batches
    hold device buffers at once (each frame's codewords and trees, 231 MB per
    committed 1080p polynomial): with three, a batch's commits never wait for the
    assembly of the batch two before it."""

    def __init__(self, layout, gate_type, in0, in1, batch: int, device: int = 0, zk: bool = False,
                 host_threads: int = 0, commit_streams: int = 8, fp2_type=None, graph: bool = True,
                 io_group: int = 0, io_ahead: int = 3, io_threads: int = 0, slots: int = 3, open_group: int = 0):
        import torch
        from .frame import BatchFrameProver
        self.torch = torch
        self.lib = native.gkr()
        self.layout = layout
        self.B = batch
        self.zk = zk
        self.fp2_type = fp2_type
        self.dev = torch.device("cuda", device)
        self.stream = torch.cuda.Stream(self.dev)
        self.upload = torch.cuda.Stream(self.dev)
        self.commit_streams = commit_streams
        self.gt, self.i0, self.i1 = (np.ascontiguousarray(a, np.int32) for a in (gate_type, in0, in1))
        self.G = self.gt.size
        self.n_out_bits = (self.G - 1).bit_length()
        self.n = layout.n_in_bits
        self.nb = layout.n_copy_bits
        self.N = layout.padded_copies * layout.n_wires
        self.cw_len = self.lib.tp_orion_codeword_len(self.N // COLUMN_SIZE)
        self.leaves = self.lib.tp_orion_tree_leaves(self.N)
        self.qc = query_count()
        self.count = correlations_needed(layout, zk)
        self.prover = BatchFrameProver([layout] * batch, self.gt, self.i0, self.i1, device=device, stream=self.stream)
        self.slots = [_Slot(self) for _ in range(max(2, slots))]
        B, nb, n = batch, self.nb, self.n
        i64 = torch.int64
        self.d_z2 = torch.empty(2 * B * nb, dtype=i64, device=self.dev)
        self.d_pt = torch.zeros(2 * B * (n + nb), dtype=i64, device=self.dev)
        self.d_states = torch.empty(B * self.lib.tp_fs_state_bytes(), dtype=torch.uint8, device=self.dev)
        self.d_vs = torch.empty(B * self.lib.tp_vole_state_bytes(), dtype=torch.uint8, device=self.dev)
        self.d_u = torch.empty(2 * B * self.count, dtype=i64, device=self.dev)
        self.d_v = torch.empty(2 * B * self.count, dtype=i64, device=self.dev)
        vs0 = ctypes.create_string_buffer(self.lib.tp_vole_state_bytes())
        native.check(self.lib, self.lib.tp_vole_state_init(vs0, 0, None), "tp_vole_state_init")
        self.vs0 = vs0.raw
        self.pool = concurrent.futures.ThreadPoolExecutor(host_threads or os.cpu_count() or 4)
        # the IO hashing on a pool of its own, so that the long hashing tasks of
        # the batches ahead never queue in front of the current batch's openings
        self.io_pool = concurrent.futures.ThreadPoolExecutor(io_threads or max(1, (os.cpu_count() or 4) - 4))
        mb = self.lib.tp_host_sha_mb_available()
        self.io_group = io_group or (16 if mb else 2)
        self.open_group = open_group or 2
        self.io_ahead = io_ahead
        # waits on device events and hashing that would otherwise hold host pool threads
        self.waiter = concurrent.futures.ThreadPoolExecutor(1)
        self.binder = concurrent.futures.ThreadPoolExecutor(1)
        # a batch's GKR results are read, and its openings run, on a thread and a
        # stream of their own while the main thread launches the next batch's GKR
        self.opener = concurrent.futures.ThreadPoolExecutor(1)
        self.open_stream = torch.cuda.Stream(self.dev)
        self._count_lock = threading.Lock()
        self.launches_last = 0
        # the first batch's rounds run launch by launch with the round autotuner on;
        # later batches replay them as one CUDA graph (BatchFrameProver.prove(graph=True))
        self.graph = graph
        self.tuned = False

    def _count(self, k: int) -> None:
        with self._count_lock:
            self.launches_last += k

    def close(self):
        self.opener.shutdown(wait=True)
        self.binder.shutdown(wait=True)
        self.waiter.shutdown(wait=True)
        self.io_pool.shutdown(wait=True)
        self.pool.shutdown(wait=True)

    # ---- stage: commits ---------------------------------------------------------
    def _start(self, slot: _Slot, pend: "_Pending") -> None:
        torch, B = self.torch, self.B
        for f in slot.assembly:          # the slot's previous batch is assembled
            f.result()
        slot.assembly = []
        batch = pend.batch
        slot.pending = pend
        slot.batch = batch
        slot.frames_host = pend.frames_host
        slot.tr = pend.tr
        if batch.get("frames_dev") is not None:
            frames_dev = list(batch["frames_dev"])
            ready = None
        else:   # uploads on their own stream (pinned frames: asynchronous), each commit waits for its frame
            frames_dev, ready = [], []
            with torch.cuda.stream(self.upload):
                for a in pend.host_t:
                    frames_dev.append(a.to(self.dev, non_blocking=True))
                    ev = torch.cuda.Event()
                    ev.record(self.upload)
                    ready.append(ev)
        slot.frames_dev = frames_dev
        slot.upload_ready = ready
        c = slot.committer
        # each frame's roots back to pinned memory right behind its own commit, with
        # an event per frame: a frame's binding waits for that commit only
        slot.root_events = [None] * B

        def roots_of(f):
            slot.roots[0, f].copy_(c.trees[f][32:64], non_blocking=True)
            if self.zk:
                slot.roots[1, f].copy_(c.mask_trees[f][32:64], non_blocking=True)
            ev = torch.cuda.Event()
            ev.record()
            slot.root_events[f] = ev

        c.commit(frames_dev, join=False, mask_seeds=batch.get("mask_seeds") if self.zk else None, ready=ready,
                 after=roots_of)
        # the main stream joins the commits only when it proves this batch (_finish)
        self._count(c.launches_last)
        # the commitment bindings, two frames per host task, each once its
        # frames are hashed and their roots are back (the bind thread waits)
        pairs = [list(range(f, min(f + 2, B))) for f in range(0, B, 2)]
        slot.io = [concurrent.futures.Future() for _ in pairs]
        self.binder.submit(self._bind_when_ready, slot, pairs, slot.io)

    # ---- stage: IO hashing (runs ahead of the commits) ------------------------
    def _prehash(self, batch: dict, group: int) -> "_Pending":
        """the batch's IO hashing, started on the IO pool before the batch has a slot"""
        torch, B = self.torch, self.B
        pend = _Pending()
        pend.batch = batch
        pend.host_t = [a if torch.is_tensor(a) else torch.from_numpy(np.ascontiguousarray(a, np.uint8).reshape(-1))
                       for a in batch["frames_host"]]
        pend.frames_host = [a.numpy() for a in pend.host_t]
        pend.tr = [LayerTranscript(batch["pids"][f], self.fp2_type) for f in range(B)]
        pend.groups = [list(range(f, min(f + group, B))) for f in range(0, B, group)]
        pend.hashed = [self.io_pool.submit(self._io_hash, pend, fs) for fs in pend.groups]
        return pend

    def _io_hash(self, pend: "_Pending", fs) -> None:
        """the IO transcript of frames fs up to the circuit's output vector, the
        vectors hashed together (tp_fs_put_circuit_outputs_pixels)"""
        L = self.layout
        n_inputs = L.padded_copies * L.n_wires
        trs = [pend.tr[f] for f in fs]
        for f, t in zip(fs, trs):
            t.fs.put(t.pid)
            t.fs.put(None, True)
            t.fs.put(["private_input_omitted", int(n_inputs)], True)
            t.fs.io.append(CircuitOutputs(pend.frames_host[f], L, self.gt, self.i0, self.i1, self.dev))
        states = (ctypes.c_void_p * len(fs))(*[ctypes.addressof(t.fs._st) for t in trs])
        pix = (ctypes.c_void_p * len(fs))(*[pend.frames_host[f].ctypes.data for f in fs])
        n_bytes = min(pend.frames_host[f].size for f in fs)
        native.check(self.lib, self.lib.tp_fs_put_circuit_outputs_pixels(
            states, pix, n_bytes, len(fs), L.copies, L.padded_copies, L.copy_size, L.n_wires, L.const_idx, L.const_val,
            self.G, self.gt.ctypes.data_as(_I32P), self.i0.ctypes.data_as(_I32P), self.i1.ctypes.data_as(_I32P)),
            "tp_fs_put_circuit_outputs_pixels")

    def _bind_when_ready(self, slot: _Slot, pairs, futs) -> None:
        """(bind thread) hands each pair of frames' commitment binding to the host
        pool once their hashing is done and their roots are on the host"""
        pend = slot.pending
        group_of = {f: g for g, fs in enumerate(pend.groups) for f in fs}
        for fs, fut in zip(pairs, futs):
            try:
                for g in sorted({group_of[f] for f in fs}):
                    pend.hashed[g].result()
                for f in fs:
                    slot.root_events[f].synchronize()
            except BaseException as e:      # handed to the pair's future
                fut.set_exception(e)
                continue
            self.pool.submit(self._io_bind_into, slot, fs, fut)

    def _io_bind_into(self, slot: _Slot, fs, fut) -> None:
        try:
            self._io_bind(slot, fs)
            fut.set_result(None)
        except BaseException as e:      # handed to the pair's future
            fut.set_exception(e)

    def _io_bind(self, slot: _Slot, fs) -> None:
        """the commitment binding of frames fs (their roots are on the host) and
        the GKR point's draws z1, z2"""
        L = self.layout
        given = slot.batch.get("manifests")
        for f in fs:
            t = slot.tr[f]
            if given is not None:
                t.manifest = given[f]
            else:
                root = slot.roots[0, f].numpy().tobytes()
                mask = slot.roots[1, f].numpy().tobytes() if self.zk else b""
                hx = lambda r: "%016x%016x%016x%016x" % tuple(np.frombuffer(r, np.uint64)[[1, 0, 3, 2]])
                t.manifest = commit_manifest(L, hx(root), hx(mask) if self.zk else "", self.zk)
            t.fs.put(commit_binding(t.manifest))
            pair = lambda x: (int(x.real), int(x.imag)) if hasattr(x, "real") else (int(x[0]), int(x[1]))
            t.z1 = [pair(t.fs.rand_ext("z1-%d" % i)) for i in range(self.n_out_bits)]
            t.z2 = [pair(t.fs.rand_ext("z2-%d" % i)) for i in range(self.nb)]

    # ---- stage: GKR -------------------------------------------------------------
    def _gkr(self, slot: _Slot) -> None:
        """(main thread) the batch's GKR launched on the main stream, its results
        copied back to the slot's pinned buffers behind it (slot.gkr_done)"""
        torch, lib, B, nb, n = self.torch, self.lib, self.B, self.nb, self.n
        slot.committer.join()      # the main stream waits for this batch's commits (and uploads)
        for f in slot.io:
            f.result()
        tr = slot.tr
        # gate weights eq(z1, g) on the host; beta's z2, transcripts, VOLE states, correlations uploaded
        zg = []
        tab = np.empty(2 << self.n_out_bits, np.uint64)
        for t in tr:
            z = np.ascontiguousarray(t.z1, np.uint64).reshape(-1)
            native.check(lib, lib.tp_eq_table_host(z.ctypes.data, self.n_out_bits, tab.ctypes.data), "eq table")
            w = tab.reshape(-1, 2)[:self.G]
            zg.append(np.stack([w[:, 0].copy(), w[:, 1].copy()]))
        h = slot.h_in
        slot.inputs_sent.synchronize()      # the slot's previous batch has sent them
        h["z2"].numpy().view(np.uint64)[:] = np.asarray([t.z2 for t in tr], np.uint64).reshape(-1)
        nst = lib.tp_fs_state_bytes()
        st = h["states"].numpy()
        for f, t in enumerate(tr):
            st[f * nst:(f + 1) * nst] = np.frombuffer(t.fs.state(), np.uint8)
        h["vs"].numpy()[:] = np.frombuffer(self.vs0 * B, np.uint8)
        corr = slot.batch["correlations"]
        u, v = h["u"].numpy().view(np.uint64).reshape(B, self.count, 2), h["v"].numpy().view(np.uint64).reshape(
            B, self.count, 2)
        for f in range(B):
            cu, cv = corr[f]
            if len(cu) < self.count:
                raise IndexError("frame %d: %d VOLE correlations given, %d needed" % (f, len(cu), self.count))
            u[f] = np.asarray(cu, np.uint64)[:self.count]
            v[f] = np.asarray(cv, np.uint64)[:self.count]
        s = self.stream
        with torch.cuda.stream(s):
            self.d_z2.copy_(h["z2"], non_blocking=True)
            self.d_states.copy_(h["states"], non_blocking=True)
            self.d_vs.copy_(h["vs"], non_blocking=True)
            self.d_u.copy_(h["u"], non_blocking=True)
            self.d_v.copy_(h["v"], non_blocking=True)
        slot.inputs_sent.record(s)
        vole = dict(states=self.d_vs, u=self.d_u, v=self.d_v, count=self.count)
        bp = self.prover
        from .frame import autotune_rounds
        if not self.tuned:
            autotune_rounds(True)
            try:
                bp.prove(slot.frames_dev, zg, self.d_z2, self.d_pt, None, transcripts=self.d_states, vole=vole)
            finally:
                autotune_rounds(False)
            self.tuned = True
        else:
            bp.prove(slot.frames_dev, zg, self.d_z2, self.d_pt, None, transcripts=self.d_states, vole=vole,
                     graph=self.graph)
        bp.prove_late(zg, transcripts=self.d_states, vole=vole, zk=self.zk)
        self._count(bp.launches_last + 1)
        o = slot.h_out
        with torch.cuda.stream(s):
            o["early"].copy_(bp.device_proof, non_blocking=True)
            o["late"].copy_(bp.late_proof, non_blocking=True)
            o["closing"].copy_(bp.closing, non_blocking=True)
            o["point"].copy_(bp.input_point, non_blocking=True)
            o["tag"].copy_(bp.input_tag, non_blocking=True)
            o["states"].copy_(self.d_states, non_blocking=True)
            o["vs"].copy_(self.d_vs, non_blocking=True)
        slot.gkr_done.record(s)

    def _read_gkr(self, slot: _Slot) -> None:
        """(opener thread) the batch's GKR results into its frames' transcripts"""
        lib, B, nb, n = self.lib, self.B, self.nb, self.n
        tr = slot.tr
        nst = lib.tp_fs_state_bytes()
        o = slot.h_out
        slot.gkr_done.synchronize()
        raw_st, raw_vs = o["states"].numpy().tobytes(), o["vs"].numpy().tobytes()
        nvs = lib.tp_vole_state_bytes()
        early = o["early"].numpy().view(np.uint64).reshape(nb, B, 5, 2)
        late = o["late"].numpy().view(np.uint64).reshape(B, 2 * n, 4, 2)
        closing = o["closing"].numpy().view(np.uint64).reshape(B, -1, 2)
        point = o["point"].numpy().view(np.uint64).reshape(B, n + nb, 2)
        tag = o["tag"].numpy().view(np.uint64).reshape(B, 2)
        for f, t in enumerate(tr):
            if struct.unpack_from("<I", raw_vs, f * nvs + 12)[0]:
                raise IndexError("frame %d: VOLE correlations ran out" % f)
            t.record(early[:, f], late[f], closing[f], point[f], tag[f], zk=self.zk)
            t.fs.set_state(raw_st[f * nst:(f + 1) * nst])
            t.point = [(int(a), int(b)) for a, b in point[f]]

    # ---- stage: openings ------------------------------------------------------
    def _open_host(self, slot: _Slot, items) -> None:
        """the opening's host part for the (frame, polynomial) pairs `items`
        (polynomial 0: the commit / the masked polynomial, 1: the mask): eq tables
        (once per frame), queried columns, node lists. The items' opening
        transcripts are hashed in lockstep (tp_orion_open_queries_multi)."""
        lib = self.lib
        eq = {}
        for f, _ in items:
            if f in eq:
                continue
            pt = slot.tr[f].point
            lg = len(pt)
            c0, c1 = pt[lg - 7:], pt[:lg - 7]
            r0 = np.empty((COLUMN_SIZE, 2), np.uint64)
            r1 = np.empty((self.N // COLUMN_SIZE, 2), np.uint64)
            z0 = np.ascontiguousarray(c0, np.uint64).reshape(-1)
            z1 = np.ascontiguousarray(c1, np.uint64).reshape(-1)
            native.check(lib, lib.tp_eq_table_host(z0.ctypes.data, len(c0), r0.ctypes.data), "eq table")
            native.check(lib, lib.tp_eq_table_host(z1.ctypes.data, len(c1), r1.ctypes.data), "eq table")
            eq[f] = (r0, r1)
        n = len(items)
        hbs = [slot.open_host[f][k] for f, k in items]
        qs = [hb["q"].numpy() for hb in hbs]
        addrs = lambda xs: np.array(xs, np.uint64)
        roots = addrs([slot.roots[k, f].data_ptr() for f, k in items])
        use_g1 = np.array([0 if k == 1 else 1 for _, k in items], np.int32)
        groups = np.array([-1 if not self.zk else k for _, k in items], np.int32)
        r0s = addrs([eq[f][0].ctypes.data for f, _ in items])
        r1s = addrs([eq[f][1].ctypes.data for f, _ in items])
        qp = addrs([q.ctypes.data for q in qs])
        native.check(lib, lib.tp_orion_open_queries_multi(n, roots.ctypes.data, self.N, use_g1.ctypes.data,
                                                          r0s.ctypes.data, COLUMN_SIZE, r1s.ctypes.data,
                                                          self.N // COLUMN_SIZE, self.cw_len, groups.ctypes.data,
                                                          self.qc, qp.ctypes.data, None),
                     "tp_orion_open_queries_multi")
        for (f, _), hb, q in zip(items, hbs, qs):
            r0, r1 = eq[f]
            hb["r0"].numpy().view(np.uint64).reshape(-1, 2)[:] = r0[:, ::-1]     # (img, real): the codeword's order
            hb["r1"].numpy().view(np.uint64).reshape(-1, 2)[:] = r1[:, ::-1]
            if self.qc and (q.min() < 0 or q.max() >= self.cw_len):
                raise IndexError("queried column outside the codeword")
            # the same positions open both trees: one node list
            hb["n_nodes"] = lib.tp_orion_path_nodes(self.leaves, q.ctypes.data, self.qc,
                                                    hb["idx"].numpy().ctypes.data, slot.max_nodes)
            native.check(lib, 0 if hb["n_nodes"] >= 0 else -1, "tp_orion_path_nodes")

    def _open_device(self, slot: _Slot, f: int, k: int) -> None:
        torch, lib = self.torch, native.gkr_launcher()
        hb, db = slot.open_host[f][k], slot.open_dev[f][k]
        c = slot.committer
        rows = (c.mask_rows[f] if k == 1 else c.rows[f]).data_ptr()
        tree = c.mask_trees[f] if k == 1 else c.trees[f]
        s = self.open_stream
        sp = s.cuda_stream
        n_nodes = hb["n_nodes"]
        with torch.cuda.stream(s):
            for key in ("r0", "r1", "q", "idx"):
                db[key].copy_(hb[key], non_blocking=True)
        native.check(lib, lib.tp_orion_combine_dev(rows, self.N, db["r0"].data_ptr(), db["comb"].data_ptr(),
                                                   db["ctree"].data_ptr(), sp), "tp_orion_combine_dev")
        native.check(lib, lib.tp_orion_answer_dev(db["comb"].data_ptr(), self.N // COLUMN_SIZE, db["r1"].data_ptr(),
                                                  db["ans"].data_ptr(), sp), "tp_orion_answer_dev")
        native.check(lib, lib.tp_orion_query_columns_async_dev(rows, self.N, db["q"].data_ptr(), self.qc,
                                                               db["cols"].data_ptr(), None, sp), "query columns")
        native.check(lib, lib.tp_orion_gather_nodes_dev(tree.data_ptr(), 2 * self.leaves, db["idx"].data_ptr(),
                                                        n_nodes, db["nodes_com"].data_ptr(), sp), "gather")
        native.check(lib, lib.tp_orion_gather_nodes_dev(db["ctree"].data_ptr(), 2 * self.leaves,
                                                        db["idx"].data_ptr(), n_nodes,
                                                        db["nodes_comb"].data_ptr(), sp), "gather")
        # combine, its leaves, its tree levels (nine per launch), answer, query, two gathers
        self._count(6 + -(-int(math.log2(self.leaves)) // 9))
        with torch.cuda.stream(s):
            hb["comb"].copy_(db["comb"], non_blocking=True)
            hb["ans"].copy_(db["ans"], non_blocking=True)
            hb["cols"].copy_(db["cols"], non_blocking=True)
            hb["ctree_root"].copy_(db["ctree"][32:64], non_blocking=True)
            hb["nodes_com"][:32 * n_nodes].copy_(db["nodes_com"][:32 * n_nodes], non_blocking=True)
            hb["nodes_comb"][:32 * n_nodes].copy_(db["nodes_comb"][:32 * n_nodes], non_blocking=True)

    def _assemble(self, slot: _Slot, f: int) -> FrameProof:
        slot.opened.synchronize()
        out = []
        for k in range(2 if self.zk else 1):
            hb = slot.open_host[f][k]
            n_nodes = hb["n_nodes"]
            idx = hb["idx"].numpy()[:n_nodes]
            com = hb["nodes_com"].numpy()[:32 * n_nodes].reshape(-1, 32)
            comb_nodes = hb["nodes_comb"].numpy()[:32 * n_nodes].reshape(-1, 32)
            msg_len = self.N // COLUMN_SIZE
            combined = hb["comb"].numpy().view(np.uint64).reshape(-1, 2)
            out.append(opening_bytes(self.N, msg_len, self.cw_len, hb["ans"].numpy().view(np.uint64),
                                     slot.roots[k, f].numpy().tobytes(), hb["ctree_root"].numpy().tobytes(),
                                     hb["q"].numpy(), hb["cols"].numpy().view(np.uint64), combined,
                                     (idx, com), (idx, comb_nodes), use_group1=0 if k == 1 else 1))
        t = slot.tr[f]
        opening = dict(masked=out[0], mask=out[1]) if self.zk else out[0]
        return FrameProof(t.pid, t, t.manifest, opening)

    def _finish(self, slot: _Slot) -> list:
        """(main thread) launches the batch's GKR and hands its openings to the
        opener thread; returns futures of its FrameProofs"""
        self._gkr(slot)
        slot.assembly = [concurrent.futures.Future() for _ in range(self.B)]
        self.opener.submit(self._open_batch, slot, slot.assembly)
        return slot.assembly

    def _open_batch(self, slot: _Slot, futs) -> None:
        """(opener thread) the GKR results into the transcripts, then the openings:
        host tasks of open_group openings each (in the zero-knowledge mode a
        frame's two polynomials side by side), their transcripts hashed in
        lockstep, each task followed by its device passes on the opening stream"""
        try:
            self.torch.cuda.set_device(self.dev)     # this thread's launches go to the pipeline's device
            self._read_gkr(slot)
            self.open_stream.wait_event(slot.gkr_done)
            items = [(f, k) for f in range(self.B) for k in range(2 if self.zk else 1)]
            per = self.open_group
            groups = [items[g:g + per] for g in range(0, len(items), per)]
            host = [self.pool.submit(self._open_host, slot, g) for g in groups]
            for g, fut in zip(groups, host):
                fut.result()
                for f, k in g:
                    self._open_device(slot, f, k)
            slot.opened.record(self.open_stream)
        except BaseException as e:      # handed to the frames' futures
            for x in futs:
                x.set_exception(e)
            return
        # the frames' assembly goes to the pool only once the openings are on the
        # host: its threads keep hashing the next batch's IO meanwhile
        self.waiter.submit(self._release_assembly, slot, futs)

    def _release_assembly(self, slot: _Slot, futs) -> None:
        try:
            slot.opened.synchronize()
        except BaseException as e:      # handed to the frames' futures
            for x in futs:
                x.set_exception(e)
            return
        for f, x in enumerate(futs):
            self.pool.submit(self._assemble_into, slot, f, x)

    def _assemble_into(self, slot: _Slot, f: int, fut) -> None:
        try:
            fut.set_result(self._assemble(slot, f))
        except BaseException as e:      # handed to the frame's future
            fut.set_exception(e)

    def run(self, batches):
        """Prove every batch (see the class docstring); yields each batch's list of
        FrameProof in order."""
        import sys
        # the host threads hold the interpreter lock in short stretches (numpy
        # assembly, transcript puts): a short switch interval lets the launching
        # thread take it back soon
        switch = sys.getswitchinterval()
        sys.setswitchinterval(5e-5)
        try:
            yield from self._run(batches)
        finally:
            sys.setswitchinterval(switch)

    def _run(self, batches):
        it = iter(batches)
        ahead = collections.deque()
        first = [True]

        def pull():
            batch = next(it, None)
            if batch is not None:
                # the first batch of a run hashes in pairs (its proofs wait on it);
                # the batches behind it in groups of io_group (host throughput)
                ahead.append(self._prehash(batch, 2 if first[0] else self.io_group))
                first[0] = False

        for _ in range(1 + self.io_ahead):
            pull()
        # a batch's proofs are handed out once the batches behind it fill the other
        # slots: the main thread launches the next GKR without waiting for them
        prev = None
        done = collections.deque()
        i = 0
        while ahead:
            pend = ahead.popleft()
            pull()
            slot = self.slots[i % len(self.slots)]
            i += 1
            self._start(slot, pend)
            if prev is not None:
                done.append(self._finish(prev))
                while len(done) > len(self.slots) - 1:
                    yield [x.result() for x in done.popleft()]
            prev = slot
        if prev is not None:
            done.append(self._finish(prev))
        while done:
            yield [x.result() for x in done.popleft()]
