"""Device-resident GKR input layer for uint8 frames (the per-frame hot path).

A frame of H x W x 3 bytes is cut into copies of `copy_size` bytes
(TruePix's layout copy-major-384-const128-pad512-v1,
TruePix-main/Orion/Orion_nonzk/include/truepix/truepix_gkr.h:11-18): wire w < 384
of copy c is byte c*384 + w, wire `const_idx` holds the circuit constant, wires
up to 512 and padded copies are zero. For one frame the prover runs, on one
stream and without host synchronisation:

  1. tp_compute_beta_dev     -> beta over the copy challenges z2
  2. tp_early_create_pixels  -> early session over the frame's bytes
  3. nCopyBits x (claim, fold)  (TruePix-main/libTruePix/layerprover.py:144-290
     drives the same calls through the bridge); rounds 0 and 1 read the bytes,
     later rounds the folded Fp2 table in HBM
  4. tp_early_finish_dev     -> the 512 folded wire values and beta
  5. tp_mle_eval_pixels      -> MLE of the input vector at the final input point
     (TruePix-main/libTruePix/circuitnizkvec_vole.py:489-498), from the bytes

mode="table" instead materialises the 2^23-entry table and the copy-major input
vector first (tp_table_from_pixels) and runs the generic table kernels.

Challenges come from the host transcript in TruePix; here they are arguments.
"""
from __future__ import annotations

import contextlib
import ctypes
import math
from dataclasses import dataclass

import numpy as np

from . import native

P61 = (1 << 61) - 1


@dataclass
class FrameLayout:
    copies: int
    copy_size: int = 384
    n_wires: int = 512
    const_idx: int = 384
    const_val: int = 128

    @property
    def padded_copies(self) -> int:
        return 1 << max(1, math.ceil(math.log2(max(2, self.copies))))

    @property
    def n_copy_bits(self) -> int:
        return int(math.log2(self.padded_copies))

    @property
    def n_in_bits(self) -> int:
        return int(math.log2(self.n_wires))

    @staticmethod
    def for_frame(height: int, width: int, channels: int = 3, copy_size: int = 384,
                  const_idx: int = 384, const_val: int = 128) -> "FrameLayout":
        n = height * width * channels
        return FrameLayout(copies=-(-n // copy_size), copy_size=copy_size,
                           const_idx=const_idx, const_val=const_val)


def pack_fp2(re: np.ndarray, im: np.ndarray) -> np.ndarray:
    """SoA limbs -> packed {re, im} uint64 pairs (viewed as int64 for torch)."""
    return np.stack([re.astype(np.uint64), im.astype(np.uint64)], axis=1).reshape(-1).view(np.int64)


def circuit_outputs(pixels, layout: FrameLayout, gate_type, in0, in1, out=None, stream=None):
    """The prover's output vector of a frame, on the device (int64 tensor holding
    u64 values): for each real copy the circuit's gate values on the copy's
    inputs, padded per copy to 2^ceil(log2 gates), the copies padded with zeros
    to layout.padded_copies -- what circuitnizkvec_vole.py:351-355 puts into the
    transcript (FiatShamir.put(values, True)). pixels: uint8 device tensor of
    layout.copies * layout.copy_size bytes. Asynchronous on `stream`."""
    import torch
    lib = native.gkr()
    gt, i0, i1 = (np.ascontiguousarray(a, np.int32) for a in (gate_type, in0, in1))
    bits = lib.tp_circuit_out_bits(len(gt))
    n = layout.padded_copies << bits
    if pixels.dtype != torch.uint8 or not pixels.is_cuda or pixels.numel() < layout.copies * layout.copy_size:
        raise ValueError("pixels: uint8 device tensor of copies * copy_size bytes expected")
    if out is None:
        out = torch.empty(n, dtype=torch.int64, device=pixels.device)
    elif out.dtype != torch.int64 or out.numel() < n or not out.is_contiguous():
        raise ValueError("out: contiguous int64 tensor of %d elements expected" % n)
    s = stream.cuda_stream if stream is not None else torch.cuda.current_stream(pixels.device).cuda_stream
    I32P = ctypes.POINTER(ctypes.c_int)
    native.check(lib, lib.tp_circuit_outputs_pixels_dev(
        pixels.data_ptr(), layout.copies, layout.padded_copies, layout.copy_size, layout.n_wires,
        layout.const_idx, layout.const_val, len(gt), gt.ctypes.data_as(I32P), i0.ctypes.data_as(I32P),
        i1.ctypes.data_as(I32P), out.data_ptr(), s), "tp_circuit_outputs_pixels_dev")
    return out


class GkrInputLayerProver:
    """Holds device buffers for one frame size and proves frames into them."""

    def __init__(self, layout: FrameLayout, gate_type, in0, in1, device: int = 0, stream=None,
                 mode: str = "pixels"):
        import torch
        assert mode in ("pixels", "table")
        self.torch = torch
        self.lib = native.gkr()
        self.L = layout
        self.mode = mode
        self.dev = torch.device("cuda", device)
        self.gt = np.ascontiguousarray(gate_type, np.int32)
        self.i0 = np.ascontiguousarray(in0, np.int32)
        self.i1 = np.ascontiguousarray(in1, np.int32)
        C, W = layout.padded_copies, layout.n_wires
        self.stream = stream
        i64 = torch.int64
        if mode == "table":
            self.table = torch.empty(2 * W * C, dtype=i64, device=self.dev)
            self.inputs = torch.empty(W * C, dtype=i64, device=self.dev)
        self.beta = torch.empty(2 * C, dtype=i64, device=self.dev)
        self.claims = torch.zeros(8 * layout.n_copy_bits, dtype=i64, device=self.dev)
        self.wires = torch.zeros(2 * (W + 1), dtype=i64, device=self.dev)
        self.mle = torch.zeros(2, dtype=i64, device=self.dev)
        self.launches_last = 0

    def _s(self):
        return self.stream.cuda_stream if self.stream is not None else \
            self.torch.cuda.current_stream(self.dev).cuda_stream

    def prove(self, pixels, z1: np.ndarray, z2_dev, point_dev, challenges: np.ndarray,
              claim_hook=None) -> None:
        """Queue the proof of one frame. pixels: uint8 cuda tensor (copies*copy_size
        bytes); z1: uint64 [2, n_gates]; z2_dev / point_dev: packed Fp2 device
        tensors of n_copy_bits / n_in_bits + n_copy_bits entries; challenges:
        uint64 [n_copy_bits, 2]. Outputs land in self.claims / wires / mle."""
        lib, L, s = self.lib, self.L, self._s()
        C, W, nb = L.padded_copies, L.n_wires, L.n_copy_bits
        launches = 0
        if self.mode == "table":
            native.check(lib, lib.tp_table_from_pixels(pixels.data_ptr(), L.copies, C,
                                                        L.copy_size, W, L.const_idx, L.const_val,
                                                        self.table.data_ptr(),
                                                        self.inputs.data_ptr(), s), "table")
            launches += 1
        native.check(lib, lib.tp_compute_beta_dev(z2_dev.data_ptr(), nb, 1, 0,
                                                  self.beta.data_ptr(), s), "beta")
        launches += 2
        z1r = np.ascontiguousarray(z1[0], np.uint64)
        z1i = np.ascontiguousarray(z1[1], np.uint64)
        if self.mode == "table":
            h = lib.tp_early_create_dev(self.gt.size, self.gt.ctypes.data, self.i0.ctypes.data,
                                        self.i1.ctypes.data, z1r.ctypes.data, z1i.ctypes.data, C,
                                        W, self.table.data_ptr(), self.beta.data_ptr(), 1, s)
        else:
            h = lib.tp_early_create_pixels(self.gt.size, self.gt.ctypes.data, self.i0.ctypes.data,
                                           self.i1.ctypes.data, z1r.ctypes.data, z1i.ctypes.data,
                                           pixels.data_ptr(), L.copies, C, L.copy_size, W,
                                           L.const_idx, L.const_val, self.beta.data_ptr(), s)
        if not h:
            native.check(lib, -1, "early_create")
        try:
            base = self.claims.data_ptr()
            if claim_hook is None:
                ch = np.ascontiguousarray(challenges, np.uint64).reshape(-1)
                native.check(lib, lib.tp_early_rounds_dev(
                    h, nb, ch.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)), base), "rounds")
            for k in range(nb if claim_hook is not None else 0):
                claim_hook(k, "pre")
                native.check(lib, lib.tp_early_claim_dev(h, base + 64 * k), "claim")
                claim_hook(k, "post")
                native.check(lib, lib.native_fp2_early_fold(h, int(challenges[k][0]),
                                                            int(challenges[k][1])), "fold")
            wp = self.wires.data_ptr()
            native.check(lib, lib.tp_early_finish_dev(h, wp, wp + 16 * W), "finish")
            launches += lib.tp_early_launches(h)
        finally:
            lib.native_fp2_early_destroy(h)
        if self.mode == "table":
            native.check(lib, lib.tp_mle_eval_base_dev(self.inputs.data_ptr(),
                                                       point_dev.data_ptr(), L.n_in_bits + nb,
                                                       self.mle.data_ptr(), s), "mle")
        else:
            native.check(lib, lib.tp_mle_eval_pixels(pixels.data_ptr(), L.copies, C, L.copy_size,
                                                     W, L.const_idx, L.const_val,
                                                     point_dev.data_ptr(), self.mle.data_ptr(),
                                                     s), "mle")
        launches += 2
        self.launches_last = launches

    def results(self):
        """(claims uint64 [nb, 8], wires uint64 [W, 2], beta (re, im), mle (re, im))."""
        W = self.L.n_wires
        c = self.claims.cpu().numpy().view(np.uint64).reshape(-1, 8)
        w = self.wires.cpu().numpy().view(np.uint64).reshape(W + 1, 2)
        m = self.mle.cpu().numpy().view(np.uint64)
        return c, w[:W], (int(w[W, 0]), int(w[W, 1])), (int(m[0]), int(m[1]))


class BatchFrameProver:
    """Many frames (sizes may differ) proven together: one kernel launch per
    sumcheck round serves every frame that still has early rounds left
    (tp_batch_*); beta tables and input MLEs are computed in one launch per
    group of frames with the same padded size. The batch object and its device
    buffers persist across prove() calls."""

    def __init__(self, layouts, gate_type, in0, in1, device: int = 0, stream=None):
        import torch
        self.torch = torch
        self.lib = native.gkr()
        self.layouts = list(layouts)
        self.B = len(self.layouts)
        self.dev = torch.device("cuda", device)
        self.stream = stream
        self.gt = np.ascontiguousarray(gate_type, np.int32)
        self.i0 = np.ascontiguousarray(in0, np.int32)
        self.i1 = np.ascontiguousarray(in1, np.int32)
        W = self.layouts[0].n_wires
        L0 = self.layouts[0]
        assert all((L.n_wires, L.copy_size, L.const_idx, L.const_val) ==
                   (W, L0.copy_size, L0.const_idx, L0.const_val) for L in self.layouts), \
            "one circuit layout per batch (copy counts may differ)"
        self.W = W
        self.max_rounds = max(L.n_copy_bits for L in self.layouts)
        i64 = torch.int64
        # frames grouped by padded size: one beta / MLE launch per group
        self.groups = {}
        for f, L in enumerate(self.layouts):
            self.groups.setdefault(L.padded_copies, []).append(f)
        self.betas = {C: torch.empty(len(fs) * 2 * C, dtype=i64, device=self.dev)
                      for C, fs in self.groups.items()}
        self.claims = torch.zeros(self.max_rounds * self.B * 8, dtype=i64, device=self.dev)
        self.wires = torch.zeros(self.B * W * 2, dtype=i64, device=self.dev)
        self.fin_beta = torch.zeros(self.B * 2, dtype=i64, device=self.dev)
        self.mle = torch.zeros(self.B * 2, dtype=i64, device=self.dev)
        self.launches_last = 0
        self.handle = self.lib.tp_batch_create(self.B, self._s())
        if not self.handle:
            native.check(self.lib, -1, "batch_create")

    def __del__(self):
        try:
            if self.handle:
                self.lib.tp_batch_destroy(self.handle)
                self.handle = None
        except Exception:
            pass

    def _s(self):
        return self.stream.cuda_stream if self.stream is not None else \
            self.torch.cuda.current_stream(self.dev).cuda_stream

    def prove(self, pixels, z1s, z2s_dev, points_dev, challenges: np.ndarray,
              round_hook=None, transcripts=None, layer: int = 0, vole=None, graph: bool = False) -> None:
        """pixels: one uint8 device tensor per frame; z1s: uint64 [2, n_gates] per
        frame; z2s_dev / points_dev: per padded size C, a packed Fp2 device tensor
        [frames of size C][log2 C] / [..][log2 W + log2 C], frames in batch order
        (dicts keyed by C; a single tensor is accepted when all frames share C);
        challenges: uint64 [max_rounds, B, 2]. round_hook(k) runs after round k's
        claims are queued (where a prover reads them back for its transcript).
        transcripts: instead of `challenges`, one Fiat-Shamir state per frame in
        device memory (uint8 tensor [B * tp_fs_state_bytes()]): every round, each
        frame's transcript puts its four claims and draws the fold challenge
        rand_ext("sc-<layer>-<round>") on the device (tp_fs_*_dev, tp_batch_fold_dev),
        with no host round trip; launch by launch all frames must then have the
        same number of rounds (the graph path below takes uneven batches: a frame
        leaves after its own last round). The drawn challenges are left in
        self.device_challenges [round][frame].
        vole: with transcripts, run each round as the reference's VOLE-committed
        round (tp_vole_round_dev): a dict of `states` (uint8 [B * 160], device),
        `u`, `v` (int64 [B * count * 2], device: each frame's correlations) and
        `count`; the round's proof elements (four commitments and the equality
        value per frame) are left in self.device_proof [rounds][B][5] Fp2.
        graph: with transcripts and vole on a stream of the caller's, every round
        and the finish run as one CUDA graph (tp_batch_vole_rounds_graph), captured
        on the first call and replayed after."""
        lib, s, b = self.lib, self._s(), self.handle
        if not isinstance(z2s_dev, dict):
            assert len(self.groups) == 1
            C = next(iter(self.groups))
            z2s_dev, points_dev = {C: z2s_dev}, {C: points_dev}
        self._z2s_dev = z2s_dev      # the layer's closing proofs read the copy part of the point
        launches = 0
        beta_of = {}
        for C, fs in self.groups.items():
            nb = int(math.log2(C))
            native.check(lib, lib.tp_compute_beta_batch_dev(z2s_dev[C].data_ptr(), nb, len(fs),
                                                            self.betas[C].data_ptr(), s), "beta")
            launches += 2
            for q, f in enumerate(fs):
                beta_of[f] = self.betas[C].data_ptr() + 16 * C * q
        lib.tp_batch_reset(b)
        keep = []
        quick = native.gkr_launcher()     # per-frame setup calls keep the interpreter lock
        for f, L in enumerate(self.layouts):
            z1r = np.ascontiguousarray(z1s[f][0], np.uint64)
            z1i = np.ascontiguousarray(z1s[f][1], np.uint64)
            keep += [z1r, z1i]
            native.check(lib, quick.tp_batch_set_pixels(
                b, f, self.gt.size, self.gt.ctypes.data, self.i0.ctypes.data, self.i1.ctypes.data,
                z1r.ctypes.data, z1i.ctypes.data, pixels[f].data_ptr(), L.copies, L.padded_copies,
                L.copy_size, L.n_wires, L.const_idx, L.const_val, beta_of[f]), "batch_set_pixels")
        base = self.claims.data_ptr()
        use_graph = graph and transcripts is not None and vole is not None and self.stream is not None
        if transcripts is not None:
            if not use_graph and any(L.n_copy_bits != self.max_rounds for L in self.layouts):
                raise ValueError("device transcripts launch by launch need frames with the same number of rounds "
                                 "(the graph path takes uneven batches)")
            if transcripts.numel() != self.B * lib.tp_fs_state_bytes():
                raise ValueError("one transcript state per frame")
            if getattr(self, "device_challenges", None) is None:
                self.device_challenges = self.torch.zeros(self.max_rounds * self.B * 2, dtype=self.torch.int64,
                                                          device=self.dev)
            if vole is not None and getattr(self, "device_proof", None) is None:
                self.device_proof = self.torch.zeros(self.max_rounds * self.B * 10, dtype=self.torch.int64,
                                                     device=self.dev)
        else:
            ch = np.ascontiguousarray(challenges, np.uint64)
        l0 = lib.tp_batch_launches(b)
        if use_graph:
            native.check(lib, lib.tp_batch_vole_rounds_graph(
                b, base, transcripts.data_ptr(), vole["states"].data_ptr(), vole["u"].data_ptr(),
                vole["v"].data_ptr(), vole["count"], layer, self.device_challenges.data_ptr(),
                self.device_proof.data_ptr(), self.wires.data_ptr(), self.fin_beta.data_ptr()),
                "tp_batch_vole_rounds_graph")
        for k in range(0 if use_graph else self.max_rounds):
            native.check(lib, lib.tp_batch_claim(b, base + 64 * self.B * k), "batch_claim")
            if round_hook is not None:
                round_hook(k)
            if transcripts is not None:
                d_ch = self.device_challenges.data_ptr() + 16 * self.B * k
                label = ("sc-%d-%d" % (layer, k)).encode()
                if vole is not None:
                    native.check(lib, lib.tp_vole_round_dev(
                        transcripts.data_ptr(), vole["states"].data_ptr(), self.B, base + 64 * self.B * k,
                        vole["u"].data_ptr(), vole["v"].data_ptr(), vole["count"], label, d_ch,
                        self.device_proof.data_ptr() + 80 * self.B * k, s), "vole round")
                else:
                    native.check(lib, lib.tp_fs_put_fp2s_dev(transcripts.data_ptr(), self.B,
                                                             base + 64 * self.B * k, 4, s), "transcript put")
                    native.check(lib, lib.tp_fs_rand_ext_dev(transcripts.data_ptr(), self.B, label, d_ch, s),
                                 "rand_ext")
                native.check(lib, lib.tp_batch_fold_dev(b, d_ch), "batch_fold_dev")
                launches += 2
                continue
            native.check(lib, lib.tp_batch_fold(
                b, ch[k].reshape(-1).ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))), "batch_fold")
        if not use_graph:
            native.check(lib, lib.tp_batch_finish(b, self.wires.data_ptr(), self.fin_beta.data_ptr()),
                         "batch_finish")
        launches += lib.tp_batch_launches(b) - l0
        L0 = self.layouts[0]
        for C, fs in self.groups.items():
            ptrs = (ctypes.c_void_p * len(fs))(*[pixels[f].data_ptr() for f in fs])
            ncop = (ctypes.c_int * len(fs))(*[self.layouts[f].copies for f in fs])
            out = self.torch.empty(2 * len(fs), dtype=self.torch.int64, device=self.dev)
            native.check(lib, lib.tp_mle_eval_pixels_batch(
                len(fs), ptrs, ncop, C, L0.copy_size, L0.n_wires, L0.const_idx, L0.const_val,
                points_dev[C].data_ptr(), out.data_ptr(), s), "mle")
            launches += 2
            if len(self.groups) == 1:
                self.mle.copy_(out)
            else:
                for q, f in enumerate(fs):
                    self.mle[2 * f:2 * f + 2].copy_(out[2 * q:2 * q + 2])
        self.launches_last = launches

    def prove_late(self, z1s, challenges=None, transcripts=None, vole=None, layer: int = 0, zk: bool = False) -> None:
        """The late rounds and the line projection of every frame, after prove():
        one launch (tp_late_rounds_dev) from the batch's wires and beta. z1s: the
        per-gate weights given to prove() (uint64 [2, n_gates] per frame).
        challenges: uint64 [B, 2 log2 W, 2]; or, instead, transcripts and vole as
        in prove() (the states continue from the early rounds; round labels
        continue at the frame's copy-bit count). Results in self.late_coefs
        [B][2 log2 W][3], self.line [B][log2 W + 1], self.late_challenges
        [B][2 log2 W] and, with vole, self.late_proof [B][2 log2 W][4] and the
        layer's closing proofs: self.closing [B][log2 W + 10] (the values put, in
        order; log2 W + 15 with zk, the zero-knowledge prover's product proof),
        self.input_point [B][log2 W + copy bits] and self.input_tag [B] (packed
        Fp2, int64 device tensors)."""
        torch, lib, s = self.torch, self.lib, self._s()
        n = int(math.log2(self.W))
        G = self.gt.size
        zg = np.stack([np.stack([np.asarray(z[0], np.uint64), np.asarray(z[1], np.uint64)], axis=1)
                       for z in z1s]).reshape(-1)
        # uploads on the launch stream, so that the kernel is ordered after them
        def on_stream():
            return torch.cuda.stream(self.stream) if self.stream is not None else contextlib.nullcontext()
        with on_stream():    # from pinned memory, asynchronously: no wait for the launch stream to drain
            d_zg = torch.from_numpy(zg.view(np.int64)).pin_memory().to(self.dev, non_blocking=True)
        i64 = torch.int64
        with on_stream():
            self.late_coefs = torch.zeros(self.B * 2 * n * 3 * 2, dtype=i64, device=self.dev)
            self.line = torch.zeros(self.B * (n + 1) * 2, dtype=i64, device=self.dev)
            self.late_challenges = torch.zeros(self.B * 2 * n * 2, dtype=i64, device=self.dev)
        I32P = ctypes.POINTER(ctypes.c_int)
        gt, i0, i1 = (a.ctypes.data_as(I32P) for a in (self.gt, self.i0, self.i1))
        keep = [d_zg]
        if transcripts is None:
            ch = np.ascontiguousarray(challenges, np.uint64).reshape(-1)
            if ch.size != self.B * 2 * n * 2:
                raise ValueError("challenges: [B, 2 log2 W, 2] expected")
            with on_stream():
                d_ch = torch.from_numpy(ch.view(np.int64).copy()).to(self.dev)
            keep.append(d_ch)
            self.late_proof = None
            rc = lib.tp_late_rounds_dev(self.B, n, G, gt, i0, i1, self.wires.data_ptr(), self.fin_beta.data_ptr(),
                                        d_zg.data_ptr(), 1, d_ch.data_ptr(), None, None, None, None, 0, layer, 0,
                                        self.late_coefs.data_ptr(), self.line.data_ptr(),
                                        self.late_challenges.data_ptr(), None, None, None, 0, 0, None, None, None, 0,
                                        s)
        else:
            if vole is None:
                raise ValueError("the late rounds on device transcripts are the VOLE-committed rounds: pass vole")
            if any(L.n_copy_bits != self.max_rounds for L in self.layouts):
                raise ValueError("device transcripts need frames with the same number of rounds")
            nb = self.max_rounds
            with on_stream():
                self.late_proof = torch.zeros(self.B * 2 * n * 4 * 2, dtype=i64, device=self.dev)
                self.closing = torch.zeros(self.B * (n + (15 if zk else 10)) * 2, dtype=i64, device=self.dev)
                self.input_point = torch.zeros(self.B * (n + nb) * 2, dtype=i64, device=self.dev)
                self.input_tag = torch.zeros(self.B * 2, dtype=i64, device=self.dev)
            z2 = next(iter(self._z2s_dev.values()))
            # early challenges: self.device_challenges [round][frame]
            rc = lib.tp_late_rounds_dev(self.B, n, G, gt, i0, i1, self.wires.data_ptr(), self.fin_beta.data_ptr(),
                                        d_zg.data_ptr(), 1, None, transcripts.data_ptr(), vole["states"].data_ptr(),
                                        vole["u"].data_ptr(), vole["v"].data_ptr(), vole["count"], layer, nb,
                                        self.late_coefs.data_ptr(), self.line.data_ptr(),
                                        self.late_challenges.data_ptr(), self.late_proof.data_ptr(), z2.data_ptr(),
                                        self.device_challenges.data_ptr(), 1, self.B, self.closing.data_ptr(),
                                        self.input_point.data_ptr(), self.input_tag.data_ptr(), int(zk), s)
        native.check(lib, rc, "tp_late_rounds_dev")
        self._late_keep = keep     # inputs stay alive until the stream has used them

    def results(self, f: int):
        """Frame f: (claims [n_copy_bits, 8], wires [W, 2], beta, mle)."""
        nb = self.layouts[f].n_copy_bits
        c = self.claims.cpu().numpy().view(np.uint64).reshape(self.max_rounds, self.B, 8)[:nb, f]
        w = self.wires.cpu().numpy().view(np.uint64).reshape(self.B, self.W, 2)[f]
        b = self.fin_beta.cpu().numpy().view(np.uint64).reshape(self.B, 2)[f]
        m = self.mle.cpu().numpy().view(np.uint64).reshape(self.B, 2)[f]
        return c, w, (int(b[0]), int(b[1])), (int(m[0]), int(m[1]))


# ---- the round launches' autotuner (tp_batch_autotune) ----------------------------

def autotune_rounds(on: bool = True) -> None:
    """Measure the claim / fold launch split of each (round kind, work bucket) the
    next immediate batched rounds meet, and keep the fastest for this device."""
    lib = native.gkr()
    native.check(lib, lib.tp_batch_autotune(1 if on else 0), "tp_batch_autotune")


def round_tuning() -> list:
    """The measured splits on this device: [(kind, bucket, CTAs per SM)]"""
    lib = native.gkr()
    n = lib.tp_batch_tune_table(None, None, None, 0)
    native.check(lib, 0 if n >= 0 else -1, "tp_batch_tune_table")
    k, b, m = (np.zeros(max(1, n), np.int32) for _ in range(3))
    n = lib.tp_batch_tune_table(k.ctypes.data, b.ctypes.data, m.ctypes.data, n)
    return [(int(k[i]), int(b[i]), int(m[i])) for i in range(n)]


def save_round_tuning(path: str) -> None:
    """round_tuning() to a JSON file, keyed by the device's name"""
    import json
    import torch
    with open(path, "w") as fh:
        json.dump({"device": torch.cuda.get_device_name(), "entries": round_tuning()}, fh)


def load_round_tuning(path: str) -> int:
    """install the splits a JSON file of save_round_tuning holds for this device's
    name; returns how many"""
    import json
    import torch
    lib = native.gkr()
    with open(path) as fh:
        d = json.load(fh)
    if d.get("device") != torch.cuda.get_device_name():
        return 0
    for kind, bucket, mult in d.get("entries", []):
        native.check(lib, lib.tp_batch_tune_set(int(kind), int(bucket), int(mult)), "tp_batch_tune_set")
    return len(d.get("entries", []))
