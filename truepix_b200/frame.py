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
