"""Orion input-layer commitment of frames on the device (include/orion_gpu.h).

The reference commits a frame in its `linearPC_multi_commit` process
(TruePix-main/Orion/Orion_nonzk/examples/multivariate_PC_test_commit.cpp:120-155):
load the 2^(9 + nCopyBits) input vector in TruePix's layout
(include/truepix/truepix_gkr.h:107-206), expander_init, commit() -> Merkle tree,
root printed by root_hex. Here each frame is committed straight from its uint8
bytes on the GPU; the codeword (kept for the opening, as the reference's
set_retain_encoded_codeword(true) keeps it) and the tree stay in HBM.

The zero-knowledge commit (TruePix-main/Orion/Orion_zk,
examples/multivariate_PC_test_commit.cpp:280-340, TruePix's default) commits the
masked polynomial (frame + mask) and the mask, the mask drawn from a per-frame
seed (include/truepix/truepix_gkr.h:286-384): two codewords and two trees.
"""
from __future__ import annotations

import numpy as np

from . import native


class FrameCommitter:
    """Commits frames of the given layouts (truepix_b200.frame.FrameLayout) from
    their device bytes. One codeword (cw_len x 128 elements, row-major) and one
    tree (2 * leaves digests) per frame, allocated once and reused."""

    def __init__(self, layouts, device: int = 0, stream=None, side_streams: int = 0, zk: bool = False):
        """side_streams > 0: frames are committed round-robin on that many extra
        streams (joined back into `stream` at the end of commit()), so that one
        frame's latency-bound phases (the tree levels, the small expander graphs)
        overlap another frame's SHA-256 leaves. zk: commit pairs (masked, mask);
        rows / trees then hold the masked polynomial's, mask_rows / mask_trees
        the mask's."""
        import torch
        self.torch = torch
        self.lib = native.gkr()
        self.layouts = list(layouts)
        self.dev = torch.device("cuda", device)
        self.stream = stream
        self.zk = zk
        self.rows, self.trees, self.cw_len, self.leaves = [], [], [], []
        self.mask_rows, self.mask_trees = [], []
        for L in self.layouts:
            n = L.padded_copies * L.n_wires
            cw = self.lib.tp_orion_codeword_len(n // 128)
            lv = self.lib.tp_orion_tree_leaves(n)
            self.cw_len.append(cw)
            self.leaves.append(lv)
            self.rows.append(torch.empty(2 * 128 * cw, dtype=torch.int64, device=self.dev))
            self.trees.append(torch.empty(64 * lv, dtype=torch.uint8, device=self.dev))
            if zk:
                self.mask_rows.append(torch.empty(2 * 128 * cw, dtype=torch.int64, device=self.dev))
                self.mask_trees.append(torch.empty(64 * lv, dtype=torch.uint8, device=self.dev))
        self.side = [torch.cuda.Stream(self.dev) for _ in range(side_streams)]
        self.launches_last = 0

    def _s(self):
        return self.stream.cuda_stream if self.stream is not None else \
            self.torch.cuda.current_stream(self.dev).cuda_stream

    def commit(self, pixels, join: bool = True, mask_seeds=None, ready=None, after=None) -> None:
        """Queue the commits of all frames (pixels: one uint8 device tensor each).
        With side streams and join=False the step's stream does not wait for them
        here (work queued on it next overlaps the commits); call join() later.
        mask_seeds: one 64-bit seed per frame, required (only) for zk.
        ready: optional CUDA events, one per frame, recorded when that frame's
        bytes are in place (e.g. after its host-to-device copy on a copy stream):
        each frame's commit waits for its own event only.
        after: optional callable after(f), called with frame f's commit stream
        current right after that commit is queued (work it queues follows the
        frame's commit, not the stream's later frames)."""
        if self.zk != (mask_seeds is not None):
            raise ValueError("mask_seeds are given exactly for a zk committer")
        torch, lib, s = self.torch, native.gkr_launcher(), self._s()
        launches = 0
        main = self.stream if self.stream is not None else torch.cuda.current_stream(self.dev)
        if self.side:
            start = torch.cuda.Event()
            start.record(main)
            for q in self.side:
                q.wait_event(start)
        for f, L in enumerate(self.layouts):
            fs = self.side[f % len(self.side)].cuda_stream if self.side else s
            if ready is not None:
                (self.side[f % len(self.side)] if self.side else main).wait_event(ready[f])
            if self.zk:
                native.check(lib, lib.tp_orion_commit_zk_pixels_dev(
                    pixels[f].data_ptr(), L.copies, L.padded_copies, L.copy_size, L.n_wires,
                    L.const_idx, L.const_val, int(mask_seeds[f]) & ((1 << 64) - 1), self.rows[f].data_ptr(),
                    self.trees[f].data_ptr(), self.mask_rows[f].data_ptr(), self.mask_trees[f].data_ptr(), fs),
                    "orion zk commit")
            else:
                native.check(lib, lib.tp_orion_commit_pixels_dev(
                    pixels[f].data_ptr(), L.copies, L.padded_copies, L.copy_size, L.n_wires,
                    L.const_idx, L.const_val, self.rows[f].data_ptr(), self.trees[f].data_ptr(), fs),
                    "orion commit")
            launches += lib.tp_orion_last_launches()
            if after is not None:
                with torch.cuda.stream(self.side[f % len(self.side)] if self.side else main):
                    after(f)
        self._pending = []
        for q in self.side:
            done = torch.cuda.Event()
            done.record(q)
            self._pending.append(done)
        if join:
            self.join()
        self.launches_last = launches

    def join(self) -> None:
        """Make the step's stream wait for the commits queued by commit(join=False)."""
        main = self.stream if self.stream is not None else self.torch.cuda.current_stream(self.dev)
        for done in getattr(self, "_pending", []):
            main.wait_event(done)
        self._pending = []

    def root(self, f: int) -> bytes:
        """the commit's root (zk: the masked polynomial's)"""
        return self.trees[f][32:64].cpu().numpy().tobytes()

    def mask_root(self, f: int) -> bytes:
        return self.mask_trees[f][32:64].cpu().numpy().tobytes()

    @staticmethod
    def hex(root: bytes) -> str:
        """truepix::root_hex: the digest's little-endian u64 words as hi(h0) lo(h0) hi(h1) lo(h1)."""
        w = np.frombuffer(root, np.uint64)
        return "%016x%016x%016x%016x" % (w[1], w[0], w[3], w[2])

    def root_hex(self, f: int) -> str:
        return self.hex(self.root(f))
