"""The Orion opening proof of a committed frame (NIZK mode; the plain commit's
and, for TruePix's default zero-knowledge commit pair, the masked polynomial's
and the mask's), as the reference's linearPC_multi_prove writes it
(TruePix-main/Orion/Orion_nonzk and Orion_zk:
examples/multivariate_PC_test_prove.cpp:127-190, src/VPD/linearPC.cpp:426-640
tensor_product_protocol, src/truepix/orion_proof.cpp:67-95 file format), with the
passes over the codeword on the device.

  host    the GKR input point reversed (truepix_gkr.h:233-239) and split into the
          column weights r0 (its top 7 coordinates) and the row weights r1 (the
          rest) as eq tables (linearPC.cpp:693-731 dfs); the Orion transcript
          (src/truepix/orion_fs.cpp, tp_orion_open_queries) absorbs
          "tensor-open", the commitment's root, N, use_group1, r0 and r1 and
          draws the 1222 queried columns
  device  combined codeword and its Merkle tree (tp_orion_combine_dev), the
          answer sum r1[i] * combined[i] (tp_orion_answer_dev), the queried
          columns (tp_orion_query_columns_dev), all over the codeword the commit
          left in HBM (truepix_b200.orion.FrameCommitter)
  host    the Merkle siblings of the queried leaves in both trees
          (orion_proof.cpp:153-174) and the proof file's bytes.

The reference also runs an in-process self-check of the combined codeword
(its EC(y1) GKR, linearPC.cpp:585-620) whose results do not enter the file; the
verifier repeats it on its side.
"""
from __future__ import annotations

import ctypes
import math
import struct

import numpy as np

from . import native

COLUMN_SIZE = 128
TARGET_DISTANCE = 0.07          # linear_code/parameter.h:4
P61 = (1 << 61) - 1


def query_count() -> int:
    """linearPC.cpp:440: -128 / log2(1 - target_distance), truncated"""
    return int(-128 / math.log2(1 - TARGET_DISTANCE))


def split_point(point):
    """The eq-table coordinates of the column weights r0 and the row weights r1
    (LSB first): open_and_verify reverses the GKR point and builds both tables
    MSB-first over the reversed halves, which is the LSB-first table over the
    point's own top 7 coordinates (r0) and its other ones (r1)."""
    lg = len(point)
    return list(point[lg - 7:]), list(point[:lg - 7])


def eq_table(lib, coords) -> np.ndarray:
    """eq(coords, i) for i < 2^len, LSB first, as (real, imag) uint64 [2^k, 2]
    (native_fp2_compute_beta, on the device)"""
    import ctypes
    k = len(coords)
    zr = np.ascontiguousarray([int(c[0]) for c in coords], np.uint64)
    zi = np.ascontiguousarray([int(c[1]) for c in coords], np.uint64)
    out_r = np.zeros(1 << k, np.uint64)
    out_i = np.zeros(1 << k, np.uint64)
    P = ctypes.POINTER(ctypes.c_uint64)
    lib.native_fp2_compute_beta(zr.ctypes.data_as(P), zi.ctypes.data_as(P), k, 1, 0, out_r.ctypes.data_as(P),
                                out_i.ctypes.data_as(P))
    native.check(lib, None, "native_fp2_compute_beta")
    return np.stack([out_r, out_i], axis=1)


def merkle_siblings(tree: np.ndarray, n_leaves: int, positions) -> tuple:
    """collect_merkle_siblings (orion_proof.cpp:153-174): for each position in
    order, the siblings on its path not taken before (heap order, root at 1)"""
    seen = set()
    idxs, digs = [], []
    for p in positions:
        node = int(p) + n_leaves
        while node != 1:
            sib = node ^ 1
            if sib not in seen:
                seen.add(sib)
                idxs.append(sib)
                digs.append(tree[sib].tobytes())
            node //= 2
    return idxs, digs


def _bytearray_uninitialised(size: int) -> bytearray:
    """a bytearray of `size` bytes left as allocated: bytearray(size) zero-fills
    (about 0.7 ms for a 1080p opening file) while holding the interpreter lock"""
    f = ctypes.pythonapi.PyByteArray_FromStringAndSize
    f.restype, f.argtypes = ctypes.py_object, [ctypes.c_void_p, ctypes.c_ssize_t]
    return f(None, size)


def opening_bytes(N, msg_len, cw_len, answer, com_root, comb_root, col_q, cols, combined, com_sparse, comb_sparse,
                  use_group1: int = 1) -> bytearray:
    """OpeningProof::write_file (orion_proof.cpp:67-95); elements as (img, real)
    uint64 pairs; com_sparse / comb_sparse: (node indices, their 32-byte digests as
    a list of bytes or an [n, 32] uint8 array). The bytes are written by the
    library (tp_orion_opening_file) into a bytearray."""
    lib = native.gkr(require_device=False)
    arr = lambda a, t: np.ascontiguousarray(a, t)

    def sparse(sp):
        idxs, digs = sp
        d = np.frombuffer(b"".join(digs), np.uint8) if isinstance(digs, list) else np.asarray(digs, np.uint8)
        return arr(idxs, np.int32), arr(d.reshape(-1), np.uint8)
    ans, q = arr(answer, np.uint64), arr(col_q, np.int64)
    cl, cb = arr(cols, np.uint64), arr(combined, np.uint64)
    (ci, cd), (bi, bd) = sparse(com_sparse), sparse(comb_sparse)
    size = lib.tp_orion_opening_file_size(msg_len, cw_len, q.size, ci.size, bi.size)
    out = _bytearray_uninitialised(size)     # every byte is written below
    buf = (ctypes.c_char * size).from_buffer(out)
    got = lib.tp_orion_opening_file(N, msg_len, cw_len, ans.ctypes.data, bytes(com_root), bytes(comb_root),
                                    q.ctypes.data, q.size, cl.ctypes.data, cb.ctypes.data, ci.ctypes.data,
                                    cd.ctypes.data, ci.size, bi.ctypes.data, bd.ctypes.data, bi.size, use_group1,
                                    ctypes.addressof(buf), size)
    native.check(lib, 0 if got == size else -1, "tp_orion_opening_file")
    return out


def query_columns(lib, root: bytes, N: int, use_group1: int, r0: np.ndarray, r1: np.ndarray, cw_len: int,
                  group: int):
    """the queried columns drawn by the opening's transcript (tp_orion_open_queries):
    any of the cw_len (group -1, the plain opening), or the even (0: the masked
    polynomial) or odd (1: the mask) columns of the zero-knowledge opening
    (Orion_zk linearPC.cpp:739-756)"""
    out = np.zeros(query_count(), np.int64)
    r0 = np.ascontiguousarray(r0, np.uint64)
    r1 = np.ascontiguousarray(r1, np.uint64)
    native.check(lib, lib.tp_orion_open_queries(root, N, use_group1, r0.ctypes.data, len(r0), r1.ctypes.data,
                                                len(r1), cw_len, group, out.size, out.ctypes.data),
                 "tp_orion_open_queries")
    return out.tolist()


def opening_proof(committer, f: int, point, polynomial: str = None, stream=None) -> bytes:
    """The NIZK opening proof of frame f of a truepix_b200.orion.FrameCommitter
    whose commit has completed, at the GKR input point (the prover's order:
    (real, imag) pairs or Fp2 values). For a zero-knowledge commit pair,
    polynomial is "masked" (orion_proof_masked.bin) or "mask"
    (orion_proof_mask.bin): TruePix's default (Orion_zk
    examples/multivariate_PC_test_prove.cpp:252-300, linearPC.cpp:701-930); for
    a plain commit it is None (orion_proof.bin)."""
    import torch
    lib = native.gkr()
    if committer.zk != (polynomial is not None) or polynomial not in (None, "masked", "mask"):
        raise ValueError("polynomial: 'masked' or 'mask' for a zero-knowledge commit pair, None otherwise")
    group = -1 if polynomial is None else (0 if polynomial == "masked" else 1)
    L = committer.layouts[f]
    N = L.padded_copies * L.n_wires
    msg_len, cw_len, leaves = N // COLUMN_SIZE, committer.cw_len[f], committer.leaves[f]
    pt = [(int(x.real), int(x.imag)) if hasattr(x, "real") else (int(x[0]), int(x[1])) for x in point]
    if len(pt) != N.bit_length() - 1:
        raise ValueError("the point has %d coordinates, the frame %d" % (len(pt), N.bit_length() - 1))
    c0, c1 = split_point(pt)
    r0, r1 = eq_table(lib, c0), eq_table(lib, c1)
    mask = polynomial == "mask"
    com_root = committer.mask_root(f) if mask else committer.root(f)
    col_q = query_columns(lib, com_root, N, 0 if mask else 1, r0, r1, cw_len, group)
    qc = len(col_q)
    dev = committer.dev
    s = stream.cuda_stream if stream is not None else torch.cuda.current_stream(dev).cuda_stream
    as_dev = lambda a: torch.from_numpy(np.ascontiguousarray(a[:, ::-1]).view(np.int64).reshape(-1).copy()).to(dev)
    d_r0, d_r1 = as_dev(r0), as_dev(r1)          # (img, real), the codeword's element order
    comb = torch.empty(2 * cw_len, dtype=torch.int64, device=dev)
    ctree = torch.empty(64 * leaves, dtype=torch.uint8, device=dev)
    ans = torch.empty(2, dtype=torch.int64, device=dev)
    q = torch.tensor(col_q, dtype=torch.int64, device=dev)
    cols = torch.empty(2 * COLUMN_SIZE * qc, dtype=torch.int64, device=dev)
    rows = (committer.mask_rows[f] if mask else committer.rows[f]).data_ptr()
    native.check(lib, lib.tp_orion_combine_dev(rows, N, d_r0.data_ptr(), comb.data_ptr(), ctree.data_ptr(), s),
                 "tp_orion_combine_dev")
    native.check(lib, lib.tp_orion_answer_dev(comb.data_ptr(), msg_len, d_r1.data_ptr(), ans.data_ptr(), s),
                 "tp_orion_answer_dev")
    native.check(lib, lib.tp_orion_query_columns_dev(rows, N, q.data_ptr(), qc, cols.data_ptr(), s),
                 "tp_orion_query_columns_dev")
    if stream is not None:
        stream.synchronize()
    torch.cuda.synchronize(dev)
    combined = comb.cpu().numpy().view(np.uint64).reshape(cw_len, 2)
    tree = (committer.mask_trees[f] if mask else committer.trees[f]).cpu().numpy().reshape(-1, 32)
    ct = ctree.cpu().numpy().reshape(-1, 32)
    return opening_bytes(N, msg_len, cw_len, ans.cpu().numpy().view(np.uint64), com_root, ct[1].tobytes(), col_q,
                         cols.cpu().numpy().view(np.uint64), combined, merkle_siblings(tree, leaves, col_q),
                         merkle_siblings(ct, leaves, col_q), use_group1=0 if mask else 1)
