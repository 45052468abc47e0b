"""Orion commitment on the GPU (include/orion_gpu.h) against the reference's
roots (tests/golden/orion_golden.npz, made by the reference sources) and the
oracle (oracle/orion_oracle.c): Merkle roots, full trees, leaves and the
expander codeword, bit for bit."""
import ctypes

import numpy as np
import pytest

from orionlib import OrionOracle, digest, elements, frame_bytes, frame_elements

pytestmark = pytest.mark.gpu

KINDS = ["random", "zero", "max", "small"]


@pytest.fixture(scope="module")
def lib():
    from truepix_b200 import native
    return native.gkr()


@pytest.fixture(scope="module")
def orc():
    return OrionOracle()


@pytest.fixture(scope="module")
def og():
    import os
    from orionlib import ROOT
    return np.load(os.path.join(ROOT, "tests", "golden", "orion_golden.npz"))


def vp(a):
    return ctypes.c_void_p(a.ctypes.data)


def host_commit(lib, src, want_codeword=False):
    n = src.size // 2
    leaves = lib.tp_orion_tree_leaves(n)
    tree = np.zeros((2 * leaves, 32), np.uint8)
    cw = None
    if want_codeword:
        cw = np.zeros(2 * 128 * lib.tp_orion_codeword_len(n // 128), np.uint64)
    rc = lib.tp_orion_commit(vp(src), n, vp(tree), vp(cw) if want_codeword else None)
    assert rc == 0, lib.tp_last_error()
    return tree, cw


def test_commit_roots_match_reference(lib, og):
    for k in og.files:
        if not k.startswith("commit_"):
            continue
        name = k[len("commit_"):]
        n, seed, kind = (int(v) for v in og["commitcase_" + name])
        tree, _ = host_commit(lib, elements(seed, n, KINDS[kind]))
        assert tree[1].tobytes() == og[k].tobytes(), name
        assert not tree[0].any()


def test_commit_codeword_leaves_and_tree_match_oracle(lib, orc):
    for n in (1 << 13, 128 * 100, 128 * 13):
        src = elements(77, n)
        tree, cw = host_commit(lib, src, want_codeword=True)
        col = n // 128
        cw_len = lib.tp_orion_codeword_len(col)
        cws = cw.reshape(128, cw_len, 2)
        for c in (0, 1, 63, 127):
            want = orc.encode(np.ascontiguousarray(src.reshape(128, col, 2)[c]).reshape(-1))
            np.testing.assert_array_equal(cws[c].reshape(-1), want, err_msg="column %d" % c)
        root, leaves = orc.commit(src, leaves=True)
        size = lib.tp_orion_tree_leaves(n)
        np.testing.assert_array_equal(tree[size:size + 2 * col], leaves)
        assert tree[1].tobytes() == root


def test_commit_dev_rows_layout(lib, orc):
    import torch
    n = 1 << 14
    src = elements(5, n)
    col = n // 128
    cw_len = lib.tp_orion_codeword_len(col)
    leaves = lib.tp_orion_tree_leaves(n)
    dev = torch.device("cuda", 0)
    d_src = torch.from_numpy(src.view(np.int64)).to(dev)
    d_rows = torch.empty(2 * 128 * cw_len, dtype=torch.int64, device=dev)
    d_tree = torch.empty(64 * leaves, dtype=torch.uint8, device=dev)
    s = torch.cuda.current_stream().cuda_stream
    assert lib.tp_orion_commit_dev(d_src.data_ptr(), n, d_rows.data_ptr(), d_tree.data_ptr(), s) == 0
    d_cols = torch.empty_like(d_rows)
    assert lib.tp_orion_rows_to_columns_dev(d_rows.data_ptr(), cw_len, d_cols.data_ptr(), s) == 0
    torch.cuda.synchronize()
    rows = d_rows.cpu().numpy().view(np.uint64).reshape(cw_len, 128, 2)
    cols = d_cols.cpu().numpy().view(np.uint64).reshape(128, cw_len, 2)
    np.testing.assert_array_equal(rows.transpose(1, 0, 2), cols)
    # the message part of the codeword is the input, column c = src[c * col ...]
    np.testing.assert_array_equal(cols[:, :col, :], src.reshape(128, col, 2))
    tree, cw = host_commit(lib, src, want_codeword=True)
    np.testing.assert_array_equal(d_tree.cpu().numpy().reshape(-1, 32), tree)
    np.testing.assert_array_equal(cols.reshape(-1), cw)


def _pixel_commit(lib, pix, copies, cs, W, ci, cv, padded):
    import torch
    n = padded * W
    col = n // 128
    cw_len = lib.tp_orion_codeword_len(col)
    leaves = lib.tp_orion_tree_leaves(n)
    dev = torch.device("cuda", 0)
    d_pix = torch.from_numpy(pix).to(dev)
    d_rows = torch.empty(2 * 128 * cw_len, dtype=torch.int64, device=dev)
    d_tree = torch.empty(64 * leaves, dtype=torch.uint8, device=dev)
    s = torch.cuda.current_stream().cuda_stream
    rc = lib.tp_orion_commit_pixels_dev(d_pix.data_ptr(), copies, padded, cs, W, ci, cv,
                                        d_rows.data_ptr(), d_tree.data_ptr(), s)
    assert rc == 0, lib.tp_last_error()
    torch.cuda.synchronize()
    return d_tree.cpu().numpy().reshape(-1, 32)


@pytest.mark.parametrize("copies,cs,ci,cv,padded", [
    (100, 384, 384, 128, 128),     # gray-like, ragged copies
    (64, 384, -1, 0, 64),          # mask-like: no constant
    (30, 385, -1, 0, 32),          # crop: 385 inputs
    (3, 384, 384, 255, 4),         # inv constant, tiny
    (5, 384, 384, 1000, 8),        # constant >= 256: no byte path for depth 0
    (200, 384, 384, 128, 256),     # byte path with more targets than one CTA row
])
def test_commit_from_pixels_matches_materialised_input(lib, orc, copies, cs, ci, cv, padded):
    pix = frame_bytes(copies + cs, copies * cs)
    tree = _pixel_commit(lib, pix, copies, cs, 512, ci, cv, padded)
    src = frame_elements(pix, copies, cs, 512, ci, cv, padded)
    assert tree[1].tobytes() == orc.commit(src)
    tree2, _ = host_commit(lib, src)
    np.testing.assert_array_equal(tree, tree2)


def test_commit_of_a_1080p_frame_matches_reference(lib, og):
    copies, cs, W, ci, cv, padded, seed = (int(x) for x in og["frame1080"])
    pix = frame_bytes(seed, copies * cs)
    for _ in range(2):   # cached encoder, reused buffers
        tree = _pixel_commit(lib, pix, copies, cs, W, ci, cv, padded)
        assert tree[1].tobytes() == og["frameroot_1080"].tobytes()


def test_commit_rejects_bad_sizes_and_values(lib):
    src = elements(1, 256)
    tree = np.zeros((1024, 32), np.uint8)
    assert lib.tp_orion_commit(vp(src), 100, vp(tree), None) == -1
    assert b"multiple of 128" in lib.tp_last_error()
    bad = src.copy()
    bad[5] = (1 << 61) - 1
    assert lib.tp_orion_commit(vp(bad), 256, vp(tree), None) == -1
    assert b"canonical" in lib.tp_last_error()
    assert lib.tp_orion_commit_pixels_dev(None, 1, 1, 384, 512, 384, 128, None, None, None) == -1


def test_opening_passes_match_reference(lib, og):
    """combine / combined tree / answer over the device codeword against the
    reference (its primitives on its retained codeword), and the queried rows."""
    import torch
    dev = torch.device("cuda", 0)
    s = torch.cuda.current_stream().cuda_stream
    for k in og.files:
        if not k.startswith("combinecase_"):
            continue
        n, seed = (int(v) for v in og[k])
        col = n // 128
        cw_len = lib.tp_orion_codeword_len(col)
        leaves = lib.tp_orion_tree_leaves(n)
        d_src = torch.from_numpy(elements(seed, n).view(np.int64)).to(dev)
        d_rows = torch.empty(2 * 128 * cw_len, dtype=torch.int64, device=dev)
        d_tree = torch.empty(64 * leaves, dtype=torch.uint8, device=dev)
        assert lib.tp_orion_commit_dev(d_src.data_ptr(), n, d_rows.data_ptr(), d_tree.data_ptr(), s) == 0
        r0 = torch.from_numpy(elements(seed + 1000, 128).view(np.int64)).to(dev)
        r1 = torch.from_numpy(elements(seed + 2000, col).view(np.int64)).to(dev)
        comb = torch.empty(2 * cw_len, dtype=torch.int64, device=dev)
        ctree = torch.empty(64 * leaves, dtype=torch.uint8, device=dev)
        ans = torch.empty(2, dtype=torch.int64, device=dev)
        assert lib.tp_orion_combine_dev(d_rows.data_ptr(), n, r0.data_ptr(), comb.data_ptr(),
                                        ctree.data_ptr(), s) == 0, lib.tp_last_error()
        assert lib.tp_orion_answer_dev(comb.data_ptr(), col, r1.data_ptr(), ans.data_ptr(), s) == 0
        q = torch.tensor([0, cw_len - 1, col, 7 % cw_len], dtype=torch.int64, device=dev)
        qout = torch.empty(2 * 128 * 4, dtype=torch.int64, device=dev)
        assert lib.tp_orion_query_columns_dev(d_rows.data_ptr(), n, q.data_ptr(), 4, qout.data_ptr(), s) == 0
        torch.cuda.synchronize()
        c = comb.cpu().numpy().view(np.uint64)
        assert digest(c) == og["combine_%d" % n].tobytes(), n
        t = ctree.cpu().numpy().reshape(-1, 32)
        assert t[1].tobytes() == og["combineroot_%d" % n].tobytes(), n
        np.testing.assert_array_equal(ans.cpu().numpy().view(np.uint64), og["combineanswer_%d" % n])
        rows = d_rows.cpu().numpy().view(np.uint64).reshape(cw_len, 256)
        np.testing.assert_array_equal(qout.cpu().numpy().view(np.uint64).reshape(4, 256),
                                      rows[[0, cw_len - 1, col, 7 % cw_len]])
        bad = torch.tensor([cw_len], dtype=torch.int64, device=dev)
        assert lib.tp_orion_query_columns_dev(d_rows.data_ptr(), n, bad.data_ptr(), 1, qout.data_ptr(), s) == -1


def test_committer_waits_for_each_frames_upload(lib, orc):
    """Frames uploaded one by one on a copy stream, each commit gated on its own
    frame's event (FrameCommitter.commit(ready=...)): same roots as the oracle."""
    import torch
    from truepix_b200.frame import FrameLayout
    from truepix_b200.orion import FrameCommitter
    layouts = [FrameLayout(copies=c) for c in (100, 64, 30, 200)]
    host = [torch.from_numpy(frame_bytes(40 + f, L.copies * 384)).pin_memory() for f, L in enumerate(layouts)]
    dev = torch.device("cuda", 0)
    dpix = [torch.empty_like(h, device=dev) for h in host]
    copy = torch.cuda.Stream(dev)
    ev = [torch.cuda.Event() for _ in layouts]
    fc = FrameCommitter(layouts, side_streams=2)
    for _ in range(2):
        copy.wait_stream(torch.cuda.current_stream(dev))
        with torch.cuda.stream(copy):
            for d, h, e in zip(dpix, host, ev):
                d.copy_(h, non_blocking=True)
                e.record(copy)
        fc.commit(dpix, ready=ev)
        torch.cuda.synchronize()
        for f, L in enumerate(layouts):
            src = frame_elements(host[f].numpy(), L.copies, 384, 512, 384, 128, L.padded_copies)
            assert fc.root(f) == orc.commit(src), f


def test_leaf_chains_split_over_launches_give_the_same_tree(lib, orc):
    """tp_orion_set_leaf_chunks: the row-leaf chains run as 1, 2, 4, 8 or 16
    launches carrying the running state in the leaf slots; the trees agree
    bit for bit (and with the oracle), other values are rejected."""
    pix = frame_bytes(77, 100 * 384)
    want = None
    try:
        for n in (1, 2, 4, 8, 16):
            assert lib.tp_orion_set_leaf_chunks(n) == 0
            tree = _pixel_commit(lib, pix, 100, 384, 512, 384, 128, 128)
            if want is None:
                want = tree
                src = frame_elements(pix, 100, 384, 512, 384, 128, 128)
                assert tree[1].tobytes() == orc.commit(src)
            np.testing.assert_array_equal(tree, want)
        for bad in (0, 3, 32, -1):
            assert lib.tp_orion_set_leaf_chunks(bad) == -1
    finally:
        lib.tp_orion_set_leaf_chunks(1)


def test_commit_of_a_4k_frame_matches_oracle(lib, orc):
    """The largest serving frame: 2160 x 3840 x 3 bytes = 64,800 copies -> 65,536
    x 512 = 2^25 elements, 128 columns of 2^18, codeword 450,887 rows."""
    copies = 2160 * 3840 * 3 // 384
    pix = frame_bytes(4096, copies * 384)
    tree = _pixel_commit(lib, pix, copies, 384, 512, 384, 128, 65536)
    src = frame_elements(pix, copies, 384, 512, 384, 128, 65536)
    assert src.size == 2 << 25
    assert lib.tp_orion_codeword_len(1 << 18) == 450887
    assert tree[1].tobytes() == orc.commit(src)
