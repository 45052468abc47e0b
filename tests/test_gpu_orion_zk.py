"""Zero-knowledge Orion commit on the GPU (tp_orion_commit_zk_pixels_dev,
tp_orion_commit_pair, tp_orion_pixel_vector_dev) against the roots and masks of
the reference's Orion_zk sources (tests/golden/orion_zk_golden.npz) and the
oracle (oracle/orion_oracle.c), bit for bit; at 1080p also through the
encoder's and the MLE's linearity (masked = frame + mask)."""
import ctypes
import os

import numpy as np
import pytest

from orionlib import P61, ROOT, OrionOracle, digest, frame_bytes

pytestmark = pytest.mark.gpu

W = 512


@pytest.fixture(scope="module")
def lib():
    from truepix_b200 import native
    return native.gkr()


@pytest.fixture(scope="module")
def orc():
    return OrionOracle()


@pytest.fixture(scope="module")
def zg():
    return np.load(os.path.join(ROOT, "tests", "golden", "orion_zk_golden.npz"))


def cases(zg, largest=True):
    for k in sorted(zg.files):
        if k.startswith("zkcase_"):
            name = k[len("zkcase_"):]
            copies, cs, ci, cv, padded, pseed = (int(x) for x in zg[k])
            if not largest and copies > 4096:
                continue
            yield name, (copies, cs, ci, cv, padded, pseed, int(zg["zkseed_" + name][0]))


def vp(a):
    return ctypes.c_void_p(a.ctypes.data)


def _dev():
    import torch
    return torch.device("cuda", 0)


def zk_commit(lib, pix, copies, cs, ci, cv, padded, mseed):
    """(masked tree, mask tree, masked rows, mask rows) from the device entry point"""
    import torch
    n = padded * W
    cw_len = lib.tp_orion_codeword_len(n // 128)
    leaves = lib.tp_orion_tree_leaves(n)
    d_pix = torch.from_numpy(pix).to(_dev())
    rows = [torch.empty(2 * 128 * cw_len, dtype=torch.int64, device=_dev()) for _ in range(2)]
    trees = [torch.full((64 * leaves,), 0xAB, dtype=torch.uint8, device=_dev()) for _ in range(2)]
    s = torch.cuda.current_stream().cuda_stream
    rc = lib.tp_orion_commit_zk_pixels_dev(d_pix.data_ptr(), copies, padded, cs, W, ci, cv, mseed,
                                           rows[0].data_ptr(), trees[0].data_ptr(), rows[1].data_ptr(),
                                           trees[1].data_ptr(), s)
    assert rc == 0, lib.tp_last_error()
    torch.cuda.synchronize()
    return [t.cpu().numpy().reshape(-1, 32) for t in trees] + rows


def pixel_vector(lib, d_pix, copies, cs, ci, cv, padded, mseed, mode):
    import torch
    out = torch.full((padded * W,), -1, dtype=torch.int64, device=_dev())
    s = torch.cuda.current_stream().cuda_stream
    rc = lib.tp_orion_pixel_vector_dev(d_pix.data_ptr(), copies, padded, cs, W, ci, cv, mseed, mode,
                                       out.data_ptr(), s)
    assert rc == 0, lib.tp_last_error()
    return out


def test_zk_commit_from_pixels_matches_reference(lib, zg):
    for name, (copies, cs, ci, cv, padded, pseed, mseed) in cases(zg):
        pix = frame_bytes(pseed, copies * cs)
        t_masked, t_mask, _, _ = zk_commit(lib, pix, copies, cs, ci, cv, padded, mseed)
        assert t_masked[1].tobytes() == zg["zkmasked_" + name].tobytes(), name
        assert t_mask[1].tobytes() == zg["zkmask_" + name].tobytes(), name
        assert not t_masked[0].any() and not t_mask[0].any()


def test_zk_pixel_vectors_match_oracle_and_reference_mask(lib, orc, zg):
    for name, (copies, cs, ci, cv, padded, pseed, mseed) in cases(zg, largest=False):
        import torch
        pix = frame_bytes(pseed, copies * cs)
        d_pix = torch.from_numpy(pix).to(_dev())
        for mode in (0, 1, 2):
            got = pixel_vector(lib, d_pix, copies, cs, ci, cv, padded, mseed, mode).cpu().numpy().view(np.uint64)
            want = orc.frame_vector(pix, copies, cs, W, ci, cv, padded, mseed, mode)
            assert np.array_equal(got, want), (name, mode)
            if mode == 2:
                words = np.zeros(2 * got.size, np.uint64)
                words[1::2] = got
                assert digest(words) == zg["zkmaskdigest_" + name].tobytes(), name


def test_commit_pair_from_host_buffers_equals_device_trees(lib, orc, zg):
    for name, (copies, cs, ci, cv, padded, pseed, mseed) in cases(zg, largest=False):
        pix = frame_bytes(pseed, copies * cs)
        src = []
        for mode in (1, 2):
            v = orc.frame_vector(pix, copies, cs, W, ci, cv, padded, mseed, mode)
            e = np.zeros(2 * v.size, np.uint64)
            e[1::2] = v
            src.append(e)
        n = padded * W
        leaves = lib.tp_orion_tree_leaves(n)
        ta = np.zeros((2 * leaves, 32), np.uint8)
        tb = np.zeros((2 * leaves, 32), np.uint8)
        assert lib.tp_orion_commit_pair(vp(src[0]), vp(src[1]), n, vp(ta), vp(tb)) == 0, lib.tp_last_error()
        d_masked, d_mask, _, _ = zk_commit(lib, pix, copies, cs, ci, cv, padded, mseed)
        np.testing.assert_array_equal(ta, d_masked)
        np.testing.assert_array_equal(tb, d_mask)
        assert ta[1].tobytes() == zg["zkmasked_" + name].tobytes()


def test_zk_1080p_codewords_and_mle_are_linear(lib, zg):
    """At the full frame size: the masked codeword is the frame's codeword plus
    the mask's (the encoder is linear), and MLE(masked) = MLE(frame) + MLE(mask)
    at a random point (the identity the ZK opening checks)."""
    import torch
    copies, cs, ci, cv, padded, pseed, mseed = dict(cases(zg))["zk1080"]
    pix = frame_bytes(pseed, copies * cs)
    n = padded * W
    cw_len = lib.tp_orion_codeword_len(n // 128)
    _, _, r_masked, r_mask = zk_commit(lib, pix, copies, cs, ci, cv, padded, mseed)
    d_pix = torch.from_numpy(pix).to(_dev())
    r_plain = torch.empty(2 * 128 * cw_len, dtype=torch.int64, device=_dev())
    tree = torch.empty(64 * lib.tp_orion_tree_leaves(n), dtype=torch.uint8, device=_dev())
    s = torch.cuda.current_stream().cuda_stream
    assert lib.tp_orion_commit_pixels_dev(d_pix.data_ptr(), copies, padded, cs, W, ci, cv, r_plain.data_ptr(),
                                          tree.data_ptr(), s) == 0
    torch.cuda.synchronize()
    a = r_plain.cpu().numpy().view(np.uint64)
    b = r_mask.cpu().numpy().view(np.uint64)
    c = r_masked.cpu().numpy().view(np.uint64)
    p = np.uint64(P61)
    assert int(c.max()) < P61 and int(b.max()) < P61
    assert np.array_equal(c, np.where(a + b >= p, a + b - p, a + b))
    del r_plain, r_mask, r_masked

    rng = np.random.default_rng(5)
    n_z = int(np.log2(n))
    z = rng.integers(0, P61, size=2 * n_z, dtype=np.uint64)
    dz = torch.from_numpy(z.view(np.int64)).to(_dev())
    mle = []
    for mode in (0, 1, 2):
        vec = pixel_vector(lib, d_pix, copies, cs, ci, cv, padded, mseed, mode)
        out = torch.zeros(2, dtype=torch.int64, device=_dev())
        assert lib.tp_mle_eval_base_dev(vec.data_ptr(), dz.data_ptr(), n_z, out.data_ptr(), s) == 0
        mle.append([int(x) for x in out.cpu().numpy().view(np.uint64)])
    assert mle[1] == [(mle[0][k] + mle[2][k]) % P61 for k in range(2)]
    # the frame vector is the GKR input layer's MLE input (tp_table_from_pixels)
    inputs = torch.empty(n, dtype=torch.int64, device=_dev())
    assert lib.tp_table_from_pixels(d_pix.data_ptr(), copies, padded, cs, W, ci, cv, None, inputs.data_ptr(),
                                    s) == 0, lib.tp_last_error()
    plain = pixel_vector(lib, d_pix, copies, cs, ci, cv, padded, mseed, 0)
    torch.cuda.synchronize()
    assert torch.equal(inputs, plain)


def test_zk_entry_points_reject_bad_arguments(lib):
    import torch
    buf = torch.zeros(1024, dtype=torch.int64, device=_dev())
    p = buf.data_ptr()
    assert lib.tp_orion_pixel_vector_dev(p, 1, 1, 384, W, 384, 128, 0, 3, p, None) == -1
    assert lib.tp_orion_commit_zk_pixels_dev(p, 1, 1, 384, W, 100, 128, 0, p, p, p, p, None) == -1
    assert b"layout" in lib.tp_last_error()
    assert lib.tp_orion_commit_zk_pixels_dev(p, 1, 1, 384, W, 384, 128, 0, None, p, p, p, None) == -1


def test_frame_committer_zk_pairs_on_side_streams(zg):
    """The Python committer in zk mode, frames of several layouts spread over
    side streams, against the reference's roots (and its hex form)."""
    import torch
    from truepix_b200.frame import FrameLayout
    from truepix_b200.orion import FrameCommitter
    chosen = [(n, c) for n, c in cases(zg, largest=False) if c[0] >= 2]
    layouts = [FrameLayout(copies=c[0], copy_size=c[1], const_idx=c[2], const_val=c[3]) for _, c in chosen]
    assert all(L.padded_copies == c[4] for L, (_, c) in zip(layouts, chosen))
    pix = [torch.from_numpy(frame_bytes(c[5], c[0] * c[1])).to(_dev()) for _, c in chosen]
    fc = FrameCommitter(layouts, side_streams=3, zk=True)
    for _ in range(2):    # buffers reused
        fc.commit(pix, mask_seeds=[c[6] for _, c in chosen])
        torch.cuda.synchronize()
        for f, (name, _) in enumerate(chosen):
            assert fc.root(f) == zg["zkmasked_" + name].tobytes(), name
            assert fc.mask_root(f) == zg["zkmask_" + name].tobytes(), name
            assert fc.root_hex(f).encode() == zg["zkmaskedhex_" + name].tobytes()[:64], name
    with pytest.raises(ValueError):
        fc.commit(pix)
