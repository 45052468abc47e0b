"""The batched early rounds on device transcripts as one CUDA graph
(tp_batch_vole_rounds_graph) against the same rounds launch by launch: the same
claims, challenges, VOLE proof elements, wires, beta, transcripts and VOLE
states, on the first call (capture) and on replays with other frames; an uneven
batch (frames of different sizes in one graph) against each frame alone; and
the round autotuner: measured splits change no value."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _setup(n_frames, copies, seed):
    import torch
    from truepix_b200 import native
    from truepix_b200.frame import BatchFrameProver, FrameLayout, pack_fp2
    from proverlib import circuit
    from truepix_b200.pipeline import correlations_needed
    lib = native.gkr()
    gt, i0, i1 = circuit("gray")
    layout = FrameLayout(copies=copies)
    rng = np.random.default_rng(seed)
    P = (1 << 61) - 1
    nb = layout.n_copy_bits
    frames = [torch.from_numpy(rng.integers(0, 256, size=copies * 384, dtype=np.uint8)).cuda()
              for _ in range(n_frames)]
    zg = [np.stack([rng.integers(0, P, size=gt.size, dtype=np.uint64),
                    rng.integers(0, P, size=gt.size, dtype=np.uint64)]) for _ in range(n_frames)]
    z2 = torch.from_numpy(pack_fp2(rng.integers(0, P, size=n_frames * nb, dtype=np.uint64),
                                   rng.integers(0, P, size=n_frames * nb, dtype=np.uint64))).cuda()
    pt = torch.zeros(2 * n_frames * (9 + nb), dtype=torch.int64, device="cuda")
    states = []
    for f in range(n_frames):
        import ctypes
        st = ctypes.create_string_buffer(lib.tp_fs_state_bytes())
        assert lib.tp_fs_init(st, b"truepix") == 0
        pre = np.array([f + 1, 7], np.uint64)
        assert lib.tp_fs_put_u64s(st, pre.ctypes.data, 2) == 0
        states.append(st.raw)
    vs = ctypes.create_string_buffer(lib.tp_vole_state_bytes())
    assert lib.tp_vole_state_init(vs, 0, None) == 0
    count = correlations_needed(layout)
    u = rng.integers(0, P, size=(n_frames, count, 2), dtype=np.uint64)
    v = rng.integers(0, P, size=(n_frames, count, 2), dtype=np.uint64)
    return lib, layout, (gt, i0, i1), frames, zg, z2, pt, b"".join(states), vs.raw * n_frames, u, v, count


def _run(bp, frames, zg, z2, pt, states, vs, u, v, count, graph):
    import torch
    d_st = torch.from_numpy(np.frombuffer(states, np.uint8).copy()).cuda()
    vole = dict(states=torch.from_numpy(np.frombuffer(vs, np.uint8).copy()).cuda(),
                u=torch.from_numpy(u.view(np.int64).reshape(-1).copy()).cuda(),
                v=torch.from_numpy(v.view(np.int64).reshape(-1).copy()).cuda(), count=count)
    bp.prove(frames, zg, z2, pt, None, transcripts=d_st, vole=vole, graph=graph)
    bp.stream.synchronize()
    return dict(claims=bp.claims.cpu().numpy().copy(), chal=bp.device_challenges.cpu().numpy().copy(),
                proof=bp.device_proof.cpu().numpy().copy(), wires=bp.wires.cpu().numpy().copy(),
                beta=bp.fin_beta.cpu().numpy().copy(), st=d_st.cpu().numpy().copy(),
                vs=vole["states"].cpu().numpy().copy())


def test_graph_rounds_match_launch_by_launch():
    import torch
    from truepix_b200.frame import BatchFrameProver
    lib, layout, gates, frames, zg, z2, pt, states, vs, u, v, count = _setup(5, 300, 1)
    s = torch.cuda.Stream()
    bp = BatchFrameProver([layout] * 5, *gates, stream=s)
    want = _run(bp, frames, zg, z2, pt, states, vs, u, v, count, graph=False)
    got = _run(bp, frames, zg, z2, pt, states, vs, u, v, count, graph=True)      # capture
    for k in want:
        np.testing.assert_array_equal(got[k], want[k], err_msg=k)
    assert lib.tp_batch_graph_replays(bp.handle) == 1
    # a replay on other frames of the same shape
    _, _, _, frames2, zg2, _, _, states2, _, u2, v2, _ = _setup(5, 300, 2)
    want2 = _run(bp, frames2, zg2, z2, pt, states2, vs, u2, v2, count, graph=False)
    got2 = _run(bp, frames2, zg2, z2, pt, states2, vs, u2, v2, count, graph=True)
    for k in want2:
        np.testing.assert_array_equal(got2[k], want2[k], err_msg=k)
    assert lib.tp_batch_graph_replays(bp.handle) == 2
    assert not np.array_equal(got2["chal"], got["chal"])


def test_autotuned_rounds_give_the_same_values():
    import torch
    from truepix_b200.frame import BatchFrameProver, autotune_rounds, round_tuning
    lib, layout, gates, frames, zg, z2, pt, states, vs, u, v, count = _setup(3, 1000, 3)
    s = torch.cuda.Stream()
    bp = BatchFrameProver([layout] * 3, *gates, stream=s)
    want = _run(bp, frames, zg, z2, pt, states, vs, u, v, count, graph=False)
    autotune_rounds(True)
    try:
        got = _run(bp, frames, zg, z2, pt, states, vs, u, v, count, graph=False)
    finally:
        autotune_rounds(False)
    for k in want:
        np.testing.assert_array_equal(got[k], want[k], err_msg=k)
    table = round_tuning()
    assert table and all(m in (2, 3, 4, 6, 8, 12, 16) for _, _, m in table)
    got_g = _run(bp, frames, zg, z2, pt, states, vs, u, v, count, graph=True)   # graph with the tuned splits
    for k in want:
        np.testing.assert_array_equal(got_g[k], want[k], err_msg=k)


def test_graph_needs_configured_frames():
    import torch
    from truepix_b200 import native
    from truepix_b200.frame import BatchFrameProver, FrameLayout
    lib = native.gkr()
    from proverlib import circuit
    gates = circuit("gray")
    bp = BatchFrameProver([FrameLayout(copies=64), FrameLayout(copies=200)], *gates, stream=torch.cuda.Stream())
    buf = torch.zeros(4096, dtype=torch.int64, device="cuda")
    p = buf.data_ptr()
    # the frames are not configured yet: rejected before any launch
    assert lib.tp_batch_vole_rounds_graph(bp.handle, p, p, p, p, p, 10, 0, p, None, p, p) == -1
    assert b"round" in lib.tp_last_error()


def test_uneven_batch_graph_matches_frames_alone():
    """frames of different sizes in one graph (each leaves the round loop after its
    own last round) against each frame proved alone launch by launch: its claims,
    challenges, VOLE proof elements, wires, beta, transcript and VOLE state"""
    import ctypes
    import torch
    from truepix_b200 import native
    from truepix_b200.frame import BatchFrameProver, FrameLayout, pack_fp2
    from truepix_b200.pipeline import correlations_needed
    from proverlib import circuit
    lib = native.gkr()
    gt, i0, i1 = circuit("gray")
    P = (1 << 61) - 1
    copies = [300, 70, 1000, 9, 300, 2]
    layouts = [FrameLayout(copies=c) for c in copies]
    B = len(layouts)
    rng = np.random.default_rng(11)
    frames = [torch.from_numpy(rng.integers(0, 256, size=c * 384, dtype=np.uint8)).cuda() for c in copies]
    zg = [np.stack([rng.integers(0, P, size=gt.size, dtype=np.uint64),
                    rng.integers(0, P, size=gt.size, dtype=np.uint64)]) for _ in range(B)]
    z2 = [rng.integers(0, P, size=(L.n_copy_bits, 2), dtype=np.uint64) for L in layouts]
    count = max(correlations_needed(L) for L in layouts)
    u = rng.integers(0, P, size=(B, count, 2), dtype=np.uint64)
    v = rng.integers(0, P, size=(B, count, 2), dtype=np.uint64)
    states = []
    for f in range(B):
        st = ctypes.create_string_buffer(lib.tp_fs_state_bytes())
        assert lib.tp_fs_init(st, b"truepix") == 0
        pre = np.array([f + 3, 5], np.uint64)
        assert lib.tp_fs_put_u64s(st, pre.ctypes.data, 2) == 0
        states.append(st.raw)
    vs0 = ctypes.create_string_buffer(lib.tp_vole_state_bytes())
    assert lib.tp_vole_state_init(vs0, 0, None) == 0

    def dev_fp2(rows):
        a = np.concatenate(rows) if rows else np.zeros((0, 2), np.uint64)
        return torch.from_numpy(pack_fp2(a[:, 0].copy(), a[:, 1].copy())).cuda()

    def run(idx, graph):
        Ls = [layouts[f] for f in idx]
        s = torch.cuda.Stream()
        bp = BatchFrameProver(Ls, gt, i0, i1, stream=s)
        z2d, ptd = {}, {}
        for C in sorted({L.padded_copies for L in Ls}):
            fs = [f for f in idx if layouts[f].padded_copies == C]
            z2d[C] = dev_fp2([z2[f] for f in fs])
            ptd[C] = torch.zeros(2 * len(fs) * (9 + int(np.log2(C))), dtype=torch.int64, device="cuda")
        d_st = torch.from_numpy(np.frombuffer(b"".join(states[f] for f in idx), np.uint8).copy()).cuda()
        vole = dict(states=torch.from_numpy(np.frombuffer(vs0.raw * len(idx), np.uint8).copy()).cuda(),
                    u=torch.from_numpy(u[idx].view(np.int64).reshape(-1).copy()).cuda(),
                    v=torch.from_numpy(v[idx].view(np.int64).reshape(-1).copy()).cuda(), count=count)
        bp.prove([frames[f] for f in idx], [zg[f] for f in idx], z2d, ptd, None, transcripts=d_st, vole=vole,
                 graph=graph)
        s.synchronize()
        R, n = bp.max_rounds, len(idx)
        return dict(claims=bp.claims.cpu().numpy().view(np.uint64).reshape(R, n, 8),
                    chal=bp.device_challenges.cpu().numpy().view(np.uint64).reshape(R, n, 2),
                    proof=bp.device_proof.cpu().numpy().view(np.uint64).reshape(R, n, 10),
                    wires=bp.wires.cpu().numpy().view(np.uint64).reshape(n, -1),
                    beta=bp.fin_beta.cpu().numpy().view(np.uint64).reshape(n, 2),
                    st=d_st.cpu().numpy().reshape(n, -1), vs=vole["states"].cpu().numpy().reshape(n, -1)), bp

    got, bp = run(list(range(B)), graph=True)
    assert lib.tp_batch_graph_replays(bp.handle) == 1
    for f in range(B):
        want, _ = run([f], graph=False)
        r = layouts[f].n_copy_bits
        np.testing.assert_array_equal(got["claims"][:r, f], want["claims"][:r, 0], err_msg="claims %d" % f)
        np.testing.assert_array_equal(got["chal"][:r, f], want["chal"][:r, 0], err_msg="chal %d" % f)
        np.testing.assert_array_equal(got["proof"][:r, f], want["proof"][:r, 0], err_msg="proof %d" % f)
        for k in ("wires", "beta", "st", "vs"):
            np.testing.assert_array_equal(got[k][f], want[k][0], err_msg="%s %d" % (k, f))
