"""Late rounds and line projection on the device (tp_late_rounds_dev,
BatchFrameProver.prove_late) against the reference: given challenges, bit-exact
with vectors made by the reference's own LayerProver (tests/golden/
late_golden.npz); the VOLE-committed rounds, bit-exact with the reference's
LayerProver + ExtVOLECommit + FiatShamir chain (tests/golden/
layer_vole_golden.npz: coefficients, commitments, equality values, challenges,
line, VOLE state, transcript digest, and the layer's closing proofs: product
proof, proofs of knowledge, equality proof, input point, its tag and value
proof); batches against the oracle; whole 1080p
frames after the device early rounds, against the oracle and against the
multilinear extension of the frame's bytes at the two late points."""
import ctypes
import struct

import numpy as np
import pytest

from latelib import golden_cases, oracle, pairs

pytestmark = pytest.mark.gpu

I32P = ctypes.POINTER(ctypes.c_int)
P61 = (1 << 61) - 1


@pytest.fixture(scope="module")
def lib():
    from truepix_b200 import native
    return native.gkr()


def dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a, np.uint64).reshape(-1).view(np.int64).copy()).cuda()


def host(t, shape):
    return t.cpu().numpy().view(np.uint64).reshape(shape)


def run_given(lib, n, gates, wires, beta, zg, chal, n_frames=1, per_frame=1):
    import torch
    gt, i0, i1 = (np.ascontiguousarray(r, np.int32) for r in gates)
    d_w, d_b, d_z, d_c = dev(wires), dev(beta), dev(zg), dev(chal)
    coefs = torch.zeros(n_frames * 12 * n, dtype=torch.int64, device="cuda")
    line = torch.zeros(n_frames * 2 * (n + 1), dtype=torch.int64, device="cuda")
    cho = torch.zeros(n_frames * 4 * n, dtype=torch.int64, device="cuda")
    rc = lib.tp_late_rounds_dev(n_frames, n, gt.size, gt.ctypes.data_as(I32P), i0.ctypes.data_as(I32P),
                                i1.ctypes.data_as(I32P), d_w.data_ptr(), d_b.data_ptr(), d_z.data_ptr(), per_frame,
                                d_c.data_ptr(), None, None, None, None, 0, 0, 0, coefs.data_ptr(), line.data_ptr(),
                                cho.data_ptr(), None, None, None, 0, 0, None, None, None, 0, None)
    assert rc == 0, lib.tp_last_error()
    torch.cuda.synchronize()
    return (host(coefs, (n_frames, 6 * n, 2)), host(line, (n_frames, n + 1, 2)), host(cho, (n_frames, 2 * n, 2)))


def test_given_challenges_match_reference_layer_prover(lib):
    n_cases = 0
    for c in golden_cases():
        n, nb = c["n_in_bits"], c["n_copy_bits"]
        coefs, line, cho = run_given(lib, n, c["gates"], c["wires"], c["beta"], c["zg"], c["chal"][nb:])
        np.testing.assert_array_equal(coefs[0], c["late"], err_msg=c["name"])
        np.testing.assert_array_equal(line[0], c["final"], err_msg=c["name"])
        np.testing.assert_array_equal(cho[0], c["chal"][nb:])
        n_cases += 1
    assert n_cases == 6


def test_vole_rounds_match_reference_chain(lib):
    import torch
    from layervole import cases, early_transcript, vole_state_fields, vole_state_mid
    n_cases = 0
    for c in cases():
        n, nb = c["n_in_bits"], c["nb"]
        st, ch = early_transcript(lib, c)
        assert [list(x) for x in ch] == [[int(a), int(b)] for a, b in c["chal"][:nb]]
        d_st = torch.frombuffer(bytearray(st.raw), dtype=torch.uint8).cuda()
        d_vs = torch.frombuffer(bytearray(vole_state_mid(c)), dtype=torch.uint8).cuda()
        gt, i0, i1 = (np.ascontiguousarray(r, np.int32) for r in c["gates"])
        d_w, d_b, d_z, d_u, d_v = dev(c["wires"]), dev(c["beta"]), dev(c["zg"]), dev(c["u"]), dev(c["v"])
        coefs = torch.zeros(12 * n, dtype=torch.int64, device="cuda")
        line = torch.zeros(2 * (n + 1), dtype=torch.int64, device="cuda")
        cho = torch.zeros(4 * n, dtype=torch.int64, device="cuda")
        proof = torch.zeros(16 * n, dtype=torch.int64, device="cuda")
        d_z2, d_w3 = dev(c["z2"]), dev(c["chal"][:nb])
        closing = torch.zeros(2 * (n + 10), dtype=torch.int64, device="cuda")
        point = torch.zeros(2 * (n + nb), dtype=torch.int64, device="cuda")
        tag = torch.zeros(2, dtype=torch.int64, device="cuda")
        st_late = None
        for close in (False, True):
            if close:   # again from the same start, now with the layer's closing proofs
                d_st.copy_(torch.frombuffer(bytearray(st.raw), dtype=torch.uint8).cuda())
                d_vs.copy_(torch.frombuffer(bytearray(vole_state_mid(c)), dtype=torch.uint8).cuda())
            rc = lib.tp_late_rounds_dev(1, n, gt.size, gt.ctypes.data_as(I32P), i0.ctypes.data_as(I32P),
                                        i1.ctypes.data_as(I32P), d_w.data_ptr(), d_b.data_ptr(), d_z.data_ptr(), 1,
                                        None, d_st.data_ptr(), d_vs.data_ptr(), d_u.data_ptr(), d_v.data_ptr(),
                                        len(c["u"]), 0, nb, coefs.data_ptr(), line.data_ptr(), cho.data_ptr(),
                                        proof.data_ptr(), d_z2.data_ptr(), d_w3.data_ptr(), 0, 1,
                                        closing.data_ptr() if close else None, point.data_ptr(), tag.data_ptr(), 0,
                                        None)
            assert rc == 0, lib.tp_last_error()
            torch.cuda.synchronize()
            if not close:
                st_late, vs_late = d_st.cpu().numpy().tobytes(), d_vs.cpu().numpy().tobytes()
        np.testing.assert_array_equal(host(coefs, (6 * n, 2)), c["coefs"][4 * nb:])
        np.testing.assert_array_equal(host(cho, (2 * n, 2)), c["chal"][nb:])
        pr = host(proof, (2 * n, 4, 2))
        np.testing.assert_array_equal(pr[:, :3].reshape(-1, 2), c["d"][4 * nb:])
        np.testing.assert_array_equal(pr[:, 3], c["vz"][nb:])
        np.testing.assert_array_equal(host(line, (n + 1, 2)), c["final"])
        f = vole_state_fields(vs_late)
        assert f["idx"] == int(c["used"][0]) and f["bad"] == 0 and f["has_prev"] == 1
        assert f["prev"] == tuple(int(x) for x in c["prev"][0])
        assert f["v_elem"] == [tuple(int(x) for x in r) for r in c["v_elem"]]
        assert f["out_elem"] == [tuple(int(x) for x in r) for r in c["out_elem"]]
        d = ctypes.create_string_buffer(32)
        assert lib.tp_fs_digest(st_late, d) == 0
        assert d.raw == c["digest"].tobytes()
        # the closing proofs, row by row (their values go into the transcript in this order)
        got = host(closing, (n + 10, 2))
        rows = [k for k in range(n + 10) if not np.array_equal(got[k], c["closing"][k])]
        assert not rows, f"{c['name']}: closing rows {rows} differ from the reference chain"
        np.testing.assert_array_equal(host(point, (n + nb, 2)), c["point"])
        np.testing.assert_array_equal(host(tag, (1, 2)), c["tag"])
        assert vole_state_fields(d_vs.cpu().numpy().tobytes())["idx"] == int(c["used_closed"][0])
        assert lib.tp_fs_digest(d_st.cpu().numpy().tobytes(), d) == 0
        assert d.raw == c["digest_closed"].tobytes()
        n_cases += 1
    assert n_cases == 2


def test_running_out_of_correlations_stops_the_frame(lib):
    """a frame whose correlations end inside the late rounds is marked bad and
    stops at that round; the other frame of the launch finishes"""
    import torch
    from layervole import cases, early_transcript, vole_state_fields, vole_state_mid
    c = [x for x in cases() if x["name"] == "random"][0]
    n, nb = c["n_in_bits"], c["nb"]
    st, _ = early_transcript(lib, c)
    used = int(c["used_mid"][0])
    count = len(c["u"])
    short = used + 3 * 4 + 1           # frame 1: enough correlations for four late rounds, not a fifth
    shift = count - short
    u = np.zeros((2, count, 2), np.uint64)
    v = np.zeros((2, count, 2), np.uint64)
    u[0], v[0] = c["u"], c["v"]
    u[1, used + shift:], v[1, used + shift:] = c["u"][used:short], c["v"][used:short]
    vs0 = bytearray(vole_state_mid(c))
    vs1 = bytearray(vs0)
    struct.pack_into("<Q", vs1, 0, used + shift)   # frame 1's next correlation: its list ends at `count`
    d_st = torch.frombuffer(bytearray(st.raw * 2), dtype=torch.uint8).cuda()
    d_vs = torch.frombuffer(vs0 + vs1, dtype=torch.uint8).cuda()
    gt, i0, i1 = (np.ascontiguousarray(r, np.int32) for r in c["gates"])
    d_w = dev(np.concatenate([c["wires"], c["wires"]]))
    d_b = dev(np.concatenate([c["beta"], c["beta"]]))
    d_z, d_u, d_v = dev(c["zg"]), dev(u), dev(v)
    coefs = torch.zeros(2 * 12 * n, dtype=torch.int64, device="cuda")
    line = torch.zeros(2 * 2 * (n + 1), dtype=torch.int64, device="cuda")
    cho = torch.zeros(2 * 4 * n, dtype=torch.int64, device="cuda")
    rc = lib.tp_late_rounds_dev(2, n, gt.size, gt.ctypes.data_as(I32P), i0.ctypes.data_as(I32P),
                                i1.ctypes.data_as(I32P), d_w.data_ptr(), d_b.data_ptr(), d_z.data_ptr(), 0, None,
                                d_st.data_ptr(), d_vs.data_ptr(), d_u.data_ptr(), d_v.data_ptr(), count, 0, nb,
                                coefs.data_ptr(), line.data_ptr(), cho.data_ptr(), None, None, None, 0, 0, None, None,
                                None, 0, None)
    assert rc == 0, lib.tp_last_error()
    torch.cuda.synchronize()
    raw = d_vs.cpu().numpy().tobytes()
    f0, f1 = vole_state_fields(raw[:160]), vole_state_fields(raw[160:])
    assert f0["bad"] == 0 and f0["idx"] == int(c["used"][0])
    assert f1["bad"] == 1 and f1["idx"] == used + shift + 12
    ch = host(cho, (2, 2 * n, 2))
    np.testing.assert_array_equal(ch[0], c["chal"][nb:])
    np.testing.assert_array_equal(ch[1][:4], c["chal"][nb:nb + 4])    # the same first four rounds
    assert (ch[1][4] == 0).all()


def test_batch_matches_oracle(lib):
    """8 frames of the gray circuit with field-size wires, one weight vector per frame"""
    import os
    from latelib import ROOT
    circ = np.load(os.path.join(ROOT, "tests", "golden", "circuits.npz"))
    gates = (circ["gray_type"], circ["gray_in0"], circ["gray_in1"])
    rng = np.random.default_rng(404)
    B, n = 8, 9
    wires = rng.integers(0, P61, size=(B, 512, 2), dtype=np.uint64)
    beta = rng.integers(0, P61, size=(B, 2), dtype=np.uint64)
    zg = rng.integers(0, P61, size=(B, 384, 2), dtype=np.uint64)
    chal = rng.integers(0, P61, size=(B, 18, 2), dtype=np.uint64)
    coefs, line, cho = run_given(lib, n, gates, wires, beta, zg, chal, n_frames=B)
    g3 = tuple([int(x) for x in a] for a in gates)
    for f in range(B):
        cf, h, _, _ = oracle.late_rounds(pairs(wires[f]), pairs(beta[f])[0], pairs(zg[f]), g3, n, pairs(chal[f]))
        assert [x for r in cf for x in r] == pairs(coefs[f]), f
        assert h == pairs(line[f]), f
    # one weight vector for every frame gives frame 0's answer for frame 0
    coefs1, line1, _ = run_given(lib, n, gates, wires, beta, zg[0], chal, n_frames=B, per_frame=0)
    np.testing.assert_array_equal(coefs1[0], coefs[0])
    np.testing.assert_array_equal(line1[0], line[0])


def test_whole_frames_after_device_early_rounds(lib):
    """Two 1080p gray frames: early rounds (BatchFrameProver.prove), then
    prove_late; the late outputs equal the oracle on the batch's own wires and
    beta, and the line's values at 0 and 1 equal the multilinear extension of
    each frame's input vector at (w1, w3) and (w2, w3) (layer.py's identity)."""
    import os
    import torch
    from latelib import ROOT
    from truepix_b200.frame import BatchFrameProver, FrameLayout, pack_fp2
    circ = np.load(os.path.join(ROOT, "tests", "golden", "circuits.npz"))
    gt, i0, i1 = circ["gray_type"], circ["gray_in0"], circ["gray_in1"]
    B = 2
    layout = FrameLayout.for_frame(1080, 1920)
    nb, n = layout.n_copy_bits, 9
    rng = np.random.default_rng(1080)
    pix = [torch.from_numpy(rng.integers(0, 256, size=layout.copies * 384, dtype=np.uint8)).cuda() for _ in range(B)]
    z1s = [rng.integers(0, P61, size=(2, 384), dtype=np.uint64) for _ in range(B)]
    z2 = rng.integers(0, P61, size=(B, nb, 2), dtype=np.uint64)
    pt = rng.integers(0, P61, size=(B, nb + 9, 2), dtype=np.uint64)
    z2d = torch.from_numpy(pack_fp2(z2[..., 0].reshape(-1), z2[..., 1].reshape(-1))).cuda()
    ptd = torch.from_numpy(pack_fp2(pt[..., 0].reshape(-1), pt[..., 1].reshape(-1))).cuda()
    early = rng.integers(0, P61, size=(nb, B, 2), dtype=np.uint64)
    late = rng.integers(0, P61, size=(B, 2 * n, 2), dtype=np.uint64)
    bp = BatchFrameProver([layout] * B, gt, i0, i1)
    bp.prove(pix, z1s, z2d, ptd, early)
    bp.prove_late(z1s, challenges=late)
    torch.cuda.synchronize()
    coefs = host(bp.late_coefs, (B, 6 * n, 2))
    line = host(bp.line, (B, n + 1, 2))
    g3 = ([int(x) for x in gt], [int(x) for x in i0], [int(x) for x in i1])
    for f in range(B):
        _, wires, beta, _ = bp.results(f)
        zg = list(zip([int(x) for x in z1s[f][0]], [int(x) for x in z1s[f][1]]))
        cf, h, v1, v2 = oracle.late_rounds(pairs(wires), beta, zg, g3, n, pairs(late[f]))
        assert [x for r in cf for x in r] == pairs(coefs[f])
        assert h == pairs(line[f])
        for t, w in ((0, late[f][:n]), (1, late[f][n:])):
            point = np.concatenate([w, early[:, f]])          # wire bits first, then copy bits
            d_pt = torch.from_numpy(pack_fp2(point[:, 0], point[:, 1])).cuda()
            out = torch.zeros(2, dtype=torch.int64, device="cuda")
            assert lib.tp_mle_eval_pixels(pix[f].data_ptr(), layout.copies, layout.padded_copies, 384, 512, 384, 128,
                                          d_pt.data_ptr(), out.data_ptr(), None) == 0
            torch.cuda.synchronize()
            m = tuple(int(x) for x in host(out, (2,)))
            if t == 0:
                assert m == h[0] == v1                      # the line at 0
            else:
                s = (0, 0)
                for x in h:
                    s = oracle.add(s, x)
                assert m == s == v2                         # the line at 1: the sum of its coefficients


def test_bad_arguments_are_rejected(lib):
    import torch
    g = np.zeros(4, np.int32)
    bufs = [torch.zeros(256, dtype=torch.int64, device="cuda") for _ in range(7)]
    wires, beta, zg, chal, coefs, line, cho = (b.data_ptr() for b in bufs)

    def call(n=3, gt=g, i0=g, i1=g, ch=chal, proof=None, closing=None):
        return lib.tp_late_rounds_dev(1, n, len(gt), np.ascontiguousarray(gt, np.int32).ctypes.data_as(I32P),
                                      np.ascontiguousarray(i0, np.int32).ctypes.data_as(I32P),
                                      np.ascontiguousarray(i1, np.int32).ctypes.data_as(I32P), wires, beta, zg, 1,
                                      ch, None, None, None, None, 0, 0, 0, coefs, line, cho, proof, None, None, 0, 0,
                                      closing, line, cho, 0, None)

    assert call() == 0
    assert call(n=10) == -1
    assert call(n=0) == -1
    assert call(gt=np.array([13, 0, 0, 0])) == -1
    assert call(i0=np.array([0, 8, 0, 0])) == -1            # 8 wires at n = 3
    assert b"gate 1" in lib.tp_last_error()
    assert call(ch=None) == -1                              # neither challenges nor transcripts
    assert call(proof=coefs) == -1                          # proof only with VOLE rounds
    assert call(closing=coefs) == -1                        # closing proofs only with VOLE rounds
    big = np.zeros(769, np.int32)
    assert call(gt=big, i0=big, i1=big) == -1
    torch.cuda.synchronize()


def test_whole_layer_proof_on_device_matches_restatement(lib):
    """Three 360p gray frames, the whole input layer's proof on the device: the
    VOLE-committed early rounds (BatchFrameProver.prove with transcripts and
    VOLE states), then prove_late: late rounds, line and closing proofs, with no
    host round trip. Per frame, the restated loop (hashlib transcript, the
    oracle's late rounds, the restated closing proofs) fed with the device's
    early claims draws the same challenges and puts the same values, and ends
    in the same transcript digest."""
    import os
    import torch
    from fslib import PyTranscript, f2add, f2mul, f2sub, interpolate_cubic, replay_lib
    from latelib import ROOT
    from layervole import closing_python
    from truepix_b200.frame import BatchFrameProver, FrameLayout, pack_fp2
    circ = np.load(os.path.join(ROOT, "tests", "golden", "circuits.npz"))
    gt, i0, i1 = circ["gray_type"], circ["gray_in0"], circ["gray_in1"]
    B, n = 3, 9
    layout = FrameLayout.for_frame(360, 640)
    nb = layout.n_copy_bits
    rng = np.random.default_rng(360)
    pix = [torch.from_numpy(rng.integers(0, 256, size=layout.copies * 384, dtype=np.uint8)).cuda() for _ in range(B)]
    z1s = [rng.integers(0, P61, size=(2, 384), dtype=np.uint64) for _ in range(B)]
    z2 = rng.integers(0, P61, size=(B, nb, 2), dtype=np.uint64)
    pt = rng.integers(0, P61, size=(B, nb + 9, 2), dtype=np.uint64)
    count = 4 * nb + 6 * n + (n + 2) + 5
    u = rng.integers(0, P61, size=(B, count, 2), dtype=np.uint64)
    v = rng.integers(0, P61, size=(B, count, 2), dtype=np.uint64)
    prefixes = [[f, 11, 7] for f in range(B)]
    states = b"".join(replay_lib(lib, "truepix", [["u64s", p]])[2].raw for p in prefixes)
    vsb = b""
    for f in range(B):
        vs = ctypes.create_string_buffer(lib.tp_vole_state_bytes())
        assert lib.tp_vole_state_init(vs, 2, None) == 0
        vsb += vs.raw
    d_fs = torch.from_numpy(np.frombuffer(states, np.uint8).copy()).cuda()
    vole = dict(states=torch.from_numpy(np.frombuffer(vsb, np.uint8).copy()).cuda(),
                u=torch.from_numpy(u.view(np.int64).reshape(-1)).cuda(),
                v=torch.from_numpy(v.view(np.int64).reshape(-1)).cuda(), count=count)
    bp = BatchFrameProver([layout] * B, gt, i0, i1)
    bp.prove(pix, z1s, torch.from_numpy(pack_fp2(z2[..., 0].reshape(-1), z2[..., 1].reshape(-1))).cuda(),
             torch.from_numpy(pack_fp2(pt[..., 0].reshape(-1), pt[..., 1].reshape(-1))).cuda(), None,
             transcripts=d_fs, vole=vole)
    bp.prove_late(z1s, transcripts=d_fs, vole=vole)
    torch.cuda.synchronize()
    claims = host(bp.claims, (nb, B, 4, 2))
    early_ch = host(bp.device_challenges, (nb, B, 2))
    late_ch = host(bp.late_challenges, (B, 2 * n, 2))
    late_pr = host(bp.late_proof, (B, 2 * n, 4, 2))
    closing = host(bp.closing, (B, n + 10, 2))
    point = host(bp.input_point, (B, n + nb, 2))
    tag = host(bp.input_tag, (B, 2))
    raw = d_fs.cpu().numpy().tobytes()
    nst = lib.tp_fs_state_bytes()
    g3 = ([int(x) for x in gt], [int(x) for x in i0], [int(x) for x in i1])
    for f in range(B):
        T = PyTranscript("truepix")
        T.u64s(prefixes[f])
        uu, vv = pairs(u[f]), pairs(v[f])
        idx, prev = 2, None
        v_elem, out_elem = [(0, 0)] * 4, [(0, 0)] * 4
        _, wires, beta, _ = bp.results(f)
        zg = list(zip([int(x) for x in z1s[f][0]], [int(x) for x in z1s[f][1]]))
        late = oracle.LateRounds(pairs(wires), beta, zg, g3, n)
        chals, late_vals = [], []
        for rd in range(nb + 2 * n):
            if rd < nb:
                cf = interpolate_cubic(*pairs(claims[rd, f]))
            else:
                cf = late.coefs()
            tags = []
            for k, x in enumerate(cf):
                tags.append(vv[idx])
                d = f2sub(x, uu[idx])
                idx += 1
                T.fp2(*d)
                if rd >= nb:
                    late_vals.append(d)
                v_elem[k] = f2add(v_elem[k], tags[-1])
                out_elem[k] = f2add(out_elem[k], x)
            now = tags[0]
            for t in tags:
                now = f2add(now, t)
            e = T.ext("eq")
            vz = f2mul(now, e) if prev is None else f2mul(f2sub(prev, now), e)
            T.fp2(*vz)
            if rd >= nb:
                late_vals.append(vz)
            r = T.ext("sc-0-%d" % rd)
            chals.append(r)
            p = tags[-1]
            for t in reversed(tags[:-1]):
                p = f2add(f2mul(p, r), t)
            prev = p
            if rd >= nb:
                late.next_round(r)
        assert chals[:nb] == pairs(early_ch[:, f]), f
        assert chals[nb:] == pairs(late_ch[f]), f
        assert late_vals == pairs(late_pr[f]), f
        w3, w1, w2 = chals[:nb], chals[nb:nb + n], chals[nb + n:]
        cl, pnt, tg, used = closing_python(T, late.line(), prev, idx, v_elem, out_elem, uu, vv, w1, w2, w3,
                                           pairs(z2[f]), zg, g3)
        assert cl == pairs(closing[f]), f
        assert pnt == pairs(point[f]) and tg == tuple(int(x) for x in tag[f])
        d = ctypes.create_string_buffer(32)
        assert lib.tp_fs_digest(raw[f * nst:(f + 1) * nst], d) == 0
        assert d.raw == T.h.digest(), f
        st = vole["states"].cpu().numpy().tobytes()[f * 160:(f + 1) * 160]
        assert struct.unpack_from("<Q", st, 0)[0] == used
