"""The Fiat-Shamir transcript (tp_fs_*): the host entry points against the
reference's own FiatShamir class (tests/golden/fs_golden.npz), and the batched
device entry points (one state per frame in device memory) against the host
ones: a batch of transcripts moved to the device absorbs each frame's four
claims and draws its challenge round after round, bit-identical to doing the
same on the host, and continues on the host after the copy back."""
import ctypes

import numpy as np
import pytest

from fslib import P61, golden, replay_lib, scripts

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib():
    from truepix_b200 import native
    return native.gkr()


def test_host_transcript_matches_reference_vectors(lib):
    g = golden()
    for name, protocol, ops in scripts(g):
        outs, digs, _ = replay_lib(lib, protocol, ops)
        np.testing.assert_array_equal(outs, g["fsout_" + name])
        assert digs == g["fsdigest_" + name].tobytes(), name


def test_device_batch_rounds_match_host(lib):
    import torch
    nb = lib.tp_fs_state_bytes()
    assert nb == 120
    n, rounds = 96, 14
    rng = np.random.default_rng(7)
    host = []
    for f in range(n):   # distinct histories of different lengths (partial blocks differ)
        _, _, st = replay_lib(lib, "truepix", [["u64s", [f] * (1 + f % 9)], ["str", "frame-%d" % f],
                                               ["ext", "z2-0"]])
        host.append(st)
    dev = torch.device("cuda", 0)
    d_states = torch.from_numpy(np.frombuffer(b"".join(s.raw for s in host), np.uint8).copy()).to(dev)
    d_claims = torch.empty(n * 8, dtype=torch.int64, device=dev)
    d_chal = torch.empty(n * 2, dtype=torch.int64, device=dev)
    s = torch.cuda.current_stream().cuda_stream
    re, im = ctypes.c_uint64(), ctypes.c_uint64()
    for rd in range(rounds):
        claims = rng.integers(0, P61, size=n * 8, dtype=np.uint64)
        claims[:8] = P61 - 1 if rd % 2 else 0
        d_claims.copy_(torch.from_numpy(claims.view(np.int64)))
        label = ("sc-0-%d" % rd).encode()
        assert lib.tp_fs_put_fp2s_dev(d_states.data_ptr(), n, d_claims.data_ptr(), 4, s) == 0, lib.tp_last_error()
        assert lib.tp_fs_rand_ext_dev(d_states.data_ptr(), n, label, d_chal.data_ptr(), s) == 0, lib.tp_last_error()
        got = d_chal.cpu().numpy().view(np.uint64).reshape(n, 2)
        c = claims.reshape(n, 4, 2)
        for f in range(n):
            r = np.ascontiguousarray(c[f, :, 0])
            i = np.ascontiguousarray(c[f, :, 1])
            assert lib.tp_fs_put_fp2s(host[f], r.ctypes.data, i.ctypes.data, 4) == 0
            assert lib.tp_fs_rand_ext(host[f], label, ctypes.byref(re), ctypes.byref(im)) == 0
            assert (int(got[f, 0]), int(got[f, 1])) == (re.value, im.value), (rd, f)
            assert re.value < P61 and im.value < P61
    back = d_states.cpu().numpy().tobytes()
    d1, d2 = ctypes.create_string_buffer(32), ctypes.create_string_buffer(32)
    for f in range(n):
        st = ctypes.create_string_buffer(back[f * nb:(f + 1) * nb], nb)
        assert lib.tp_fs_digest(st, d1) == 0 and lib.tp_fs_digest(host[f], d2) == 0
        assert d1.raw == d2.raw
        # the device state continues on the host like the host one
        a = ctypes.c_uint64(), ctypes.c_uint64()
        assert lib.tp_fs_rand_ext(st, b"tau-0", ctypes.byref(a[0]), ctypes.byref(a[1])) == 0
        assert lib.tp_fs_rand_ext(host[f], b"tau-0", ctypes.byref(re), ctypes.byref(im)) == 0
        assert (a[0].value, a[1].value) == (re.value, im.value)


def test_transcript_rejects_bad_arguments(lib):
    import torch
    st = ctypes.create_string_buffer(lib.tp_fs_state_bytes())
    assert lib.tp_fs_init(st, b"truepix") == 0
    re, im = ctypes.c_uint64(), ctypes.c_uint64()
    assert lib.tp_fs_rand_ext(st, b"x" * 65, ctypes.byref(re), ctypes.byref(im)) == -1
    assert b"64 bytes" in lib.tp_last_error()
    assert lib.tp_fs_put_u64s(st, None, 0) == -1
    buf = torch.zeros(120, dtype=torch.uint8, device="cuda")
    assert lib.tp_fs_rand_ext_dev(buf.data_ptr(), 0, b"a", buf.data_ptr(), None) == -1


def test_batched_rounds_with_device_transcripts_match_host_transcripts(lib):
    """BatchFrameProver driven by device transcripts (claims put and challenges
    drawn on the device, tp_batch_fold_dev) against the same batch driven by host
    transcripts fed with the claims read back every round: identical claims,
    challenges, wires, beta, MLE and final transcript states."""
    import torch
    from truepix_b200.frame import BatchFrameProver, FrameLayout, pack_fp2
    import os
    from fslib import ROOT
    c = np.load(os.path.join(ROOT, "tests", "golden", "circuits.npz"))
    gt, i0, i1 = c["gray_type"], c["gray_in0"], c["gray_in1"]
    B = 6
    layout = FrameLayout.for_frame(240, 426)
    nb = layout.n_copy_bits
    rng = np.random.default_rng(99)
    dev = torch.device("cuda", 0)
    pix = [torch.from_numpy(rng.integers(0, 256, size=layout.copies * 384, dtype=np.uint8)).to(dev)
           for _ in range(B)]
    z1 = np.stack([rng.integers(0, P61, size=384, dtype=np.uint64) for _ in range(2)])
    z2 = rng.integers(0, P61, size=(nb, 2), dtype=np.uint64)
    pt = rng.integers(0, P61, size=(nb + 9, 2), dtype=np.uint64)
    z2d = torch.from_numpy(pack_fp2(z2[:, 0], z2[:, 1])).to(dev).repeat(B)
    ptd = torch.from_numpy(pack_fp2(pt[:, 0], pt[:, 1])).to(dev).repeat(B)
    states = [replay_lib(lib, "truepix", [["u64s", [f, 7]], ["ext", "z2-0"]])[2] for f in range(B)]

    # host transcripts: read each round's claims back, draw the challenges on the host
    host_prover = BatchFrameProver([layout] * B, gt, i0, i1)
    chal = np.zeros((nb, B, 2), np.uint64)
    hstates = [ctypes.create_string_buffer(s.raw, len(s.raw)) for s in states]
    re, im = ctypes.c_uint64(), ctypes.c_uint64()

    def hook(k):
        torch.cuda.synchronize()
        cl = host_prover.claims.cpu().numpy().view(np.uint64).reshape(nb, B, 4, 2)[k]
        for f in range(B):
            r, i = np.ascontiguousarray(cl[f, :, 0]), np.ascontiguousarray(cl[f, :, 1])
            assert lib.tp_fs_put_fp2s(hstates[f], r.ctypes.data, i.ctypes.data, 4) == 0
            assert lib.tp_fs_rand_ext(hstates[f], ("sc-0-%d" % k).encode(), ctypes.byref(re), ctypes.byref(im)) == 0
            chal[k, f] = (re.value, im.value)

    host_prover.prove(pix, [z1] * B, z2d, ptd, chal, round_hook=hook)
    torch.cuda.synchronize()

    dev_prover = BatchFrameProver([layout] * B, gt, i0, i1)
    d_states = torch.from_numpy(np.frombuffer(b"".join(s.raw for s in states), np.uint8).copy()).to(dev)
    dev_prover.prove(pix, [z1] * B, z2d, ptd, None, transcripts=d_states)
    torch.cuda.synchronize()

    got_ch = dev_prover.device_challenges.cpu().numpy().view(np.uint64).reshape(nb, B, 2)
    np.testing.assert_array_equal(got_ch, chal)
    for f in range(B):
        a, b = host_prover.results(f), dev_prover.results(f)
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]) and a[2] == b[2] and a[3] == b[3], f
    back = d_states.cpu().numpy().tobytes()
    d1, d2 = ctypes.create_string_buffer(32), ctypes.create_string_buffer(32)
    n = lib.tp_fs_state_bytes()
    for f in range(B):
        st = ctypes.create_string_buffer(back[f * n:(f + 1) * n], n)
        assert lib.tp_fs_digest(st, d1) == 0 and lib.tp_fs_digest(hstates[f], d2) == 0
        assert d1.raw == d2.raw


def _vole_case(g, name):
    return {k[len(name) + 1:]: g[k] for k in g.files if k.startswith(name + "_")}


def test_vole_round_kernel_matches_reference_vectors(lib):
    """tp_vole_round_dev round after round on the golden cases (made from the
    reference's util / ExtVOLECommit / FiatShamir): every challenge, equality
    value, the final previous value, correlations used, running sums, digest."""
    import os
    import torch
    from fslib import ROOT
    g = np.load(os.path.join(ROOT, "tests", "golden", "vole_round_golden.npz"))
    dev = torch.device("cuda", 0)
    for name in ("r3", "r14", "r11_prev"):
        c = _vole_case(g, name)
        _, _, st = replay_lib(lib, "truepix", [["u64s", [int(x) for x in c["prefix"]]]])
        vs = ctypes.create_string_buffer(lib.tp_vole_state_bytes())
        prev = np.ascontiguousarray(c["prev0"], np.uint64)
        assert lib.tp_vole_state_init(vs, int(c["start"][0]), prev.ctypes.data if c["has_prev"][0] else None) == 0
        d_fs = torch.from_numpy(np.frombuffer(st.raw, np.uint8).copy()).to(dev)
        d_vs = torch.from_numpy(np.frombuffer(vs.raw, np.uint8).copy()).to(dev)
        d_u = torch.from_numpy(np.ascontiguousarray(c["u"]).view(np.int64).reshape(-1)).to(dev)
        d_v = torch.from_numpy(np.ascontiguousarray(c["v"]).view(np.int64).reshape(-1)).to(dev)
        count = c["u"].shape[0]
        d_cl = torch.empty(8, dtype=torch.int64, device=dev)
        d_ch = torch.empty(2, dtype=torch.int64, device=dev)
        d_pf = torch.empty(10, dtype=torch.int64, device=dev)
        s = torch.cuda.current_stream().cuda_stream
        for rd, cl in enumerate(c["claims"]):
            d_cl.copy_(torch.from_numpy(np.ascontiguousarray(cl).view(np.int64).reshape(-1)))
            assert lib.tp_vole_round_dev(d_fs.data_ptr(), d_vs.data_ptr(), 1, d_cl.data_ptr(), d_u.data_ptr(),
                                         d_v.data_ptr(), count, ("sc-0-%d" % rd).encode(), d_ch.data_ptr(),
                                         d_pf.data_ptr(), s) == 0, lib.tp_last_error()
            np.testing.assert_array_equal(d_ch.cpu().numpy().view(np.uint64), c["chals"][rd])
            np.testing.assert_array_equal(d_pf.cpu().numpy().view(np.uint64)[8:], c["vzs"][rd])
        w = d_vs.cpu().numpy()
        idx = int(w[:8].view(np.uint64)[0])
        has_prev, bad = w[8:16].view(np.uint32)
        words = w[16:].view(np.uint64).reshape(9, 2)
        assert idx == int(c["used"][0]) and bad == 0 and has_prev == 1
        np.testing.assert_array_equal(words[0], c["prev"][0])
        np.testing.assert_array_equal(words[1:5], c["v_elem"])
        np.testing.assert_array_equal(words[5:9], c["out_elem"])
        dg = ctypes.create_string_buffer(32)
        st2 = ctypes.create_string_buffer(d_fs.cpu().numpy().tobytes(), len(st.raw))
        assert lib.tp_fs_digest(st2, dg) == 0 and dg.raw == c["digest"].tobytes()


def test_batched_vole_rounds_match_restatement_and_stop_when_correlations_run_out(lib):
    """BatchFrameProver with per-frame transcripts and VOLE states: each frame's
    challenges equal the restated round loop replayed on that frame's claims;
    a frame given too few correlations is marked and draws nothing."""
    import os
    import torch
    from truepix_b200.frame import BatchFrameProver, FrameLayout, pack_fp2
    from fslib import ROOT, vole_rounds_python
    c = np.load(os.path.join(ROOT, "tests", "golden", "circuits.npz"))
    gt, i0, i1 = c["gray_type"], c["gray_in0"], c["gray_in1"]
    B = 5
    layout = FrameLayout.for_frame(180, 320)
    nb = layout.n_copy_bits
    rng = np.random.default_rng(5)
    dev = torch.device("cuda", 0)
    pix = [torch.from_numpy(rng.integers(0, 256, size=layout.copies * 384, dtype=np.uint8)).to(dev)
           for _ in range(B)]
    z1 = np.stack([rng.integers(0, P61, size=384, dtype=np.uint64) for _ in range(2)])
    z2 = rng.integers(0, P61, size=(nb, 2), dtype=np.uint64)
    pt = rng.integers(0, P61, size=(nb + 9, 2), dtype=np.uint64)
    count = 4 * nb + 3
    u = rng.integers(0, P61, size=(B, count, 2), dtype=np.uint64)
    v = rng.integers(0, P61, size=(B, count, 2), dtype=np.uint64)
    prefixes = [[f, 11] for f in range(B)]
    fs = b"".join(replay_lib(lib, "truepix", [["u64s", p]])[2].raw for p in prefixes)
    vsb = []
    for f in range(B):
        vs = ctypes.create_string_buffer(lib.tp_vole_state_bytes())
        assert lib.tp_vole_state_init(vs, 3 if f != B - 1 else count - 4, None) == 0
        vsb.append(vs.raw)
    d_fs = torch.from_numpy(np.frombuffer(fs, np.uint8).copy()).to(dev)
    vole = dict(states=torch.from_numpy(np.frombuffer(b"".join(vsb), np.uint8).copy()).to(dev),
                u=torch.from_numpy(u.view(np.int64).reshape(-1)).to(dev),
                v=torch.from_numpy(v.view(np.int64).reshape(-1)).to(dev), count=count)
    prover = BatchFrameProver([layout] * B, gt, i0, i1)
    prover.prove(pix, [z1] * B, torch.from_numpy(pack_fp2(z2[:, 0], z2[:, 1])).to(dev).repeat(B),
                 torch.from_numpy(pack_fp2(pt[:, 0], pt[:, 1])).to(dev).repeat(B), None, transcripts=d_fs, vole=vole)
    torch.cuda.synchronize()
    ch = prover.device_challenges.cpu().numpy().view(np.uint64).reshape(nb, B, 2)
    claims = prover.claims.cpu().numpy().view(np.uint64).reshape(nb, B, 4, 2)
    for f in range(B - 1):
        g = {"x_prefix": np.array(prefixes[f], np.uint64), "x_u": u[f], "x_v": v[f], "x_start": np.array([3]),
             "x_prev0": np.zeros(2, np.uint64), "x_has_prev": np.array([0]), "x_claims": claims[:, f]}
        want, _, _, _, used = vole_rounds_python(g, "x")
        np.testing.assert_array_equal(ch[:, f], want)
        assert used == 3 + 4 * nb
    st = vole["states"].cpu().numpy()[(B - 1) * 160:B * 160]
    assert st[12:16].view(np.uint32)[0] == 1       # the last frame ran out after one round
    assert not ch[1:, B - 1].any()


def _random_absorbs(lib, rng, trials):
    """random mixes of raw absorbs, int-list puts and Fp2 puts of many lengths
    (block-boundary cases) through the host entry points, against hashlib"""
    import hashlib
    import struct
    d = ctypes.create_string_buffer(32)
    for trial in range(trials):
        st = ctypes.create_string_buffer(lib.tp_fs_state_bytes())
        assert lib.tp_fs_init(st, b"truepix") == 0
        h = hashlib.sha256(b"TruePix,truepix,binhash1,")
        for _ in range(int(rng.integers(1, 6))):
            n = int(rng.choice([0, 1, 5, 55, 63, 64, 65, 127, 128, 129, 1000, 4096, 9999]))
            kind = int(rng.integers(0, 3))
            if kind == 0:
                b = rng.integers(0, 256, size=n, dtype=np.uint8).tobytes()
                assert lib.tp_fs_absorb(st, b, len(b)) == 0
                h.update(b)
            elif kind == 1 and n:
                v = rng.integers(0, 2 ** 63, size=n, dtype=np.uint64) * np.uint64(2) + np.uint64(1)
                assert lib.tp_fs_put_u64s(st, v.ctypes.data, n) == 0
                h.update(b"\x01" + struct.pack("<I", n) + v.tobytes())
            else:
                re = rng.integers(0, P61, size=n, dtype=np.uint64)
                im = rng.integers(0, P61, size=n, dtype=np.uint64)
                assert lib.tp_fs_put_fp2s(st, re.ctypes.data, im.ctypes.data, n) == 0
                h.update(b"".join(b"\x03" + struct.pack("<QQ", int(a), int(c)) for a, c in zip(re, im)))
        assert lib.tp_fs_digest(st, d) == 0
        assert d.raw == h.digest(), trial


def test_host_bulk_absorb_matches_hashlib(lib):
    """Long absorbs are compressed block by block straight from the caller's
    bytes (with the x86 SHA extensions where the CPU has them): same digests as
    hashlib for every split, and an 8 MiB int list (a frame's circuit outputs are
    64 MiB) in one put."""
    import hashlib
    import struct
    rng = np.random.default_rng(5)
    _random_absorbs(lib, rng, 120)
    a = rng.integers(0, 256, size=1 << 20, dtype=np.uint64)
    st = ctypes.create_string_buffer(lib.tp_fs_state_bytes())
    assert lib.tp_fs_init(st, b"truepix") == 0
    assert lib.tp_fs_put_u64s(st, a.ctypes.data, a.size) == 0
    d = ctypes.create_string_buffer(32)
    assert lib.tp_fs_digest(st, d) == 0
    assert d.raw == hashlib.sha256(b"TruePix,truepix,binhash1,\x01" + struct.pack("<I", a.size) + a.tobytes()).digest()


def test_host_portable_compression_matches_hashlib():
    """the same with the portable compression (TRUEPIX_HOST_SHA_PORTABLE=1), in a
    child process so that the choice is made afresh"""
    import os
    import subprocess
    import sys
    from fslib import ROOT
    code = ("import numpy as np, sys; sys.path[:0] = [%r, %r]\n"
            "from truepix_b200 import native\n"
            "import test_gpu_transcript as t\n"
            "t._random_absorbs(native.gkr(require_device=False), np.random.default_rng(6), 60)\n"
            % (ROOT, os.path.join(ROOT, "tests")))
    env = dict(os.environ, TRUEPIX_HOST_SHA_PORTABLE="1")
    r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
