"""The Orion oracle (oracle/orion_oracle.c) against the reference's own outputs.

tests/golden/orion_golden.npz was produced by the reference sources
(tests/golden/gen_orion_golden.py); these tests pin the C restatement to it so
that the GPU tests may use the oracle as their checker. CPU only.
"""
import ctypes
import hashlib
import os
import subprocess

import numpy as np
import pytest

from orionlib import ORION_ORACLE_LIB, P61, ROOT, OrionOracle, digest, elements

KINDS = ["random", "zero", "max", "small"]


@pytest.fixture(scope="module")
def orc():
    if not os.path.exists(ORION_ORACLE_LIB):
        subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "all"])
    return OrionOracle()


@pytest.fixture(scope="module")
def og():
    return np.load(os.path.join(ROOT, "tests", "golden", "orion_golden.npz"))


def test_sha256_matches_hashlib(orc):
    rng = np.random.default_rng(0)
    for msg in (bytes(64), bytes(range(64)), b"\xff" * 64, rng.bytes(64), rng.bytes(64)):
        assert orc.sha256_64(msg) == hashlib.sha256(msg).digest()


def test_glibc_rand_matches_libc(orc):
    libc = ctypes.CDLL("libc.so.6")
    for seed in (1, 2, 12345):
        libc.srand(seed)
        want = [libc.rand() for _ in range(2000)]
        assert orc.glibc_rand(seed, 2000) == want


def test_commit_roots(orc, og):
    for k in og.files:
        if not k.startswith("commit_"):
            continue
        name = k[len("commit_"):]
        n, seed, kind = (int(v) for v in og["commitcase_" + name])
        root = orc.commit(elements(seed, n, KINDS[kind]))
        assert root == og[k].tobytes(), name


def test_commit_root_hex_format(orc, og):
    # root_hex (truepix_gkr.h) prints h0.hi, h0.lo, h1.hi, h1.lo as %016llx of
    # the little-endian 64-bit words of the digest
    root = og["commit_r13"].tobytes()
    w = np.frombuffer(root, np.uint64)
    hx = "%016x%016x%016x%016x" % (w[1], w[0], w[3], w[2])
    assert hx.encode() == og["commithex_r13"].tobytes()


def test_encode(orc, og):
    for k in og.files:
        if not k.startswith("encode_"):
            continue
        n = int(k.split("_")[1])
        cw = orc.encode(elements(100 + n, n))
        assert cw.size // 2 == int(og["encodelen_%d" % n][0]) == orc.encode_len(n)
        assert digest(cw) == og[k].tobytes(), n
    np.testing.assert_array_equal(orc.encode(elements(164, 64)), og["encodefull_64"])


def test_fft_ifft(orc, og):
    for k in og.files:
        if not k.startswith("fft_"):
            continue
        m, o = (int(v) for v in k.split("_")[1:])
        r = orc.fft(elements(200 + m + o, m), o)
        assert digest(r) == og[k].tobytes(), (m, o)
        ri = orc.ifft(elements(300 + m + o, o), m)
        assert digest(ri) == og["ifft_%d_%d" % (m, o)].tobytes(), (m, o)


def test_fft_then_ifft_is_identity(orc):
    a = elements(9, 1 << 12)
    np.testing.assert_array_equal(orc.ifft(orc.fft(a, 1 << 12), 1 << 12), a)
    # evaluations on a larger domain sub-sample back to the coefficients
    np.testing.assert_array_equal(orc.ifft(orc.fft(a, 1 << 15), 1 << 12), a)


def test_rs_commit(orc, og):
    for k in og.files:
        if not k.startswith("rs_"):
            continue
        lg = int(k.split("_")[1])
        root, cw = orc.rs_commit(elements(400 + lg, 1 << lg), lg, want_codeword=True)
        assert digest(cw) == og["rscw_%d" % lg].tobytes(), lg
        assert root == og[k].tobytes(), lg


def test_elements_are_canonical():
    for kind in KINDS:
        e = elements(3, 1000, kind)
        assert e.dtype == np.uint64 and e.size == 2000 and int(e.max()) < P61


def test_commit_root_of_a_1080p_frame(orc, og):
    from orionlib import frame_bytes, frame_elements
    copies, cs, W, ci, cv, padded, seed = (int(x) for x in og["frame1080"])
    src = frame_elements(frame_bytes(seed, copies * cs), copies, cs, W, ci, cv, padded)
    assert src.size == 2 << 23
    assert orc.commit(src) == og["frameroot_1080"].tobytes()


def test_opening_combine(orc, og):
    for k in og.files:
        if not k.startswith("combinecase_"):
            continue
        n, seed = (int(v) for v in og[k])
        comb, root, ans = orc.combine(elements(seed, n), elements(seed + 1000, 128),
                                      elements(seed + 2000, n // 128))
        assert digest(comb) == og["combine_%d" % n].tobytes(), n
        assert root == og["combineroot_%d" % n].tobytes(), n
        np.testing.assert_array_equal(ans, og["combineanswer_%d" % n])


def test_virgo_update(orc, og):
    from orionlib import virgo_inputs
    for k in og.files:
        if not k.startswith("virgocase_"):
            continue
        phase, n, bit, seed = (int(v) for v in og[k])
        key = k[len("virgocase_"):]
        vma, addv, ams, r = virgo_inputs(n, seed)
        outs, ret = orc.virgo_update(vma, addv, ams, r, bit)
        assert b"".join(digest(o) for o in outs) == og["virgotables_" + key].tobytes(), key
        np.testing.assert_array_equal(ret, og["virgoret_" + key])


def test_fri_step(orc, og):
    for k in og.files:
        if not k.startswith("fricase_"):
            continue
        lm, seed = (int(v) for v in og[k])
        nxt, root = orc.fri_step(elements(seed, (1 << lm) * 64), lm, elements(seed + 1, 1))
        assert digest(nxt) == og["frinext_%d" % lm].tobytes(), lm
        assert root == og["friroot_%d" % lm].tobytes(), lm


@pytest.fixture(scope="module")
def zg():
    return np.load(os.path.join(ROOT, "tests", "golden", "orion_zk_golden.npz"))


def zk_cases(zg, largest=True):
    for k in sorted(zg.files):
        if k.startswith("zkcase_"):
            name = k[len("zkcase_"):]
            copies, cs, ci, cv, padded, pseed = (int(x) for x in zg[k])
            if not largest and copies > 4096:
                continue
            yield name, (copies, cs, ci, cv, padded, pseed, int(zg["zkseed_" + name][0]))


def test_zk_commit_pair_and_mask(orc, zg):
    """The ZK commit phase (Orion_zk commit_pair of the masked polynomial and the
    mask drawn from the seed) against the reference's roots and mask."""
    from orionlib import frame_bytes
    for name, (copies, cs, ci, cv, padded, pseed, mseed) in zk_cases(zg):
        pix = frame_bytes(pseed, copies * cs)
        mask = orc.frame_vector(pix, copies, cs, 512, ci, cv, padded, mseed, 2)
        words = np.zeros(2 * mask.size, np.uint64)
        words[1::2] = mask
        assert digest(words) == zg["zkmaskdigest_" + name].tobytes(), name
        plain = orc.frame_vector(pix, copies, cs, 512, ci, cv, padded, mseed, 0)
        masked = orc.frame_vector(pix, copies, cs, 512, ci, cv, padded, mseed, 1)
        assert np.array_equal(masked, (plain + mask) % np.uint64(P61)), name
        ra, rb = orc.zk_commit(pix, copies, cs, 512, ci, cv, padded, mseed)
        assert ra == zg["zkmasked_" + name].tobytes(), name
        assert rb == zg["zkmask_" + name].tobytes(), name


def test_zk_mask_only_hides_private_wires(orc):
    from orionlib import frame_bytes
    pix = frame_bytes(1, 5 * 384)
    m = orc.frame_vector(pix, 5, 384, 512, 384, 128, 8, 77, 2).reshape(8, 512)
    assert not m[:, 384:].any() and not m[5:].any()
    assert m[:5, :384].all()       # a zero draw has probability ~2^-50 here


def test_virgo_layer_inits(orc):
    """sumcheck_phase1_init / phase2_init restated (every gate type) against the
    reference's tables (digests in tests/golden/virgo_init_golden.npz)."""
    from orionlib import virgo_layer
    g = np.load(os.path.join(ROOT, "tests", "golden", "virgo_init_golden.npz"))
    n = 0
    for k in g.files:
        if not k.startswith("vinitcase_"):
            continue
        phase, seed, lg, lu = (int(x) for x in g[k])
        outs = orc.virgo_init(phase, virgo_layer(seed, lg, lu))
        assert b"".join(digest(o) for o in outs) == g["vinit_" + k[len("vinitcase_"):]].tobytes(), k
        n += 1
    assert n >= 12


def test_virgo_init_rejects_out_of_range_gates(orc):
    from orionlib import virgo_layer
    L = virgo_layer(3, 4, 4, types=(0,))
    L["u"][5] = 1 << 4
    with pytest.raises(ValueError):
        orc.virgo_init(1, L)
