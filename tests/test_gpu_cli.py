"""The process boundaries on the device.

./fft_gkr (truepix_b200/bin/fft_gkr, the device GKR of the reference's
src/VPD/fft_circuit_GKR.cpp): every claim, the last sumcheck tables, every
circuit layer (lg <= 6) and the proof size equal the reference's own run
(tests/golden/fft_gkr_golden.json, made by the reference source's harness);
and the reference's linearPC_multi_prove runs with it as its ./fft_gkr.

linearPC_multi_{commit,prove,open} (truepix_b200/bin, one source over the
library): on the plain frames of tests/golden/opening_golden.npz the manifest's
root is the reference program's, orion_proof.bin is byte-identical to the one
the reference's linearPC_multi_prove wrote, our open accepts it and reports the
opening value, the reference's own linearPC_multi_open (oracle/_ref, where
present) accepts our file, and both reject the same tampered files with the same
first message. The zero-knowledge programs (TruePix's default) against the
reference's prove_zk and open_zk, and inputs beyond a byte against the reference's
prove programs."""
import json
import os
import struct
import sys

import numpy as np
import pytest

from clilib import env_for, first_error, lay_out, manifest, ours, reference, run, sha256_file
from test_opening_host import cases

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))


def _split(trace: str) -> dict:
    sys.path.insert(0, os.path.join(HERE, "golden"))
    from gen_fft_gkr_golden import split
    return split(trace)


def test_fft_gkr_matches_the_reference_run(tmp_path):
    g = json.load(open(os.path.join(HERE, "golden", "fft_gkr_golden.json")))
    for lg, want in g.items():
        out, tr = str(tmp_path / ("o%s.txt" % lg)), str(tmp_path / ("t%s.txt" % lg))
        r = run(ours("fft_gkr"), str(tmp_path), dict(os.environ), lg, out, tr, timeout=120)
        assert r.returncode == 0 and "failed" not in r.stderr, (lg, r.stderr)
        got = _split(open(tr).read())
        assert got["layers"] == want["layers"], lg
        for a, b in zip(got["lines"], want["lines"]):
            assert a == b, (lg, a, b)
        assert len(got["lines"]) == len(want["lines"])
        v_time, proof_size, p_time = open(out).read().split()
        assert int(proof_size) == want["program_proof_size"] and float(v_time) >= 0 and float(p_time) > 0


def test_fft_gkr_rejects_sizes_out_of_range(tmp_path):
    for lg in ("-1", "21"):
        r = run(ours("fft_gkr"), str(tmp_path), dict(os.environ), lg, str(tmp_path / "o.txt"), timeout=60)
        assert r.returncode == 1 and "outside" in r.stderr


def _plain_cases():
    for c in cases():
        copies, cs, ci, cv, seed = json.loads(c["layout"].tobytes().decode())
        if seed is None:
            yield c, copies, cs, ci, cv


def _root_hex(root: bytes) -> str:
    w = struct.unpack("<4Q", root)
    return "".join("%016x" % w[i] for i in (1, 0, 3, 2))


def test_orion_programs_match_the_reference(tmp_path):
    n = 0
    for c, copies, cs, ci, cv in _plain_cases():
        d = str(tmp_path / c["name"])
        os.makedirs(d)
        lay_out(d, c["pix"], copies, cs, [(int(a), int(b)) for a, b in c["point"]])
        env = env_for(d, cs, ci, cv, TRUEPIX_ORION_RESULT_FILE=os.path.join(d, "result.json"))
        r = run(ours("linearPC_multi_commit"), d, env, copies, 0)
        assert r.returncode == 0 and "Commit time" in r.stdout, r.stderr
        m = json.load(open(os.path.join(d, "orion_commit.json")))
        assert m["masked_root"] == _root_hex(c["com_root"].tobytes()) and m["zk"] is False
        assert m == manifest(copies, cs, ci, cv, m["masked_root"])
        r = run(ours("linearPC_multi_prove"), d, env, copies, 0)
        assert r.returncode == 0 and "check pass" in r.stdout and "Open time" in r.stdout, r.stdout + r.stderr
        assert "Proof size for tensor IOP" in r.stdout and "Verification time" in r.stdout
        path = os.path.join(d, "orion_proof.bin")
        assert os.path.getsize(path) == int(c["size"][0])
        assert sha256_file(path) == c["sha256"].tobytes(), c["name"]
        r = run(ours("linearPC_multi_open"), d, env, copies, 0)
        assert r.returncode == 0 and "check pass" in r.stdout and "succ" in r.stdout, r.stdout + r.stderr
        res = json.load(open(os.path.join(d, "result.json")))
        im, re = (int(x) for x in c["answer"][0])
        assert res == {"ok": True, "value": [re, im]}
        if os.path.exists(reference("linearPC_multi_open")):
            os.remove(os.path.join(d, "result.json"))
            os.symlink(ours("fft_gkr"), os.path.join(d, "fft_gkr"))   # its EC(y1) check runs ./fft_gkr
            rr = run(reference("linearPC_multi_open"), d, env, copies, 0)
            assert rr.returncode == 0 and "check pass" in rr.stdout, rr.stdout[-2000:] + rr.stderr[-2000:]
            assert json.load(open(os.path.join(d, "result.json"))) == res
        n += 1
    assert n == 2


def test_reference_prove_runs_with_our_fft_gkr(tmp_path):
    """the reference's linearPC_multi_prove, whose verifier self-check runs
    ./fft_gkr from its working directory, with ours there: same proof bytes"""
    if not os.path.exists(reference("linearPC_multi_prove")):
        pytest.skip("oracle/_ref/linearPC_multi_prove not built")
    c, copies, cs, ci, cv = next(_plain_cases())
    d = str(tmp_path)
    lay_out(d, c["pix"], copies, cs, [(int(a), int(b)) for a, b in c["point"]],
            manifest(copies, cs, ci, cv, _root_hex(c["com_root"].tobytes())))
    os.symlink(ours("fft_gkr"), os.path.join(d, "fft_gkr"))
    r = run(reference("linearPC_multi_prove"), d, env_for(d, cs, ci, cv), copies, 0)
    assert r.returncode == 0 and "check pass" in r.stdout, r.stdout[-3000:] + r.stderr[-2000:]
    assert "Error, fft gkr failed" not in r.stdout + r.stderr
    v_time, proof_size, p_time = open(os.path.join(d, "log_fftgkr.txt")).read().split()
    assert int(proof_size) > 0
    assert sha256_file(os.path.join(d, "orion_proof.bin")) == c["sha256"].tobytes()


# tampered proof files: (what, byte offset from a field, new bytes)
def _tamper(proof: bytes, kind: str) -> bytes:
    b = bytearray(proof)
    qc = struct.unpack_from("<I", b, 8 + 8 + 32)[0]
    msg_len, cw_len = struct.unpack_from("<QQ", b, 8 + 8 + 16)
    off_ans = 8 + 8 + 36
    off_q = off_ans + 16 + 64
    off_cols = off_q + 8 * qc
    off_comb = off_cols + 16 * 128 * qc
    off_msg = off_comb + 16 * cw_len
    off_sparse = off_msg + 16 * msg_len
    if kind == "answer":
        b[off_ans + 8] ^= 1
    elif kind == "query":
        q = struct.unpack_from("<q", b, off_q + 8 * 5)[0]
        struct.pack_into("<q", b, off_q + 8 * 5, (q + 1) % cw_len)
    elif kind == "column":
        b[off_cols + 16 * (128 * 7 + 3) + 8] ^= 4
    elif kind == "sibling":
        b[off_sparse + 8 + 4 + 5] ^= 1
    elif kind == "message":
        b[off_msg + 16 * 3 + 8] ^= 2
    elif kind == "root":
        b[off_ans + 16 + 3] ^= 1
    elif kind == "truncated":
        del b[len(b) - 10:]
    return bytes(b)


@pytest.mark.parametrize("kind", ["answer", "query", "column", "sibling", "message", "root", "truncated"])
def test_open_rejects_tampered_proofs_like_the_reference(tmp_path, kind):
    c, copies, cs, ci, cv = next(_plain_cases())
    d = str(tmp_path)
    lay_out(d, c["pix"], copies, cs, [(int(a), int(b)) for a, b in c["point"]])
    env = env_for(d, cs, ci, cv)
    assert run(ours("linearPC_multi_commit"), d, env, copies, 0).returncode == 0
    assert run(ours("linearPC_multi_prove"), d, env, copies, 0).returncode == 0
    path = os.path.join(d, "orion_proof.bin")
    good = open(path, "rb").read()
    open(path, "wb").write(_tamper(good, kind))
    r = run(ours("linearPC_multi_open"), d, env, copies, 0)
    assert r.returncode == 1 and "check notpass" in r.stdout, (kind, r.stdout, r.stderr)
    if os.path.exists(reference("linearPC_multi_open")):
        os.symlink(ours("fft_gkr"), os.path.join(d, "fft_gkr"))
        rr = run(reference("linearPC_multi_open"), d, env, copies, 0)
        assert rr.returncode == 1
        assert first_error(r) == first_error(rr), (kind, r.stderr, rr.stderr)


def _zk_case():
    for c in cases():
        copies, cs, ci, cv, seed = json.loads(c["layout"].tobytes().decode())
        if seed is not None:
            return c, copies, cs, ci, cv, seed
    raise AssertionError("no zero-knowledge case")


def test_zk_programs_match_the_reference(tmp_path):
    """the Orion_zk programs (TruePix's default): with the fixture's mask seed the
    two opening files are byte-identical to the reference program's; our open
    accepts them and reports masked - mask = the plaintext MLE; the reference's
    open accepts our files"""
    c, copies, cs, ci, cv, seed = _zk_case()
    d = str(tmp_path)
    m = manifest(copies, cs, ci, cv, _root_hex(c["com_root"].tobytes()), zk=True)
    m["mask_root"] = _root_hex(c["mask_com_root"].tobytes())
    lay_out(d, c["pix"], copies, cs, [(int(a), int(b)) for a, b in c["point"]], m)
    with open(os.path.join(d, "orion_mask_seed.txt"), "w") as fh:
        fh.write("%d\n" % seed)
    env = env_for(d, cs, ci, cv, TRUEPIX_ORION_RESULT_FILE=os.path.join(d, "result.json"))
    r = run(ours("linearPC_multi_prove_zk"), d, env, copies, 0)
    assert r.returncode == 0 and "check pass" in r.stdout and "Commit time(mask)" in r.stdout, r.stdout + r.stderr
    for tag, name in (("", "orion_proof_masked.bin"), ("mask_", "orion_proof_mask.bin")):
        assert sha256_file(os.path.join(d, name)) == c[tag + "sha256"].tobytes(), name
    r = run(ours("linearPC_multi_open_zk"), d, env, copies, 0)
    assert r.returncode == 0 and "check pass" in r.stdout, r.stdout + r.stderr
    ours_res = json.load(open(os.path.join(d, "result.json")))
    assert ours_res["ok"] is True
    if os.path.exists(reference("linearPC_multi_open_zk")):
        os.remove(os.path.join(d, "result.json"))
        os.symlink(ours("fft_gkr"), os.path.join(d, "fft_gkr"))
        rr = run(reference("linearPC_multi_open_zk"), d, env, copies, 0)
        assert rr.returncode == 0 and "check pass" in rr.stdout, rr.stdout[-2000:] + rr.stderr[-2000:]
        assert json.load(open(os.path.join(d, "result.json"))) == ours_res


def test_zk_commit_prove_open_round_trip(tmp_path):
    """a fresh commit (seed from /dev/urandom, written to the seed file), then
    prove and open; the reference's prove with the same seed writes the same files"""
    c, copies, cs, ci, cv, _ = _zk_case()
    d = str(tmp_path / "ours")
    os.makedirs(d)
    lay_out(d, c["pix"], copies, cs, [(int(a), int(b)) for a, b in c["point"]])
    env = env_for(d, cs, ci, cv)
    r = run(ours("linearPC_multi_commit_zk"), d, env, copies, 0)
    assert r.returncode == 0 and "Commit time(mask)" in r.stdout, r.stderr
    m = json.load(open(os.path.join(d, "orion_commit.json")))
    assert m["zk"] is True and len(m["masked_root"]) == 64 and len(m["mask_root"]) == 64
    assert run(ours("linearPC_multi_prove_zk"), d, env, copies, 0).returncode == 0
    r = run(ours("linearPC_multi_open_zk"), d, env, copies, 0)
    assert r.returncode == 0 and "check pass" in r.stdout, r.stdout + r.stderr
    if os.path.exists(reference("linearPC_multi_prove_zk")):
        e = str(tmp_path / "ref")
        os.makedirs(e)
        for f in ("input.txt", "gkr_point_prover.txt", "orion_commit.json", "orion_mask_seed.txt"):
            with open(os.path.join(d, f)) as src, open(os.path.join(e, f), "w") as dst:
                dst.write(src.read())
        os.symlink(ours("fft_gkr"), os.path.join(e, "fft_gkr"))
        rr = run(reference("linearPC_multi_prove_zk"), e, env_for(e, cs, ci, cv), copies, 0)
        assert rr.returncode == 0 and "check pass" in rr.stdout, rr.stdout[-2000:] + rr.stderr[-2000:]
        for name in ("orion_proof_masked.bin", "orion_proof_mask.bin"):
            assert sha256_file(os.path.join(d, name)) == sha256_file(os.path.join(e, name)), name


@pytest.mark.parametrize("zk", [False, True])
def test_programs_take_values_above_255(tmp_path, zk):
    """input.txt values beyond a byte (the element-vector path of the commits):
    our commit, prove and open agree with each other, and the reference's prove
    program, given our manifest (and seed), passes its root check and writes the
    same opening files"""
    if not os.path.exists(reference("linearPC_multi_prove" + ("_zk" if zk else ""))):
        pytest.skip("oracle/_ref reference programs not built")
    rng = np.random.default_rng(21)
    copies, cs, ci, cv = 64, 384, 384, 128
    vals = rng.integers(0, 5000, size=copies * cs, dtype=np.int64)
    point = [(int(a), int(b)) for a, b in rng.integers(0, (1 << 61) - 1, size=(15, 2), dtype=np.uint64)]
    sfx = "_zk" if zk else ""
    d, e = str(tmp_path / "ours"), str(tmp_path / "ref")
    os.makedirs(d)
    os.makedirs(e)
    lay_out(d, vals, copies, cs, point)
    env = env_for(d, cs, ci, cv)
    r = run(ours("linearPC_multi_commit" + sfx), d, env, copies, 0)
    assert r.returncode == 0, r.stderr
    r = run(ours("linearPC_multi_prove" + sfx), d, env, copies, 0)
    assert r.returncode == 0 and "check pass" in r.stdout, r.stdout + r.stderr
    r = run(ours("linearPC_multi_open" + sfx), d, env, copies, 0)
    assert r.returncode == 0 and "check pass" in r.stdout, r.stdout + r.stderr
    for f in ("input.txt", "gkr_point_prover.txt", "orion_commit.json") + (("orion_mask_seed.txt",) if zk else ()):
        with open(os.path.join(d, f)) as src, open(os.path.join(e, f), "w") as dst:
            dst.write(src.read())
    os.symlink(ours("fft_gkr"), os.path.join(e, "fft_gkr"))
    rr = run(reference("linearPC_multi_prove" + sfx), e, env_for(e, cs, ci, cv), copies, 0)
    assert rr.returncode == 0 and "check pass" in rr.stdout, rr.stdout[-2000:] + rr.stderr[-2000:]
    for name in (("orion_proof_masked.bin", "orion_proof_mask.bin") if zk else ("orion_proof.bin",)):
        assert sha256_file(os.path.join(d, name)) == sha256_file(os.path.join(e, name)), name
