"""The process boundaries on the CPU (no GPU here): the programs in
truepix_b200/bin are built and linked to the in-tree library; they refuse bad
arguments, environments and files with the reference programs' own messages
(compared with oracle/_ref's builds of examples/multivariate_PC_test_*.cpp where
present) and fail loudly, before any work, when no CUDA device is present; the
fft_gkr fixture is pinned to the reference source's harness."""
import json
import os
import subprocess

import numpy as np
import pytest

from clilib import env_for, first_error, lay_out, manifest, ours, reference, run

PROGS = ("linearPC_multi_commit", "linearPC_multi_prove", "linearPC_multi_open")
ZK = tuple(p + "_zk" for p in PROGS)
HERE = os.path.dirname(os.path.abspath(__file__))


def test_programs_are_built_against_the_in_tree_library():
    lib = os.path.realpath(os.path.join(HERE, "..", "truepix_b200", "lib", "libnative_fp2_gpu.so"))
    for name in PROGS + ZK + ("fft_gkr",):
        path = ours(name)
        assert os.access(path, os.X_OK), path
        out = subprocess.run(["ldd", path], capture_output=True, text=True).stdout
        line = [ln for ln in out.splitlines() if "libnative_fp2_gpu.so" in ln]
        assert line and os.path.realpath(line[0].split("=>")[1].split()[0]) == lib, out


def _frame(copies=4, cs=384):
    rng = np.random.default_rng(7)
    return rng.integers(0, 256, size=copies * cs, dtype=np.uint8)


# (program index, argv, env overrides, files) -> both reject with the same first message
CASES = [
    (0, [], {}, "input"),
    (0, ["x", "0"], {}, "input"),
    (1, ["4", "2"], {}, "input"),
    (0, ["4", "1"], {}, "input"),
    (0, ["4", "0"], {"TRUEPIX_CONST_IDX": "5"}, "input"),
    (0, ["4", "0"], {"TRUEPIX_COPY_SIZE": "600"}, "input"),
    (0, ["4", "0"], {}, "short_line"),
    (0, ["4", "0"], {}, "negative"),
    (0, ["4", "0"], {}, "few_lines"),
    (1, ["4", "0"], {}, "input"),                 # no manifest
    (1, ["4", "0"], {}, "zk_manifest"),
    (2, ["4", "0"], {}, "other_layout"),
    (1, ["4", "0"], {}, "no_point"),
    (2, ["4", "0"], {}, "bad_point"),
    (1, ["4", "0"], {"TRUEPIX_GKR_POINT_FILE": "/nonexistent/p.json"}, "manifest"),
    (4, ["4", "0"], {}, "manifest"),              # zero-knowledge program, plain manifest
    (5, ["4", "0"], {}, "zk_manifest"),           # no mask seed file
    (4, ["4", "0"], {}, "zk_seed_no_point"),
    (5, ["4", "0"], {"TRUEPIX_CONST_IDX": "5"}, "input"),
    (4, ["4", "1"], {}, "input"),
]
ALL = PROGS + ZK


def _files(d, kind):
    pix = _frame()
    lg = 11
    point = [(3, 4)] * lg
    if kind == "short_line":
        with open(os.path.join(d, "input.txt"), "w") as fh:
            fh.write("1 2 3\n")
        return
    if kind == "negative":
        lay_out(d, pix, 4, 384)
        txt = open(os.path.join(d, "input.txt")).read().split("\n")
        txt[1] = "-1 " + txt[1]
        open(os.path.join(d, "input.txt"), "w").write("\n".join(txt))
        return
    if kind == "few_lines":
        lay_out(d, pix[:2 * 384], 2, 384)
        return
    m = None
    if kind in ("manifest", "no_point", "bad_point"):
        m = manifest(4, 384, 384, 128, "00" * 32)
    elif kind in ("zk_manifest", "zk_seed_no_point"):
        m = manifest(4, 384, 384, 128, "00" * 32, zk=True)
        if kind == "zk_seed_no_point":
            open(os.path.join(d, "orion_mask_seed.txt"), "w").write("12345\n")
    elif kind == "other_layout":
        m = manifest(8, 384, 384, 128, "00" * 32)
    if kind == "bad_point":
        point = [(3, 4)] * (lg - 1)
    lay_out(d, pix, 4, 384, None if kind in ("no_point", "zk_seed_no_point") else point, m)


@pytest.mark.parametrize("k", range(len(CASES)))
def test_refusals_match_the_reference_programs(k, tmp_path):
    idx, argv, extra, kind = CASES[k]
    if not os.path.exists(reference(PROGS[1])):
        pytest.skip("oracle/_ref reference programs not built")
    got = {}
    if not os.path.exists(reference(ALL[idx])):
        pytest.skip("reference program missing")
    for who, path in (("ours", ours(ALL[idx])), ("ref", reference(ALL[idx]))):
        d = tmp_path / who
        d.mkdir()
        _files(str(d), kind)
        env = env_for(str(d), 384, 384, 128, **extra)
        if kind in ("no_point", "zk_seed_no_point"):
            env.pop("TRUEPIX_GKR_POINT_FILE")
        r = run(path, str(d), env, *argv, timeout=60)
        got[who] = (r.returncode != 0, first_error(r).replace(path, "PROG"))
    assert got["ours"] == got["ref"], got


def test_no_device_fails_loudly(tmp_path):
    """valid inputs, no GPU: each program stops with a message and status 1"""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    for names, zk in ((PROGS, False), (ZK, True)):
        d = str(tmp_path / str(zk))
        os.makedirs(d)
        lay_out(d, _frame(), 4, 384, [(3, 4)] * 11, manifest(4, 384, 384, 128, "00" * 32, zk=zk))
        open(os.path.join(d, "orion_mask_seed.txt"), "w").write("12345\n")
        env = env_for(d, 384, 384, 128)
        for name in names:
            r = run(ours(name), d, env, 4, 0, timeout=60)
            assert r.returncode == 1 and "no CUDA device" in r.stderr, (name, r.stdout, r.stderr)
            assert not [f for f in os.listdir(d) if f.endswith(".bin")]
    d = str(tmp_path)
    env = env_for(d, 384, 384, 128)
    r = run(ours("fft_gkr"), d, env, 4, os.path.join(d, "out.txt"), timeout=60)
    assert r.returncode == 1 and r.stderr.startswith("fft_gkr: ") and not os.path.exists(os.path.join(d, "out.txt"))


def test_fft_gkr_fixture_is_the_reference_harness_output():
    """tests/golden/fft_gkr_golden.json against oracle/_ref/fft_gkr_harness (the
    reference source compiled with the harness), when built here"""
    import sys
    sys.path.insert(0, os.path.join(HERE, "golden"))
    from gen_fft_gkr_golden import split
    g = json.load(open(os.path.join(HERE, "golden", "fft_gkr_golden.json")))
    harness = reference("fft_gkr_harness")
    if not os.path.exists(harness):
        pytest.skip("oracle/_ref/fft_gkr_harness not built")
    for lg in ("0", "3", "6", "10"):
        tr = subprocess.run([harness, lg], check=True, capture_output=True, text=True).stdout
        assert split(tr) == {k: v for k, v in g[lg].items() if k != "program_proof_size"}, lg
    for lg, rec in g.items():
        assert "result 1" in rec["lines"]
        assert rec["program_proof_size"] == int(rec["lines"][-1].split()[1])
