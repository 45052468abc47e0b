"""The late-round CTA's code (late::run_frame, truepix_b200/csrc/late.cuh) run
on the CPU by tests/late_host_emu.cu, a host loop over the CTA's thread indices
with a barrier between steps, against the fixtures made by the reference:
given challenges (tests/golden/late_golden.npz, the reference LayerProver) and
the VOLE-committed rounds with the layer's closing proofs (tests/golden/
layer_vole_golden.npz, the reference prover's own proof methods). The device
kernel runs the same steps; tests/test_gpu_late.py checks it on the GPU."""
import ctypes
import os
import shutil
import subprocess

import numpy as np
import pytest

from latelib import golden_cases

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
P = lambda a: ctypes.c_void_p(a.ctypes.data)


def u64(a):
    return np.ascontiguousarray(np.asarray(a, np.uint64).reshape(-1))


@pytest.fixture(scope="module")
def emu(tmp_path_factory):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not available")
    out = str(tmp_path_factory.mktemp("late_emu") / "late_host_emu.so")
    # -O2 with strict aliasing on: the host build follows the same type rules
    # as the device compiler
    subprocess.run([nvcc, "-O2", "-std=c++17", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC,-fstrict-aliasing",
                    "-shared", "-Wno-deprecated-gpu-targets", "-o", out,
                    os.path.join(ROOT, "tests", "late_host_emu.cu")], check=True)
    lib = ctypes.CDLL(out)
    lib.emu_late_frame.restype = ctypes.c_int
    return lib


def run(emu, c, n, gates, chal=None, st=None, vs=None, uv=None, round0=0, close=None):
    gt, i0, i1 = (np.ascontiguousarray(r, np.int32) for r in gates)
    wires, beta, zg = u64(c["wires"]), u64(c["beta"]), u64(c["zg"])
    coefs, line, cho = np.zeros(12 * n, np.uint64), np.zeros(2 * (n + 1), np.uint64), np.zeros(4 * n, np.uint64)
    proof = np.zeros(16 * n, np.uint64)
    nb = round0
    closing, point, tag = np.zeros(2 * (n + 10), np.uint64), np.zeros(2 * (n + nb), np.uint64), np.zeros(2, np.uint64)
    z2 = u64(close[0]) if close else np.zeros(2, np.uint64)
    w3 = u64(close[1]) if close else np.zeros(2, np.uint64)
    u, v = (u64(uv[0]), u64(uv[1])) if uv else (np.zeros(2, np.uint64), np.zeros(2, np.uint64))
    ch = u64(chal) if chal is not None else None
    rc = emu.emu_late_frame(n, gt.size, P(gt), P(i0), P(i1), P(wires), P(beta), P(zg),
                            P(ch) if ch is not None else None, st, vs, P(u), P(v),
                            ctypes.c_longlong(len(u) // 2 if uv else 0), 0, round0, P(coefs), P(line), P(cho),
                            P(proof) if ch is None else None, P(z2), P(w3), P(closing) if close else None, P(point),
                            P(tag), 0)
    assert rc == 0
    return dict(coefs=coefs.reshape(-1, 2), line=line.reshape(-1, 2), chal=cho.reshape(-1, 2),
                proof=proof.reshape(2 * n, 4, 2), closing=closing.reshape(-1, 2), point=point.reshape(-1, 2),
                tag=tag.reshape(-1, 2))


def test_given_challenges_match_reference_layer_prover(emu):
    n_cases = 0
    for c in golden_cases():
        n, nb = c["n_in_bits"], c["n_copy_bits"]
        r = run(emu, c, n, c["gates"], chal=c["chal"][nb:])
        np.testing.assert_array_equal(r["coefs"], c["late"], err_msg=c["name"])
        np.testing.assert_array_equal(r["line"], c["final"], err_msg=c["name"])
        np.testing.assert_array_equal(r["chal"], c["chal"][nb:])
        n_cases += 1
    assert n_cases == 6


def test_vole_rounds_and_closing_match_reference_chain(emu):
    from layervole import cases, early_transcript, vole_state_fields, vole_state_mid
    from truepix_b200 import native
    lib = native.gkr(require_device=False)   # its host transcript only
    n_cases = 0
    for c in cases():
        n, nb = c["n_in_bits"], c["nb"]
        for close in (False, True):
            st, ch = early_transcript(lib, c)
            assert [list(x) for x in ch] == [[int(a), int(b)] for a, b in c["chal"][:nb]]
            vs = ctypes.create_string_buffer(vole_state_mid(c), 160)
            r = run(emu, c, n, c["gates"], st=st, vs=vs, uv=(c["u"], c["v"]), round0=nb,
                    close=(c["z2"], c["chal"][:nb]) if close else None)
            np.testing.assert_array_equal(r["coefs"], c["coefs"][4 * nb:])
            np.testing.assert_array_equal(r["chal"], c["chal"][nb:])
            np.testing.assert_array_equal(r["proof"][:, :3].reshape(-1, 2), c["d"][4 * nb:])
            np.testing.assert_array_equal(r["proof"][:, 3], c["vz"][nb:])
            np.testing.assert_array_equal(r["line"], c["final"])
            f = vole_state_fields(vs.raw)
            d = ctypes.create_string_buffer(32)
            assert lib.tp_fs_digest(st.raw, d) == 0
            if not close:
                assert f["idx"] == int(c["used"][0]) and f["bad"] == 0 and f["has_prev"] == 1
                assert f["prev"] == tuple(int(x) for x in c["prev"][0])
                assert f["v_elem"] == [tuple(int(x) for x in r_) for r_ in c["v_elem"]]
                assert f["out_elem"] == [tuple(int(x) for x in r_) for r_ in c["out_elem"]]
                assert d.raw == c["digest"].tobytes()
            else:
                rows = [k for k in range(n + 10) if not np.array_equal(r["closing"][k], c["closing"][k])]
                assert not rows, f"{c['name']}: closing rows {rows} differ"
                np.testing.assert_array_equal(r["point"], c["point"])
                np.testing.assert_array_equal(r["tag"], c["tag"])
                assert f["idx"] == int(c["used_closed"][0])
                assert d.raw == c["digest_closed"].tobytes()
        n_cases += 1
    assert n_cases == 2
