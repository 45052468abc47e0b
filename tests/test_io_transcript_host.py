"""The prover's IO transcript put of a frame's circuit outputs computed on the
host from the frame's bytes (tp_fs_put_circuit_outputs_pixels): the transcript
state after it equals the state after put(output vector) of the vector the
reference's circuit evaluator writes (the golden vectors of tests/golden/
circuit_outputs_golden.npz, and the oracle's restatement for larger frames),
for several frames at once, at equal and unequal offsets in the pending block,
in groups of up to 16, with the AVX-512 multi-buffer compression, the x86 SHA
extensions and the portable compression."""
import ctypes
import os
import subprocess
import sys

import numpy as np
import pytest

from circuitlib import golden_cases, oracle_outputs

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _lib():
    from truepix_b200 import native
    return native.gkr(require_device=False)


def _state(lib, prefix: bytes = b""):
    st = ctypes.create_string_buffer(lib.tp_fs_state_bytes())
    assert lib.tp_fs_init(st, b"truepix") == 0
    if prefix:
        assert lib.tp_fs_absorb(st, prefix, len(prefix)) == 0
    return st


def _put_fused(lib, states, frames, c):
    gt, i0, i1 = (np.ascontiguousarray(c[k], np.int32) for k in ("gt", "i0", "i1"))
    pix = [np.ascontiguousarray(f, np.uint8) for f in frames]
    st_arr = (ctypes.c_void_p * len(states))(*[ctypes.cast(s, ctypes.c_void_p) for s in states])
    px_arr = (ctypes.c_void_p * len(pix))(*[p.ctypes.data for p in pix])
    ip = ctypes.POINTER(ctypes.c_int)
    n_bytes = min(f.size for f in pix)
    return lib.tp_fs_put_circuit_outputs_pixels(st_arr, px_arr, n_bytes, len(states), c["copies"], c["padded"], c["cs"],
                                                c["n_wires"], c["const_idx"], c["const_val"], gt.size,
                                                gt.ctypes.data_as(ip), i0.ctypes.data_as(ip), i1.ctypes.data_as(ip))


def _key(st):
    """the part of a state that enters any later hash: chaining words, the pending
    bytes, byte count, draw counter (bytes of the block buffer past the pending
    ones are stale and never hashed)"""
    import struct
    raw = st.raw
    total, rnum, nbuf = struct.unpack_from("<QQI", raw, 96)
    return raw[:32], raw[32:32 + nbuf], total, rnum, nbuf


def _put_vector(lib, st, vec):
    vec = np.ascontiguousarray(vec, np.uint64)
    assert lib.tp_fs_put_u64s(st, vec.ctypes.data, vec.size) == 0


def _frame_case(name, copies, padded, cs, n_wires, ci, cv, seed):
    c = np.load(os.path.join(ROOT, "tests", "golden", "circuits.npz"))
    rng = np.random.default_rng(seed)
    return dict(name=name, copies=copies, padded=padded, cs=cs, n_wires=n_wires, const_idx=ci, const_val=cv,
                gt=c[name + "_type"], i0=c[name + "_in0"], i1=c[name + "_in1"],
                pix=rng.integers(0, 256, size=copies * cs, dtype=np.uint8))


def _cases():
    for c in golden_cases():
        yield c, [c["pix"]], c["out"]
    # larger frames of the four circuits (gray / inv with the constant, mask without, crop with 385 inputs)
    for name, cs, ci, cv in (("gray", 384, 384, 128), ("inv", 384, 384, 255), ("mask", 384, -1, 0),
                             ("Crop", 385, -1, 0)):
        c = _frame_case(name, 300, 512, cs, 512, ci, cv, 7)
        frames = [c["pix"], np.random.default_rng(8).integers(0, 256, size=c["pix"].size, dtype=np.uint8)]
        yield c, frames, None


def test_fused_put_matches_put_of_the_output_vector():
    lib = _lib()
    n = 0
    for c, frames, out in _cases():
        # the same prefix for every frame: the lockstep pairs
        sts = [_state(lib, b"prefix") for _ in frames]
        assert _put_fused(lib, sts, frames, c) == 0, lib.tp_last_error()
        for f, frame in enumerate(frames):
            vec = out if out is not None else oracle_outputs(frame, c["copies"], c["padded"], c["cs"], c["n_wires"],
                                                             c["const_idx"], c["const_val"], c["gt"], c["i0"],
                                                             c["i1"])
            want = _state(lib, b"prefix")
            _put_vector(lib, want, vec)
            assert _key(sts[f]) == _key(want), (c["name"], f)
        n += 1
    assert n >= 5


def test_unequal_offsets_and_three_frames():
    """frames whose transcripts stand at different offsets hash alone; a third
    frame of a group of three pairs with none"""
    lib = _lib()
    c = _frame_case("gray", 200, 256, 384, 512, 384, 128, 11)
    rng = np.random.default_rng(12)
    frames = [rng.integers(0, 256, size=c["pix"].size, dtype=np.uint8) for _ in range(3)]
    prefixes = [b"a", b"bb" * 17, b"a"]
    sts = [_state(lib, p) for p in prefixes]
    assert _put_fused(lib, sts, frames, c) == 0
    for f in range(3):
        want = _state(lib, prefixes[f])
        _put_vector(lib, want, oracle_outputs(frames[f], c["copies"], c["padded"], c["cs"], c["n_wires"],
                                              c["const_idx"], c["const_val"], c["gt"], c["i0"], c["i1"]))
        assert _key(sts[f]) == _key(want), f


def test_groups_of_sixteen_and_eight_lanes():
    """29 frames in one call: 25 at one offset (a group of 16 lanes, one of 8 and
    a single frame), 4 at another (lockstep pairs), each frame's state equal to
    the put of its own output vector"""
    lib = _lib()
    c = _frame_case("inv", 40, 64, 384, 512, 384, 255, 13)
    rng = np.random.default_rng(14)
    frames = [rng.integers(0, 256, size=c["pix"].size, dtype=np.uint8) for _ in range(29)]
    prefixes = [b"q" if f % 7 else b"rr" * 20 for f in range(29)]
    sts = [_state(lib, p) for p in prefixes]
    assert _put_fused(lib, sts, frames, c) == 0
    for f in range(29):
        want = _state(lib, prefixes[f])
        _put_vector(lib, want, oracle_outputs(frames[f], c["copies"], c["padded"], c["cs"], c["n_wires"],
                                              c["const_idx"], c["const_val"], c["gt"], c["i0"], c["i1"]))
        assert _key(sts[f]) == _key(want), f


def test_short_frames_read_as_zero_padded():
    """a frame whose bytes end inside its last copy (a crop of 385-byte copies)
    hashes as the same frame zero-padded to whole copies"""
    lib = _lib()
    c = _frame_case("Crop", 50, 64, 385, 512, -1, 0, 21)
    short = c["pix"][:50 * 385 - 200].copy()
    padded = np.zeros(50 * 385, np.uint8)
    padded[:short.size] = short
    st = _state(lib, b"p")
    assert _put_fused(lib, [st], [short], c) == 0
    want = _state(lib, b"p")
    _put_vector(lib, want, oracle_outputs(padded, c["copies"], c["padded"], c["cs"], c["n_wires"], c["const_idx"],
                                          c["const_val"], c["gt"], c["i0"], c["i1"]))
    assert _key(st) == _key(want)


def test_bad_arguments_are_rejected():
    lib = _lib()
    c = _frame_case("gray", 4, 4, 384, 512, 384, 128, 1)
    st = _state(lib)
    c_bad = dict(c, padded=6)
    assert _put_fused(lib, [st], [c["pix"]], c_bad) == -1
    assert b"bad arguments" in lib.tp_last_error()
    c_bad = dict(c, i0=np.full_like(c["i0"], 600))
    assert _put_fused(lib, [st], [c["pix"]], c_bad) == -1
    assert b"out of range" in lib.tp_last_error()


@pytest.mark.parametrize("setting", ["TRUEPIX_HOST_SHA_PORTABLE", "TRUEPIX_HOST_SHA_NO_MULTIBUFFER"])
def test_other_compressions_give_the_same_state(setting):
    """TRUEPIX_HOST_SHA_PORTABLE=1 (the portable compression for every chain) and
    TRUEPIX_HOST_SHA_NO_MULTIBUFFER=1 (groups on the SHA extensions' lockstep
    pairs instead of the AVX-512 lanes), each read once per process: a child
    process per setting"""
    code = ("import sys; sys.path[:0] = [%r, %r]\n"
            "import test_io_transcript_host as t\n"
            "t.test_fused_put_matches_put_of_the_output_vector()\n"
            "t.test_unequal_offsets_and_three_frames()\n"
            "t.test_groups_of_sixteen_and_eight_lanes()\n" % (ROOT, os.path.join(ROOT, "tests")))
    env = dict(os.environ, **{setting: "1"})
    r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
