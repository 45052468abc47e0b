"""Circuit evaluation on the device (tp_circuit_outputs_pixels_dev,
truepix_b200.frame.circuit_outputs): the output vector the prover puts into its
transcript, bit-exact against vectors made by the reference's own
ArithCircuitBuilder (tests/golden/circuit_outputs_golden.npz), against the
oracle for the four TruePix circuits on whole 1080p frames and a 2160p frame,
argument checks, and the transcript's IO prefix of circuitnizkvec_vole.py
(pid, muxbits, input length, outputs; then the GKR point) drawn through the
drop-in FiatShamir class with the outputs straight from the device."""
import ctypes
import os
import struct

import numpy as np
import pytest

from circuitlib import ROOT, golden_cases, oracle_outputs
from fslib import P61, PyTranscript, encode_put

pytestmark = pytest.mark.gpu

I32P = ctypes.POINTER(ctypes.c_int)


@pytest.fixture(scope="module")
def lib():
    from truepix_b200 import native
    return native.gkr()


def _run(lib, pix_d, copies, padded, cs, n_wires, ci, cv, gt, i0, i1):
    import torch
    bits = lib.tp_circuit_out_bits(len(gt))
    out = torch.full((padded << bits,), -1, dtype=torch.int64, device="cuda")
    gt, i0, i1 = (np.ascontiguousarray(a, np.int32) for a in (gt, i0, i1))
    rc = lib.tp_circuit_outputs_pixels_dev(pix_d.data_ptr(), copies, padded, cs, n_wires, ci, cv, len(gt),
                                          gt.ctypes.data_as(I32P), i0.ctypes.data_as(I32P),
                                          i1.ctypes.data_as(I32P), out.data_ptr(), None)
    return rc, out


def test_outputs_match_reference_vectors(lib):
    import torch
    n = 0
    for c in golden_cases():
        pix_d = torch.from_numpy(c["pix"].copy()).cuda()
        rc, out = _run(lib, pix_d, c["copies"], c["padded"], c["cs"], c["n_wires"], c["const_idx"], c["const_val"],
                       c["gt"], c["i0"], c["i1"])
        assert rc == 0, lib.tp_last_error()
        torch.cuda.synchronize()
        np.testing.assert_array_equal(out.cpu().numpy().view(np.uint64), c["out"], err_msg=c["name"])
        n += 1
    assert n == 8


CIRCUITS = {"gray": (384, 384, 128), "inv": (384, 384, 255), "mask": (384, -1, 0), "Crop": (385, 385, 128)}


@pytest.mark.parametrize("name,height,width", [("gray", 1080, 1920), ("inv", 1080, 1920), ("mask", 1080, 1920),
                                               ("Crop", 1080, 1920), ("gray", 2160, 3840), ("inv", 240, 426)])
def test_whole_frames_match_oracle(lib, name, height, width):
    """full-size frames (2^23 and 2^25 outputs) through the Python helper"""
    import torch
    from truepix_b200.frame import FrameLayout, circuit_outputs
    c = np.load(os.path.join(ROOT, "tests", "golden", "circuits.npz"))
    cs, ci, cv = CIRCUITS[name]
    n = height * width * 3
    layout = FrameLayout(copies=-(-n // 384), copy_size=cs, const_idx=ci, const_val=cv)
    rng = np.random.default_rng(height + len(name))
    pix = rng.integers(0, 256, size=layout.copies * cs, dtype=np.uint8)
    gt, i0, i1 = c[name + "_type"], c[name + "_in0"], c[name + "_in1"]
    out = circuit_outputs(torch.from_numpy(pix).cuda(), layout, gt, i0, i1)
    torch.cuda.synchronize()
    want = oracle_outputs(pix, layout.copies, layout.padded_copies, cs, 512, ci, cv, gt, i0, i1)
    got = out.cpu().numpy().view(np.uint64)
    assert got.size == layout.padded_copies * 512
    np.testing.assert_array_equal(got, want)


def test_bad_arguments_are_rejected(lib):
    import torch
    pix = torch.zeros(4 * 384, dtype=torch.uint8, device="cuda")
    g = np.zeros(4, np.int32)
    ok = dict(copies=4, padded=4, cs=384, n_wires=512, ci=384, cv=128)

    def call(**kw):
        a = dict(ok, **{k: v for k, v in kw.items() if k in ok})
        return _run(lib, pix, a["copies"], a["padded"], a["cs"], a["n_wires"], a["ci"], a["cv"],
                    kw.get("gt", g), kw.get("i0", g), kw.get("i1", g))[0]

    assert call() == 0
    assert call(padded=6) == -1                      # not a power of two
    assert call(padded=2) == -1                      # fewer than the copies
    assert call(ci=100) == -1                        # constant inside the bytes
    assert call(cv=P61) == -1                        # non-canonical constant
    assert call(n_wires=1 << 15) == -1
    assert call(gt=np.array([13], np.int32), i0=np.zeros(1, np.int32), i1=np.zeros(1, np.int32)) == -1
    assert call(gt=g, i0=np.array([0, 0, 512, 0], np.int32), i1=g) == -1
    assert b"gate 2" in lib.tp_last_error()
    assert call(gt=np.zeros(961, np.int32), i0=np.zeros(961, np.int32), i1=np.zeros(961, np.int32)) == -1
    torch.cuda.synchronize()


def test_io_prefix_of_the_transcript(lib):
    """circuitnizkvec_vole.py:277-375 up to the GKR point: put(pid), put(muxbits
    = None, io), put(["private_input_omitted", n], io), put(outputs, io), then
    rand_ext("z1-i") for the output bits and rand_ext("z2-j") for the copy bits;
    the outputs come from the device into a numpy array and go through the
    drop-in class, against the hashlib restatement fed with the oracle's outputs."""
    import torch
    from truepix_b200.fiatshamir import FiatShamir
    from truepix_b200.frame import FrameLayout, circuit_outputs
    c = np.load(os.path.join(ROOT, "tests", "golden", "circuits.npz"))
    gt, i0, i1 = c["gray_type"], c["gray_in0"], c["gray_in1"]
    layout = FrameLayout.for_frame(360, 640)
    rng = np.random.default_rng(31)
    pix = rng.integers(0, 256, size=layout.copies * 384, dtype=np.uint8)
    outs = circuit_outputs(torch.from_numpy(pix).cuda(), layout, gt, i0, i1).cpu().numpy().view(np.uint64)
    n_in = layout.padded_copies * 512
    pid = 4242

    fs = FiatShamir(P61, fp2_type=lambda re, im, q: (re, im))
    fs.put(pid)
    fs.put(None, True)
    fs.put(["private_input_omitted", n_in], True)
    fs.put(outs, True)
    got = [fs.rand_ext("z1-%d" % i) for i in range(9)] + \
          [fs.rand_ext("z2-%d" % j) for j in range(layout.n_copy_bits)]

    want_outs = oracle_outputs(pix, layout.copies, layout.padded_copies, 384, 512, 384, 128, gt, i0, i1)
    t = PyTranscript("truepix")
    t.h.update(encode_put(pid) + encode_put(None) + encode_put(["private_input_omitted", n_in]))
    t.h.update(b"\x01" + struct.pack("<I", want_outs.size) + want_outs.tobytes())
    want = [t.ext("z1-%d" % i) for i in range(9)] + [t.ext("z2-%d" % j) for j in range(layout.n_copy_bits)]
    assert got == want
    assert fs.digest() == t.h.digest()
    assert len(fs.io) == 3 and isinstance(fs.io[2], np.ndarray)
    # the verifier side replays the io queue with take(take_io=True)
    v = FiatShamir.from_string(fs.to_string())
    v._fp2 = lambda re, im, q: (re, im)
    assert v.take() == [pid]
    for _ in range(3):
        v.take(take_io=True)
    assert [v.rand_ext("z1-%d" % i) for i in range(9)] == want[:9]
