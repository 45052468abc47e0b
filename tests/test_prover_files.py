"""The files the reference prover reads, taken as arguments by
truepix_b200.prover: the binary VOLE prover file (ExtVOLEGen.py:25-50, 130-186)
and the Orion commitment manifest's binding (fp2_link.py:487-504). Host code
only."""
import json
import struct

import numpy as np
import pytest

from proverlib import cases

P61 = (1 << 61) - 1


def write_vole(path, u, v, magic=b"EVOL", version=1, role=1, reps=1, prime=P61, cut=0):
    with open(path, "wb") as fh:
        fh.write(struct.pack("<4sIIIIQ", magic, version, role, reps, len(u), prime))
        data = b"".join(np.ascontiguousarray(a).tobytes() for a in (u[:, 0], u[:, 1], v[:, 0], v[:, 1]))
        fh.write(data[:len(data) - cut])


def test_vole_prover_file_round_trip_and_errors(tmp_path):
    from truepix_b200.prover import read_vole_prover_file
    c = next(cases())
    p = str(tmp_path / "vole_ext_prover_1.json")
    write_vole(p, c["u"], c["v"])
    u, v = read_vole_prover_file(p)
    np.testing.assert_array_equal(u, c["u"])
    np.testing.assert_array_equal(v, c["v"])
    for kw in (dict(magic=b"EVOX"), dict(role=2), dict(reps=2), dict(version=2), dict(prime=97), dict(cut=8)):
        write_vole(p, c["u"], c["v"], **kw)
        with pytest.raises(ValueError):
            read_vole_prover_file(p)


def test_commit_binding_fields():
    from truepix_b200.prover import LAYOUT_ID, commit_binding
    for c in cases():
        m = c["manifest"]
        b = commit_binding(m)
        assert b[:4] == ["orion-commit", "truepix", LAYOUT_ID, 1 if m["zk"] else 0]
        assert b[4:12] == [int(m[k]) for k in ("copies", "padded_copies", "copy_size", "padded_copy_size",
                                               "const_idx", "const_val", "n", "lg_n")]
        assert b[12:] == [m["masked_root"], m["mask_root"] or ""]
        json.dumps(b)


def test_commit_manifest_of_a_layout():
    """the manifest of the commit phase for a frame layout: the fields of
    make_layout (padded copies, 512-entry copies, n, lg_n) and the roots as
    root_hex strings (pinned to the reference's hex of its own roots)"""
    import os
    from proverlib import ROOT
    from truepix_b200.frame import FrameLayout
    from truepix_b200.orion import FrameCommitter
    from truepix_b200.prover import commit_manifest
    g = np.load(os.path.join(ROOT, "tests", "golden", "orion_zk_golden.npz"))
    root = g["zkmasked_gray40"].tobytes()
    hx = FrameCommitter.hex(root)
    assert hx == g["zkmaskedhex_gray40"].tobytes().decode()
    L = FrameLayout.for_frame(1080, 1920)
    m = commit_manifest(L, hx, "00" * 32, zk=True)
    assert (m["copies"], m["padded_copies"], m["copy_size"], m["padded_copy_size"]) == (16200, 16384, 384, 512)
    assert (m["const_idx"], m["const_val"], m["n"], m["lg_n"]) == (384, 128, 1 << 23, 23)
    assert m["masked_root"] == hx and m["mask_root"] == "00" * 32 and m["zk"] is True
    m = commit_manifest(FrameLayout(copies=5, copy_size=384, const_idx=-1, const_val=0), hx, zk=False)
    assert m["mask_root"] == "" and m["zk"] is False and m["padded_copies"] == 8 and m["const_idx"] == -1


def test_point_file_for_the_open_phase(tmp_path):
    """the input point in fp2_link.write_point_file's two forms"""
    from truepix_b200.prover import write_point_file
    c = next(cases())
    pts = [(int(a), int(b)) for a, b in c["point"]]
    j, t = write_point_file(str(tmp_path / "gkr_point_prover.json"), pts)
    d = json.load(open(j))
    assert d == {"protocol": "truepix", "field": "fp2-mersenne61", "layout": "copy-major-384-const128-pad512-v1",
                 "point": [list(p) for p in pts]}
    lines = open(t).read().splitlines()
    assert lines[0] == str(len(pts)) and lines[1:] == ["%d %d" % p for p in pts]
