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
