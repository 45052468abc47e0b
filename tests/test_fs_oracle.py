"""The Fiat-Shamir golden vectors (made by the reference's own FiatShamir class)
replayed by a hashlib restatement of its binary format, on CPU."""
import numpy as np

from fslib import golden, replay_python, scripts


def test_transcript_restatement_matches_reference_vectors():
    g = golden()
    n = 0
    for name, protocol, ops in scripts(g):
        outs, digs = replay_python(protocol, ops)
        np.testing.assert_array_equal(outs, g["fsout_" + name])
        assert digs == g["fsdigest_" + name].tobytes(), name
        n += 1
    assert n == 4


def test_vole_round_restatement_matches_reference_vectors():
    """The VOLE-committed round (interpolation, commitments, equality proof,
    challenge, next value) restated, against vectors made from the reference's
    own util / ExtVOLECommit / FiatShamir (tests/golden/vole_round_golden.npz)."""
    import os
    from fslib import ROOT, vole_rounds_python
    g = np.load(os.path.join(ROOT, "tests", "golden", "vole_round_golden.npz"))
    for name in ("r3", "r14", "r11_prev"):
        chals, vzs, prev, dig, used = vole_rounds_python(g, name)
        np.testing.assert_array_equal(chals, g[name + "_chals"])
        np.testing.assert_array_equal(vzs, g[name + "_vzs"])
        assert prev == tuple(int(x) for x in g[name + "_prev"][0])
        assert dig == g[name + "_digest"].tobytes()
        assert used == int(g[name + "_used"][0])
