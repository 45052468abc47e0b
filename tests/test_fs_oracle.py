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
    assert n == 3
