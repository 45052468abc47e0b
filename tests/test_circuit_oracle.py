"""The oracle's circuit evaluation against output vectors made by the
reference's own ArithCircuitBuilder (tests/golden/circuit_outputs_golden.npz):
the four TruePix circuits, random gate tables of every non-multiplexer type with
a large constant, one gate, one copy."""
import numpy as np

from circuitlib import golden_cases, oracle_outputs


def test_oracle_matches_reference_circuit_evaluator():
    n = 0
    for c in golden_cases():
        got = oracle_outputs(c["pix"], c["copies"], c["padded"], c["cs"], c["n_wires"], c["const_idx"],
                             c["const_val"], c["gt"], c["i0"], c["i1"])
        np.testing.assert_array_equal(got, c["out"], err_msg=c["name"])
        n += 1
    assert n == 8
