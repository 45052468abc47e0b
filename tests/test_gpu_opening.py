"""truepix_b200.opening on the device: the NIZK opening proof of a frame
committed by FrameCommitter is byte-identical (SHA-256 of the whole file) to the
orion_proof.bin that the reference's own linearPC_multi_prove writes for the same
frame and point (tests/golden/opening_golden.npz), for a gray frame of 64 copies
and a crop frame of 100."""
import hashlib
import json

import numpy as np
import pytest

from test_opening_host import cases

pytestmark = pytest.mark.gpu


def test_opening_proofs_match_reference_program():
    import torch
    from truepix_b200.frame import FrameLayout
    from truepix_b200.opening import opening_proof
    from truepix_b200.orion import FrameCommitter
    n = 0
    for c in cases():
        copies, cs, ci, cv = json.loads(c["layout"].tobytes().decode())
        layout = FrameLayout(copies=copies, copy_size=cs, const_idx=ci, const_val=cv)
        pix = torch.from_numpy(c["pix"].copy()).cuda()
        fc = FrameCommitter([layout])
        fc.commit([pix])
        torch.cuda.synchronize()
        assert fc.root(0) == c["com_root"].tobytes(), c["name"]
        proof = opening_proof(fc, 0, [(int(a), int(b)) for a, b in c["point"]])
        assert len(proof) == int(c["size"][0]), c["name"]
        assert hashlib.sha256(proof).digest() == c["sha256"].tobytes(), c["name"]
        n += 1
    assert n == 2


def test_zk_committer_is_refused():
    import torch
    from truepix_b200.frame import FrameLayout
    from truepix_b200.opening import opening_proof
    from truepix_b200.orion import FrameCommitter
    c = next(cases())
    copies, cs, ci, cv = json.loads(c["layout"].tobytes().decode())
    layout = FrameLayout(copies=copies, copy_size=cs, const_idx=ci, const_val=cv)
    fc = FrameCommitter([layout], zk=True)
    with pytest.raises(ValueError):
        opening_proof(fc, 0, [(0, 0)] * 15)
    torch.cuda.synchronize()
