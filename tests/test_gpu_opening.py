"""truepix_b200.opening on the device: the NIZK opening proofs of a frame
committed by FrameCommitter are byte-identical (SHA-256 of the whole file) to
the files the reference's own linearPC_multi_prove programs write for the same
frame and point (tests/golden/opening_golden.npz): orion_proof.bin for plain
commits of a gray frame of 64 copies and a crop frame of 100, and for the
zero-knowledge commit pair of a gray frame of 80 copies (TruePix's default)
orion_proof_masked.bin and orion_proof_mask.bin."""
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
        copies, cs, ci, cv, seed = json.loads(c["layout"].tobytes().decode())
        layout = FrameLayout(copies=copies, copy_size=cs, const_idx=ci, const_val=cv)
        pix = torch.from_numpy(c["pix"].copy()).cuda()
        fc = FrameCommitter([layout], zk=seed is not None)
        fc.commit([pix], mask_seeds=None if seed is None else [seed])
        torch.cuda.synchronize()
        point = [(int(a), int(b)) for a, b in c["point"]]
        for tag, poly in ([("", "masked"), ("mask_", "mask")] if seed is not None else [("", None)]):
            root = fc.mask_root(0) if poly == "mask" else fc.root(0)
            assert root == c[tag + "com_root"].tobytes(), c["name"] + tag
            proof = opening_proof(fc, 0, point, poly)
            assert len(proof) == int(c[tag + "size"][0]), c["name"] + tag
            assert hashlib.sha256(proof).digest() == c[tag + "sha256"].tobytes(), c["name"] + tag
            n += 1
    assert n == 4


def test_library_transcript_draws_the_reference_queries():
    """tp_orion_open_queries (host code of the library) against every golden proof's queries"""
    import numpy as np
    from test_opening_host import eq
    from truepix_b200 import native
    from truepix_b200.opening import query_columns, split_point
    lib = native.gkr(require_device=False)
    n = 0
    for c in cases():
        seed = json.loads(c["layout"].tobytes().decode())[4]
        for tag, group in ([("", 0), ("mask_", 1)] if seed is not None else [("", -1)]):
            N, cw = int(c[tag + "header"][2]), int(c[tag + "header"][5])
            c0, c1 = split_point([(int(a), int(b)) for a, b in c["point"]])
            q = query_columns(lib, c[tag + "com_root"].tobytes(), N, 0 if tag else 1, np.array(eq(c0), np.uint64),
                              np.array(eq(c1), np.uint64), cw, group)
            assert q == [int(x) for x in c[tag + "col_q"]], c["name"] + tag
            n += 1
    assert n == 4


def test_polynomial_must_match_the_commit():
    import torch
    from truepix_b200.frame import FrameLayout
    from truepix_b200.opening import opening_proof
    from truepix_b200.orion import FrameCommitter
    c = next(cases())
    copies, cs, ci, cv, _ = json.loads(c["layout"].tobytes().decode())
    layout = FrameLayout(copies=copies, copy_size=cs, const_idx=ci, const_val=cv)
    for zk, poly in ((True, None), (False, "mask"), (True, "other")):
        fc = FrameCommitter([layout], zk=zk)
        with pytest.raises(ValueError):
            opening_proof(fc, 0, [(0, 0)] * 15, poly)
    torch.cuda.synchronize()
