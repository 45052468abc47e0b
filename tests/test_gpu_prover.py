"""truepix_b200.prover against proofs made by the reference prover itself
(CircuitProverNIZK.run of circuitnizkvec_vole.py and of its zero-knowledge
variant, tests/golden/prover_golden.npz: gray, inv and crop frames with fixed
pids, VOLE correlations and commitment manifests): the proof
container assembled from the restated values is byte-identical to the
reference's proof, and prove_frames, with every step after the IO prefix on the
device, produces the same bytes."""
import numpy as np
import pytest

from proverlib import cases, circuit, fp2_type, restated_proof

pytestmark = pytest.mark.gpu


def test_container_from_restated_values_matches_reference_proof():
    from truepix_b200.prover import LayerTranscript
    F = fp2_type()
    n = 0
    for c in cases():
        t = LayerTranscript(c["pid"], fp2_type=F)
        digest = restated_proof(c, t)
        assert t.proof_bytes() == c["proof"].tobytes(), c["name"]
        assert digest == c["digest"].tobytes()
        assert [(x.real, x.imag) for x in t.final_input_point] == [tuple(int(v) for v in p) for p in c["point"]]
        n += 1
    assert n == 5


def test_device_proofs_match_reference_proofs():
    import torch
    from truepix_b200.frame import FrameLayout
    from truepix_b200.prover import prove_frames
    F = fp2_type()
    n = 0
    for c in cases():
        gt, i0, i1 = circuit(c["circ"])
        layout = FrameLayout(copies=c["copies"], copy_size=c["cs"], const_idx=c["ci"], const_val=c["cv"])
        pix = torch.from_numpy(c["pix"].copy()).cuda()
        tr = prove_frames([pix], layout, gt, i0, i1, [c["pid"]], [(c["u"], c["v"])], [c["manifest"]], fp2_type=F,
                          zk=c["zk"])
        t = tr[0]
        assert t.proof_bytes() == c["proof"].tobytes(), c["name"]
        assert t.fs.digest() == c["digest"].tobytes()
        assert (t.final_input_tag.real, t.final_input_tag.imag) == tuple(int(v) for v in c["tag"][0])
        n += 1
    assert n == 5
    # a batch of the same frame twice under two pids: the first proof is the reference's
    c = next(cases())
    gt, i0, i1 = circuit(c["circ"])
    layout = FrameLayout(copies=c["copies"], copy_size=c["cs"], const_idx=c["ci"], const_val=c["cv"])
    pix = torch.from_numpy(c["pix"].copy()).cuda()
    tr = prove_frames([pix, pix], layout, gt, i0, i1, [c["pid"], c["pid"] + 1], [(c["u"], c["v"])] * 2,
                      [c["manifest"]] * 2, fp2_type=F, zk=c["zk"])
    assert tr[0].proof_bytes() == c["proof"].tobytes()
    assert tr[1].proof_bytes() != c["proof"].tobytes()


def test_too_few_correlations_raise():
    import torch
    from truepix_b200.frame import FrameLayout
    from truepix_b200.prover import prove_frames
    c = next(cases())
    gt, i0, i1 = circuit(c["circ"])
    layout = FrameLayout(copies=c["copies"], copy_size=c["cs"], const_idx=c["ci"], const_val=c["cv"])
    pix = torch.from_numpy(c["pix"].copy()).cuda()
    with pytest.raises(IndexError):
        prove_frames([pix], layout, gt, i0, i1, [c["pid"]], [(c["u"][:40], c["v"][:40])], [c["manifest"]])


def test_commit_then_prove():
    """The commit phase and the proof in one process: the frame committed on the
    device (zero-knowledge commit pair), its manifest built from the roots
    (manifests_of), the proof bound to it equal to the restated proof of the same
    frame under the same manifest."""
    import torch
    from truepix_b200.frame import FrameLayout
    from truepix_b200.orion import FrameCommitter
    from truepix_b200.prover import LayerTranscript, manifests_of, prove_frames
    F = fp2_type()
    c = [x for x in cases() if x["name"] == "gray4zk"][0]
    gt, i0, i1 = circuit(c["circ"])
    layout = FrameLayout(copies=c["copies"], copy_size=c["cs"], const_idx=c["ci"], const_val=c["cv"])
    pix = torch.from_numpy(c["pix"].copy()).cuda()
    fc = FrameCommitter([layout], zk=True)
    fc.commit([pix], mask_seeds=[0x5EED])
    torch.cuda.synchronize()
    [m] = manifests_of(fc)
    assert m["masked_root"] == fc.root_hex(0) and len(m["mask_root"]) == 64 and m["zk"]
    [t] = prove_frames([pix], layout, gt, i0, i1, [c["pid"]], [(c["u"], c["v"])], [m], fp2_type=F, zk=True)
    c2 = dict(c, manifest=m)
    t2 = LayerTranscript(c["pid"], fp2_type=F)
    restated_proof(c2, t2)
    assert t.proof_bytes() == t2.proof_bytes()
