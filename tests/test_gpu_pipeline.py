"""truepix_b200.pipeline.ProofPipeline on the device: batches of frames proved
end to end with the stages of two batches overlapped. Its proof containers are
byte-identical to the reference prover's own proofs (tests/golden/
prover_golden.npz: gray, inv and crop frames of both provers, with the
reference's manifests bound), and for device-committed frames every proof and
every Orion opening file equals what prove_frames and opening_proof (pinned to
the reference prover and to the reference's linearPC_multi_prove program by
tests/test_gpu_prover.py and tests/test_gpu_opening.py) give for the same frame,
plain and zero-knowledge, device-resident and host (pinned) frames."""
import numpy as np
import pytest

from proverlib import cases, circuit, fp2_type

pytestmark = pytest.mark.gpu


def _layout(c):
    from truepix_b200.frame import FrameLayout
    return FrameLayout(copies=c["copies"], copy_size=c["cs"], const_idx=c["ci"], const_val=c["cv"])


def test_pipeline_proofs_match_reference_proofs():
    from truepix_b200.pipeline import ProofPipeline
    F = fp2_type()
    n = 0
    for c in cases():
        gt, i0, i1 = circuit(c["circ"])
        layout = _layout(c)
        pipe = ProofPipeline(layout, gt, i0, i1, batch=2, zk=c["zk"], fp2_type=F, host_threads=4, commit_streams=2)
        batch = dict(frames_host=[c["pix"], c["pix"]], pids=[c["pid"], c["pid"] + 1],
                     correlations=[(c["u"], c["v"])] * 2, manifests=[c["manifest"]] * 2,
                     mask_seeds=[1, 2] if c["zk"] else None)
        [proofs] = list(pipe.run([batch]))
        assert proofs[0].proof_bytes() == c["proof"].tobytes(), c["name"]
        assert proofs[1].proof_bytes() != c["proof"].tobytes()
        pipe.close()
        n += 1
    assert n == 5


def _frames(rng, layout, k):
    return [rng.integers(0, 256, size=layout.copies * layout.copy_size, dtype=np.uint8) for _ in range(k)]


@pytest.mark.parametrize("zk", [False, True])
@pytest.mark.parametrize("resident", [True, False])
def test_pipeline_matches_step_by_step_proofs_and_openings(zk, resident):
    """four batches of two 90-copy gray frames through the pipeline (device slots
    reused, IO hashed ahead: the first batch in pairs, the rest in one group per
    batch), against commit + prove_frames + opening_proof of each frame on its own"""
    import torch
    from truepix_b200.frame import FrameLayout
    from truepix_b200.opening import opening_proof
    from truepix_b200.orion import FrameCommitter
    from truepix_b200.pipeline import ProofPipeline, correlations_needed
    from truepix_b200.prover import prove_frames
    F = fp2_type()
    gt, i0, i1 = circuit("gray")
    layout = FrameLayout(copies=90)
    rng = np.random.default_rng(5 + zk + 2 * resident)
    count = correlations_needed(layout, zk) + 3
    B = 2
    batches, want = [], []
    for b in range(4):
        frames = _frames(rng, layout, B)
        corr = [(rng.integers(0, (1 << 61) - 1, size=(count, 2), dtype=np.uint64),
                 rng.integers(0, (1 << 61) - 1, size=(count, 2), dtype=np.uint64)) for _ in range(B)]
        host = [torch.from_numpy(f).pin_memory() for f in frames] if not resident else frames
        batch = dict(frames_host=host, pids=[100 * b + f for f in range(B)], correlations=corr,
                     mask_seeds=[7 * b + f for f in range(B)] if zk else None)
        if resident:
            batch["frames_dev"] = [torch.from_numpy(f).cuda() for f in frames]
        batches.append(batch)
    pipe = ProofPipeline(layout, gt, i0, i1, batch=B, zk=zk, fp2_type=F, host_threads=4, commit_streams=2,
                         slots=3 if resident else 2, io_ahead=2)
    got = list(pipe.run(batches))
    pipe.close()
    assert len(got) == 4
    for b, batch in enumerate(batches):
        frames = [np.asarray(x) if not hasattr(x, "numpy") else x.numpy() for x in batch["frames_host"]]
        for f in range(B):
            pix = torch.from_numpy(frames[f].copy()).cuda()
            fc = FrameCommitter([layout], zk=zk)
            fc.commit([pix], mask_seeds=[batch["mask_seeds"][f]] if zk else None)
            torch.cuda.synchronize()
            p = got[b][f]
            from truepix_b200.prover import manifests_of
            [m] = manifests_of(fc)
            assert p.manifest == m, (b, f)
            [t] = prove_frames([pix], layout, gt, i0, i1, [batch["pids"][f]], [batch["correlations"][f]], [m],
                               fp2_type=F, zk=zk)
            assert p.proof_bytes() == t.proof_bytes(), (b, f)
            pt = [(int(x.real), int(x.imag)) for x in t.final_input_point]
            if zk:
                assert p.opening["masked"] == opening_proof(fc, 0, pt, "masked"), (b, f)
                assert p.opening["mask"] == opening_proof(fc, 0, pt, "mask"), (b, f)
            else:
                assert p.opening == opening_proof(fc, 0, pt), (b, f)


def test_too_few_correlations_raise():
    from truepix_b200.frame import FrameLayout
    from truepix_b200.pipeline import ProofPipeline, correlations_needed
    gt, i0, i1 = circuit("gray")
    layout = FrameLayout(copies=20)
    rng = np.random.default_rng(1)
    short = correlations_needed(layout) - 1
    corr = [(np.zeros((short, 2), np.uint64), np.zeros((short, 2), np.uint64))]
    pipe = ProofPipeline(layout, gt, i0, i1, batch=1, host_threads=2, commit_streams=1)
    with pytest.raises(IndexError):
        list(pipe.run([dict(frames_host=_frames(rng, layout, 1), pids=[1], correlations=corr)]))
    pipe.close()
