"""The serving loop (truepix_b200.serving): requests of mixed operations and
resolutions join and leave one running batch, each on its own device
transcript; every request leaves with its whole proof (the proof container and
the Orion opening file). A proof made in the mix is byte-identical to the same
request served alone and to the step-by-step path (commit, prove_frames,
opening_proof: pinned to the reference prover's proofs and the reference
program's opening files by tests/test_gpu_prover.py and test_gpu_opening.py);
admission keeps the HBM footprint within the budget."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
P61 = (1 << 61) - 1


def circuits():
    from truepix_b200.serving import Circuit
    c = np.load(os.path.join(ROOT, "tests", "golden", "circuits.npz"))
    g = lambda n: (c[n + "_type"], c[n + "_in0"], c[n + "_in1"])
    return {"gray": Circuit("gray", *g("gray"), 384, 384, 128),
            "inv": Circuit("inv", *g("inv"), 384, 384, 255),
            "mask": Circuit("mask", *g("mask"), 384, -1, 0),
            "crop": Circuit("crop", *g("Crop"), 385, -1, 0)}


def requests():
    from truepix_b200.pipeline import correlations_needed
    from truepix_b200.serving import Request, layout_for
    cs = circuits()
    sizes = [(120, 160), (360, 640), (240, 426), (480, 854), (720, 1280), (120, 160), (360, 640),
             (1080, 1920), (240, 426), (480, 854)]
    ops = ["gray", "crop", "mask", "inv", "gray", "crop", "gray", "gray", "mask", "crop"]
    out = []
    for i, ((h, w), op) in enumerate(zip(sizes, ops)):
        rng = np.random.default_rng(100 + i)
        count = correlations_needed(layout_for(cs[op], h, w)) + i
        corr = (rng.integers(0, P61, size=(count, 2), dtype=np.uint64),
                rng.integers(0, P61, size=(count, 2), dtype=np.uint64))
        out.append(Request(i, cs[op], h, w, rng.integers(0, 256, size=h * w * 3, dtype=np.uint8), pid=500 + i,
                           correlations=corr, arrival=0.0))
    return out


def test_proofs_in_the_mix_equal_proofs_alone():
    from truepix_b200.serving import ProofServer
    srv = ProofServer(slots=6, hbm_budget=8e9, max_height=1080, max_width=1920, host_threads=4, commit_streams=3)
    peak = [0.0]
    admit = srv._admit

    def watch(req):
        admit(req)
        peak[0] = max(peak[0], srv.used)
    srv._admit = watch
    mixed = {r.rid: r for r in srv.run(requests(), realtime=False)}
    srv.close()
    assert sorted(mixed) == list(range(10))
    assert peak[0] <= 8e9 or len(mixed) == 1
    alone_srv = ProofServer(slots=2, max_height=1080, max_width=1920, host_threads=2, commit_streams=1)
    for r in requests():
        [alone] = alone_srv.run([r], realtime=False)
        assert alone.proof.proof_bytes() == mixed[r.rid].proof.proof_bytes(), r.rid
        assert alone.proof.opening == mixed[r.rid].proof.opening, r.rid
        assert alone.latency > 0
    alone_srv.close()


def test_serving_matches_the_step_by_step_path():
    import torch
    from truepix_b200.opening import opening_proof
    from truepix_b200.orion import FrameCommitter
    from truepix_b200.prover import manifests_of, prove_frames
    from truepix_b200.serving import ProofServer, layout_for
    for k in (4, 1):                       # gray 720p, crop 360p
        r = requests()[k]
        srv = ProofServer(slots=2, max_height=1080, max_width=1920, host_threads=2, commit_streams=1)
        [res] = srv.run([r], realtime=False)
        srv.close()
        L = layout_for(r.circuit, r.height, r.width)
        padded = np.zeros(L.copies * L.copy_size, np.uint8)     # the last copy zero-padded
        padded[:min(padded.size, r.pixels.size)] = r.pixels[:padded.size]
        pix = torch.from_numpy(padded).cuda()
        fc = FrameCommitter([L])
        fc.commit([pix])
        torch.cuda.synchronize()
        [m] = manifests_of(fc)
        assert res.proof.manifest == m
        c = r.circuit
        [t] = prove_frames([pix], L, c.gate_type, c.in0, c.in1, [r.pid], [r.correlations], [m], zk=False)
        assert res.proof.proof_bytes() == t.proof_bytes(), k
        pt = [(int(x.real), int(x.imag)) if hasattr(x, "real") else (int(x[0]), int(x[1]))
              for x in t.final_input_point]
        assert res.proof.opening == opening_proof(fc, 0, pt), k


def test_too_few_correlations_are_refused():
    from truepix_b200.serving import ProofServer
    r = requests()[0]
    r.correlations = (r.correlations[0][:10], r.correlations[1][:10])
    srv = ProofServer(slots=1, max_height=240, max_width=320, host_threads=1, commit_streams=1)
    with pytest.raises(IndexError):
        srv.run([r], realtime=False)
    srv.close()
