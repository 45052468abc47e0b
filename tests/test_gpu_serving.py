"""Continuous batching (truepix_b200.serving): frames of mixed operations and
resolutions join and leave one running batch between rounds; every result must
be bit-identical to the same request proven alone, and to the single-frame path
(truepix_b200.frame.GkrInputLayerProver + truepix_b200.orion.FrameCommitter)."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def circuits():
    from truepix_b200.serving import Circuit
    c = np.load(os.path.join(ROOT, "tests", "golden", "circuits.npz"))
    g = lambda n: (c[n + "_type"], c[n + "_in0"], c[n + "_in1"])
    return {"gray": Circuit("gray", *g("gray"), 384, 384, 128),
            "inv": Circuit("inv", *g("inv"), 384, 384, 255),
            "mask": Circuit("mask", *g("mask"), 384, -1, 0),
            "crop": Circuit("crop", *g("Crop"), 385, -1, 0)}


def requests():
    from truepix_b200.serving import Request
    cs = circuits()
    sizes = [(120, 160), (360, 640), (240, 426), (480, 854), (720, 1280), (120, 160), (360, 640),
             (1080, 1920), (240, 426), (480, 854)]
    ops = ["gray", "crop", "mask", "inv", "gray", "crop", "gray", "gray", "mask", "crop"]
    arrivals = [0, 0, 1, 2, 3, 5, 8, 9, 12, 13]
    out = []
    for i, ((h, w), op, t) in enumerate(zip(sizes, ops, arrivals)):
        rng = np.random.default_rng(100 + i)
        out.append(Request(i, cs[op], h, w, rng.integers(0, 256, size=h * w * 3, dtype=np.uint8),
                           seed=500 + i, arrival=float(t)))
    return out


def by_rid(results):
    return {r.rid: r for r in results}


def same(a, b):
    return (np.array_equal(a.claims, b.claims) and np.array_equal(a.wires, b.wires) and a.beta == b.beta
            and a.mle == b.mle and a.root == b.root)


def test_results_in_the_mix_equal_results_alone():
    from truepix_b200.serving import ProofServer
    reqs = requests()
    srv = ProofServer(slots=6, hbm_budget=8e9)
    mixed = by_rid(srv.run(reqs, realtime=False))
    assert sorted(mixed) == list(range(len(reqs)))
    alone_srv = ProofServer(slots=2)
    for r in requests():
        alone = alone_srv.run([r], realtime=False)
        assert len(alone) == 1
        assert same(mixed[r.rid], alone[0]), r.rid
        from truepix_b200.serving import layout_for
        assert mixed[r.rid].claims.shape == (layout_for(r.circuit, r.height, r.width).n_copy_bits, 8)


def test_serving_matches_the_single_frame_path():
    import torch
    from truepix_b200.frame import GkrInputLayerProver, pack_fp2
    from truepix_b200.orion import FrameCommitter
    from truepix_b200.serving import ProofServer, layout_for, transcript_values
    r = requests()[4]                     # gray 720p, 13 rounds
    res = ProofServer(slots=2).run([r], realtime=False)[0]
    L = layout_for(r.circuit, r.height, r.width)
    z1, z2, point, chal = transcript_values(r.seed, r.circuit.gate_type.size, L.n_copy_bits, L.n_in_bits)
    dev = torch.device("cuda", 0)
    pix = torch.from_numpy(np.ascontiguousarray(r.pixels[:L.copies * L.copy_size])).to(dev)
    plain = GkrInputLayerProver(L, r.circuit.gate_type, r.circuit.in0, r.circuit.in1)
    plain.prove(pix, z1, torch.from_numpy(pack_fp2(z2[:, 0], z2[:, 1])).to(dev),
                torch.from_numpy(pack_fp2(point[:, 0], point[:, 1])).to(dev), chal)
    fc = FrameCommitter([L])
    fc.commit([pix])
    torch.cuda.synchronize()
    c, w, b, m = plain.results()
    assert np.array_equal(c, res.claims) and np.array_equal(w, res.wires)
    assert b == res.beta and m == res.mle
    assert fc.root(0) == res.root


def test_admission_respects_the_hbm_budget():
    from truepix_b200.serving import ProofServer
    reqs = requests()
    from truepix_b200.serving import layout_for
    budget = 2 * max(ProofServer.footprint(layout_for(q.circuit, q.height, q.width)) for q in reqs)
    srv = ProofServer(slots=8, hbm_budget=budget)
    peak = [0.0]
    orig = srv._start

    def start(req):
        orig(req)
        peak[0] = max(peak[0], srv.used)
    srv._start = start
    out = srv.run(reqs, realtime=False)
    assert len(out) == len(reqs)
    assert peak[0] <= budget


def test_pinned_tensor_frames_equal_numpy_frames():
    """Frames handed over in pinned host memory (copied straight to the device)
    and as numpy arrays (through the staging buffers), in one realtime run with
    small commit and slot pools: identical results."""
    import torch
    from truepix_b200.serving import ProofServer
    base = by_rid(ProofServer(slots=4).run(requests(), realtime=False))
    reqs = requests()
    for k, r in enumerate(reqs):
        if k % 2 == 0:
            r.pixels = torch.from_numpy(r.pixels).pin_memory()
        r.arrival = 0.002 * k
    srv = ProofServer(slots=3, commit_buffers=2)
    got = by_rid(srv.run(reqs, realtime=True))
    assert sorted(got) == sorted(base)
    for rid in base:
        assert same(got[rid], base[rid]), rid
    with pytest.raises(ValueError):
        srv.run([type(reqs[0])(99, reqs[0].circuit, 120, 160, torch.zeros(120 * 160 * 3, dtype=torch.uint8),
                               seed=1)], realtime=False)
