"""Replays the golden fixtures against any library bound by fp2lib.Fp2Lib."""
import numpy as np

from fp2lib import run_session


def check_all(lib, G):
    for k in range(3):
        ore, oim = lib.fold(G[f"fold{k}_re"], G[f"fold{k}_im"], G[f"fold{k}_r"])
        assert np.array_equal(ore, G[f"fold{k}_ore"]) and np.array_equal(oim, G[f"fold{k}_oim"]), f"fold{k}"
    ore, oim = lib.expand(G["exp_re"], G["exp_im"], 3)
    assert np.array_equal(ore, G["exp_ore"]) and np.array_equal(oim, G["exp_oim"]), "expand"
    for k in range(3):
        p = f"sc{k}_"
        n_gates, n_wires, n_copies = (int(x) for x in G[p + "shape"])
        z, v, f0, f1 = G[p + "z"], G[p + "v"], G[p + "f0"], G[p + "f1"]
        b, bf0, bf1 = G[p + "b"], G[p + "bf0"], G[p + "bf1"]
        out = lib.sumcheck_early(G[p + "gt"], G[p + "i0"], G[p + "i1"], z[0], z[1], n_copies,
                                 n_wires, v[0], v[1], f0[0], f0[1], f1[0], f1[1], b[0], b[1],
                                 bf0[0], bf0[1], bf1[0], bf1[1])
        assert np.array_equal(out, G[p + "out"]), f"sumcheck_early{k}"
    for k in range(3):
        z = G[f"beta{k}_z"]
        ore, oim = lib.compute_beta(z[0].copy(), z[1].copy(), G[f"beta{k}_init"])
        assert np.array_equal(ore, G[f"beta{k}_ore"]) and np.array_equal(oim, G[f"beta{k}_oim"]), f"beta{k}"
    for k in range(5):
        z = G[f"mle{k}_z"]
        o = lib.mle_eval_base(G[f"mle{k}_x"], z[0].copy(), z[1].copy())
        assert o == tuple(int(x) for x in G[f"mle{k}_out"]), f"mle{k}"
    for k in range(int(G["n_sessions"][0])):
        p = f"sess{k}_"
        n_gates, n_wires, n_copies = (int(x) for x in G[p + "shape"])
        z, v, b = G[p + "z"], G[p + "v"], G[p + "b"]
        claims, wre, wim, beta, _ = run_session(
            lib, G[p + "gt"], G[p + "i0"], G[p + "i1"], z[0].copy(), z[1].copy(), n_copies,
            n_wires, v[0].copy(), v[1].copy(), b[0].copy(), b[1].copy(), G[p + "chal"])
        assert np.array_equal(claims, G[p + "claims"]), f"session{k} claims"
        assert np.array_equal(wre, G[p + "wires"][0]) and np.array_equal(wim, G[p + "wires"][1]), f"session{k} wires"
        assert beta == tuple(int(x) for x in G[p + "beta"]), f"session{k} beta"
