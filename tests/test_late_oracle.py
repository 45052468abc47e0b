"""The oracle's late rounds and line projection against vectors made by the
reference's own LayerProver (tests/golden/late_golden.npz): gray and crop
circuits (384 gates, 512 wires), random circuits of every non-multiplexer type
with field-size inputs."""
from latelib import golden_cases, oracle, pairs


def test_oracle_matches_reference_layer_prover():
    n = 0
    for c in golden_cases():
        gt, i0, i1 = ([int(x) for x in row] for row in c["gates"])
        nb, nin = c["n_copy_bits"], c["n_in_bits"]
        coefs, h, v1, v2 = oracle.late_rounds(pairs(c["wires"]), pairs(c["beta"])[0], pairs(c["zg"]), (gt, i0, i1),
                                              nin, pairs(c["chal"])[nb:])
        assert [x for cf in coefs for x in cf] == pairs(c["late"]), c["name"]
        assert h == pairs(c["final"]), c["name"]
        # the final coefficients are the line's values: h(0) = V(w1), h(1) = V(w2)
        assert h[0] == v1
        n += 1
    assert n == 6


def test_vole_chain_restatement_matches_reference():
    """The whole layer's VOLE-committed rounds and closing proofs restated (hashlib transcript, the
    commit / equality / challenge / Horner steps, the oracle's late rounds fed
    round by round with the drawn challenges) against the reference's
    LayerProver + ExtVOLECommit + FiatShamir chain (tests/golden/
    layer_vole_golden.npz). The early rounds' coefficients are the golden ones
    (their computation is pinned by the native_fp2 vectors)."""
    from fslib import PyTranscript, f2add, f2mul, f2sub
    from layervole import cases, closing_python
    n_cases = 0
    for c in cases():
        n, nb = c["n_in_bits"], c["nb"]
        gates = tuple([int(x) for x in row] for row in c["gates"])
        T = PyTranscript("truepix")
        T.u64s([int(x) for x in c["prefix"]])
        u, v = pairs(c["u"]), pairs(c["v"])
        idx, prev = int(c["start"][0]), None
        v_elem, out_elem = [(0, 0)] * 4, [(0, 0)] * 4
        late = oracle.LateRounds(pairs(c["wires"]), pairs(c["beta"])[0], pairs(c["zg"]), gates, n)
        early = pairs(c["coefs"])[:4 * nb]
        chals, ds, vzs, coefs = [], [], [], []
        for rd in range(nb + 2 * n):
            cf = early[4 * rd:4 * rd + 4] if rd < nb else late.coefs()
            tags = []
            for k, x in enumerate(cf):
                tags.append(v[idx])
                d = f2sub(x, u[idx])
                idx += 1
                T.fp2(*d)
                ds.append(d)
                v_elem[k] = f2add(v_elem[k], tags[-1])
                out_elem[k] = f2add(out_elem[k], x)
            now = tags[0]
            for t in tags:
                now = f2add(now, t)
            e = T.ext("eq")
            vz = f2mul(now, e) if prev is None else f2mul(f2sub(prev, now), e)
            T.fp2(*vz)
            vzs.append(vz)
            r = T.ext("sc-0-%d" % rd)
            chals.append(r)
            p = tags[-1]
            for t in reversed(tags[:-1]):
                p = f2add(f2mul(p, r), t)
            prev = p
            coefs += cf
            if rd >= nb:
                late.next_round(r)
        assert chals == pairs(c["chal"]), c["name"]
        assert ds == pairs(c["d"]) and vzs == pairs(c["vz"]) and coefs == pairs(c["coefs"])
        assert late.line() == pairs(c["final"])
        assert prev == pairs(c["prev"])[0] and idx == int(c["used"][0])
        assert v_elem == pairs(c["v_elem"]) and out_elem == pairs(c["out_elem"])
        assert T.h.digest() == c["digest"].tobytes()
        # the layer's closing proofs
        chal = pairs(c["chal"])
        w3, w1, w2 = chal[:nb], chal[nb:nb + n], chal[nb + n:]
        closing, point, tag, used = closing_python(T, late.line(), prev, idx, v_elem, out_elem, u, v, w1, w2, w3,
                                                   pairs(c["z2"]), pairs(c["zg"]), gates)
        assert closing == pairs(c["closing"]), c["name"]
        assert point == pairs(c["point"]) and tag == pairs(c["tag"])[0]
        assert used == int(c["used_closed"][0])
        assert T.h.digest() == c["digest_closed"].tobytes()
        n_cases += 1
    assert n_cases == 2
