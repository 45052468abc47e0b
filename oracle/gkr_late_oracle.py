"""CPU restatement of the late rounds of the GKR input layer's sumcheck and of
the line projection that ends it -- TEST INFRASTRUCTURE ONLY: tests/ use it as
the checker of the CUDA late-round kernel; the shipped library never imports it.

Follows the reference's Python prover literally (pure Python, small sizes):
  * per-gate outputs of a late round, layerprover.py:231-247 with
    gateprover.py:105-140 (compute_outputs_late): the value at 0 or 1 (by the
    gate's input bit) and at the third point -1, each times the gate's
    accumulated wiring weight, summed over gates, times beta's final value;
  * updates, layerprover.py:268-290 and gateprover.py:142-185 (next_round): the
    input table folded by the challenge (layercompute.py:74-150, LayerComputeV,
    expanded outputs, restarted after the first pass), the gate's input value
    re-read from it, its weight times r or 1 - r;
  * interpolate_quadratic (util.py:91-113) on the values at 0, 1, -1;
  * the line projection (layercompute.py:152-247, LayerComputeH): the input
    values at w1 + t (w2 - w1) for t = 0..n_in_bits (t = 0, 1 from the two
    passes, the others from tables folded by those points), then the
    coefficients of the degree-n_in_bits polynomial through them
    (util.lagrange_interpolate: the unique interpolant, here by Newton's
    divided differences).
Pinned by tests/golden/late_golden.npz, made by the reference's LayerProver.
"""
from __future__ import annotations

P = (1 << 61) - 1


def add(a, b): return ((a[0] + b[0]) % P, (a[1] + b[1]) % P)
def sub(a, b): return ((a[0] - b[0]) % P, (a[1] - b[1]) % P)
def mul(a, b): return ((a[0] * b[0] - a[1] * b[1]) % P, (a[0] * b[1] + a[1] * b[0]) % P)
def scale(a, k): return (a[0] * k % P, a[1] * k % P)


ONE = (1, 0)


def gatefn(t, x, y):
    """native_fp2_core.hpp:32-51 (the type index of native_fp2_bridge.py:450-472)"""
    if t == 0: return mul(x, y)
    if t == 1: return add(x, y)
    if t == 2: return sub(x, y)
    if t == 3: return x
    if t == 4: return y
    if t == 5: return sub(add(x, y), mul(x, y))
    if t == 6: return sub(add(x, y), scale(mul(x, y), 2))
    if t == 7: return sub(ONE, x)
    if t == 8: return sub(ONE, mul(x, y))
    if t == 9: return sub(add(ONE, mul(x, y)), add(x, y))
    if t == 10: return sub(add(ONE, scale(mul(x, y), 2)), add(x, y))
    if t == 11: return mul(sub(ONE, x), y)
    return x


def fold(a, b, r):
    """fold_val: a + r (b - a)"""
    return add(a, mul(r, sub(b, a)))


class _V:
    """LayerComputeV with expanded outputs and one extra point (-1), restarted per pass"""

    def __init__(self, inputs):
        self.inputs = list(inputs)
        self.v1v2 = []
        self.reset()

    def reset(self):
        self.scratch = list(self.inputs)
        self.outputs = list(self.inputs)
        self.fact = self._expand((-1 % P, 0))

    def _expand(self, r):
        n = len(self.inputs)
        half = len(self.scratch) // 2
        res = [fold(self.scratch[2 * i], self.scratch[2 * i + 1], r) for i in range(half)]
        rep = n // half
        return [res[i // rep] for i in range(n)], res

    def next_round(self, r):
        (self.outputs, self.scratch) = self._expand(r)
        if len(self.scratch) == 1:
            self.v1v2.append(self.scratch[0])
            self.prev = self.scratch[0]
            self.reset()
        else:
            self.fact = self._expand((-1 % P, 0))
        # fact holds (expanded values at -1, scratch); only the expanded part is read

    def at_m1(self, idx):
        return self.fact[0][idx]


def interpolate_quadratic(f0, f1, fm1):
    """util.interpolate_quadratic: coefficients from the values at 0, 1, -1"""
    half = (P + 1) // 2
    a = sub((0, 0), f0)
    c2 = add(scale(add(f1, fm1), half), a)
    c1 = add(sub(f1, c2), a)
    return [f0, c1, c2]


def mle(vals, point):
    """the multilinear extension of vals at point, LSB first (fold pairs by point[0] first)"""
    t = list(vals)
    for r in point:
        t = [fold(t[2 * i], t[2 * i + 1], r) for i in range(len(t) // 2)]
    return t[0]


def interpolate(ys):
    """coefficients (constant first) of the polynomial through (t, ys[t]), t = 0..len - 1"""
    n = len(ys) - 1
    d = list(ys)
    for lvl in range(1, n + 1):
        inv = pow(lvl, P - 2, P)
        for i in range(n, lvl - 1, -1):
            d[i] = scale(sub(d[i], d[i - 1]), inv)
    c = [d[n]]
    for i in range(n - 1, -1, -1):
        # c(t) * (t - i) + d[i]
        nc = [(0, 0)] * (len(c) + 1)
        for k, ck in enumerate(c):
            nc[k + 1] = add(nc[k + 1], ck)
            nc[k] = sub(nc[k], scale(ck, i))
        nc[0] = add(nc[0], d[i])
        c = nc
    return c


class LateRounds:
    """The late phase of one layer, round by round: coefs() gives the round's
    three coefficients, next_round(r) binds the challenge, line() the final
    coefficients after all 2 n rounds."""

    def __init__(self, wires, beta, zg, gates, n_in_bits):
        self.n = n_in_bits
        self.gt, self.i0, self.i1 = gates
        self.wires = list(wires)
        self.beta = beta
        self.V = _V(wires)
        self.A = list(zg)
        self.X = [wires[a] for a in self.i0]
        self.Y = [wires[b] for b in self.i1]
        self.rd = 0
        self.w = []

    def coefs(self):
        n, rd, V = self.n, self.rd, self.V
        gt, i0, i1, A, X, Y = self.gt, self.i0, self.i1, self.A, self.X, self.Y
        f = [(0, 0), (0, 0), (0, 0)]
        for g in range(len(gt)):
            if rd < n:
                bit = (i0[g] >> rd) & 1
                two = gatefn(gt[g], V.at_m1(i0[g]), Y[g])
            else:
                bit = (i1[g] >> (rd - n)) & 1
                two = gatefn(gt[g], X[g], V.at_m1(i1[g]))
            third = sub((0, 0), A[g]) if bit else scale(A[g], 2)
            f[2] = add(f[2], mul(two, third))
            f[bit] = add(f[bit], mul(A[g], gatefn(gt[g], X[g], Y[g])))
        f = [mul(v, self.beta) for v in f]
        return interpolate_quadratic(f[0], f[1], f[2])

    def next_round(self, r):
        n, rd, V = self.n, self.rd, self.V
        V.next_round(r)
        for g in range(len(self.gt)):
            if rd < n:
                bit = (self.i0[g] >> rd) & 1
                self.X[g] = V.outputs[self.i0[g]] if rd < n - 1 else V.prev
            else:
                bit = (self.i1[g] >> (rd - n)) & 1
                self.Y[g] = V.outputs[self.i1[g]] if rd < 2 * n - 1 else V.prev
            self.A[g] = mul(self.A[g], r if bit else sub(ONE, r))
        self.w.append(r)
        self.rd += 1

    def line(self):
        n = self.n
        w1, w2 = self.w[:n], self.w[n:2 * n]
        hv = [self.V.v1v2[0], self.V.v1v2[1]]
        for t in range(2, n + 1):
            pt = [add(a, scale(sub(b, a), t)) for a, b in zip(w1, w2)]
            hv.append(mle(self.wires, pt))
        return interpolate(hv)


def late_rounds(wires, beta, zg, gates, n_in_bits, chal):
    """(per-round coefficients [2 n][3], line coefficients [n + 1], v1, v2)

    wires: the 2^n_in_bits input values after the early rounds (Fp2 pairs);
    beta: beta's final value; zg: per-gate weights (accum_z1); gates: (type, in0,
    in1) lists; chal: the 2 n_in_bits late challenges."""
    L = LateRounds(wires, beta, zg, gates, n_in_bits)
    coefs = []
    for rd in range(2 * n_in_bits):
        coefs.append(L.coefs())
        L.next_round(chal[rd])
    return coefs, L.line(), L.V.v1v2[0], L.V.v1v2[1]
