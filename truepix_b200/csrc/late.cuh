// Late rounds of the GKR input layer's sumcheck and the line projection that
// ends it, one frame per CTA (TruePix-main/libTruePix/layerprover.py:231-290,
// gateprover.py:105-185, layercompute.py:16-247).
//
// After the early rounds every wire w holds one value V[w] (the input table at
// the copy point) and beta one value; gate g carries a weight A_g (its z1 eq
// value). Rounds 0..n-1 bind the bits of in0 (LSB first), rounds n..2n-1 the
// bits of in1. In round j of a phase, with T the table V folded by that phase's
// earlier challenges and b the gate's input bit j:
//   x / y      the gate's input values: in phase 1 x = T[in0 >> j] and
//              y = V[in1]; in phase 2 x = V(w1) (phase 1's last value) and
//              y = T[in1 >> j]
//   at 0 or 1  A_g * gate(x, y) added to the value at b
//   at -1      gate(x', y') * (b ? -A_g : 2 A_g), the bound input taken at -1
//              along bit j: 2 T[2k] - T[2k + 1], k = in >> (j + 1)
// summed over gates, times beta, interpolated at 0, 1, -1 (util.py:91-113);
// then the challenge r folds T (T'[k] = T[2k] + r (T[2k+1] - T[2k])) and
// A_g *= (b ? r : 1 - r). Phase 2 starts again from V. The line projection: the
// input values on the line w1 + t (w2 - w1), t = 0..n (t = 0, 1 are the two
// phases' last values, the others multilinear evaluations of V), and the
// coefficients of the degree-n polynomial through them.
//
// The CTA's work is written as steps between barriers, each step a function of
// (workspace, thread index) in which a thread reads only what earlier steps
// wrote and writes only its own slots: the device runs them with __syncthreads()
// between, a host loop over the thread indices runs the same code.
#pragma once
#include <stdint.h>

#include "fp2.cuh"
#include "transcript.cuh"
#include "vole.cuh"

namespace tp {
namespace late {

constexpr int kThreads = 256;
constexpr int kMaxInBits = 9;
constexpr int kMaxWires = 1 << kMaxInBits;
constexpr int kMaxGates = 768;

// packed gate table: type << 28 | in0 << 14 | in1
struct Gates {
    uint32_t g[kMaxGates];
};

// native_fp2_core.hpp:32-51 on canonical Fp2 values
TP_HD fp2 gatefn(unsigned t, fp2 x, fp2 y)
{
    const fp2 one = mk(1, 0);
    switch (t) {
    case 0: return f2mul(x, y);
    case 1: return f2add(x, y);
    case 2: return f2sub(x, y);
    case 3: return x;
    case 4: return y;
    case 5: return f2sub(f2add(x, y), f2mul(x, y));
    case 6: return f2sub(f2add(x, y), f2dbl(f2mul(x, y)));
    case 7: return f2sub(one, x);
    case 8: return f2sub(one, f2mul(x, y));
    case 9: return f2sub(f2add(one, f2mul(x, y)), f2add(x, y));
    case 10: return f2sub(f2add(one, f2dbl(f2mul(x, y))), f2add(x, y));
    case 11: return f2mul(f2sub(one, x), y);
    default: return x;
    }
}

// gateprover_vole.py p_com_gatefn_ (GateFunctionsPC, :706-720): a gate's value on
// committed x, y and x*y, by the native type index
TP_HD fp2 pc_gatefn(unsigned t, fp2 x, fp2 y, fp2 xy)
{
    const fp2 one = mk(1, 0);
    switch (t) {
    case 0: return xy;
    case 1: return f2add(x, y);
    case 2: return f2sub(x, y);
    case 3: return x;
    case 4: return y;
    case 5: return f2sub(f2add(x, y), xy);
    case 6: return f2sub(f2add(x, y), f2dbl(xy));
    case 7: return f2sub(one, x);
    case 8: return f2sub(one, xy);
    case 9: return f2sub(f2add(one, xy), f2add(x, y));
    case 10: return f2sub(f2add(one, f2dbl(xy)), f2add(x, y));
    case 11: return f2sub(y, xy);
    default: return x;
    }
}

// one frame's inputs and outputs (pointers already at the frame)
struct Frame {
    const fp2* wires;      // 2^n
    const fp2* beta;       // 1
    const fp2* zg;         // n_gates
    const fp2* chal;       // 2n given challenges, or null: drawn by the VOLE rounds
    fs::State* st;         // VOLE mode: the frame's transcript,
    vole::State* vs;       // its VOLE state,
    const fp2* u;          // and correlations (count each)
    const fp2* v;
    fp2* coefs;            // 2n x 3
    fp2* h;                // n + 1
    fp2* chal_out;         // 2n
    fp2* proof;            // VOLE mode, optional: 2n x 4 (three d, the equality value)
    // the layer's closing proofs (VOLE mode, optional)
    const fp2* z2;         // nb: the copy part of the layer's point
    const fp2* w3;         // the early challenges: w3[k * w3_stride], k < nb
    long long w3_stride;
    fp2* closing;          // n + 10 (zero-knowledge prover: n + 15) values in the order they are put
    fp2* point;            // n + nb: the input point
    fp2* tag;              // 1: its tag
};

struct Shape {
    int n;           // input bits
    int n_gates;
    long long count; // correlations per frame
    int layer;       // labels "sc-<layer>-<round0 + round>"
    int round0;      // the early rounds before (their count: nb)
    int zk;          // closing proofs of the zero-knowledge prover (circuitnizkvec_vole_ZK.py)
};

// the CTA's workspace (shared memory on the device)
struct Work {
    fp2 V[kMaxWires];
    fp2 T[kMaxWires];
    fp2 Tn[kMaxWires / 2];
    fp2 A[kMaxGates];
    fp2 red[3][kThreads];
    fp2 w[2 * kMaxInBits];     // the challenges
    fp2 pt[kMaxInBits];        // a point on the line
    fp2 h[kMaxInBits + 1];     // the line's values
    fp2 hc[kMaxInBits + 1];    // its coefficients
    fp2 vv[kMaxInBits + 1];    // closing: the coefficients' tags
    fp2 pr[3];                 // closing: tags of x, of the line's sum, of the product
    fp2 beta, v1, r;
    fs::State st;
    vole::State vs;
    int bad;
};

static_assert(sizeof(Work) <= 48 * 1024, "the workspace fits the static shared memory of a CTA");

// ---- steps -------------------------------------------------------------------

TP_HD void step_load(Work& w, const Frame& f, const Shape& sh, int tid)
{
    const int W = 1 << sh.n;
    for (int k = tid; k < W; k += kThreads) w.V[k] = w.T[k] = f.wires[k];
    for (int g = tid; g < sh.n_gates; g += kThreads) w.A[g] = f.zg[g];
    if (tid == 0) {
        w.beta = *f.beta;
        w.bad = 0;
        if (!f.chal) {
            w.st = *f.st;
            w.vs = *f.vs;
        }
    }
}

// per-thread partial values at 0, 1, -1 of round rd
TP_HD void step_sums(Work& w, const uint32_t* gates, const Shape& sh, int rd, int tid)
{
    const bool ph1 = rd < sh.n;
    const int j = ph1 ? rd : rd - sh.n;
    fp2 s0 = f2zero(), s1 = f2zero(), s2 = f2zero();
    for (int g = tid; g < sh.n_gates; g += kThreads) {
        const uint32_t t = gates[g];
        const unsigned type = t >> 28;
        const int in0 = (int)((t >> 14) & 0x3FFFu), in1 = (int)(t & 0x3FFFu);
        const int idx = ph1 ? in0 : in1;
        const int bit = (idx >> j) & 1, k = idx >> (j + 1);
        const fp2 t0 = w.T[2 * k], t1 = w.T[2 * k + 1];
        const fp2 cur = bit ? t1 : t0, m1 = f2at_m1(t0, t1);
        fp2 v01, two;
        if (ph1) {
            const fp2 y = w.V[in1];
            v01 = gatefn(type, cur, y);
            two = gatefn(type, m1, y);
        } else {
            v01 = gatefn(type, w.v1, cur);
            two = gatefn(type, w.v1, m1);
        }
        const fp2 a = w.A[g];
        v01 = f2mul(a, v01);
        s2 = f2add(s2, f2mul(two, bit ? f2sub(f2zero(), a) : f2dbl(a)));
        if (bit)
            s1 = f2add(s1, v01);
        else
            s0 = f2add(s0, v01);
    }
    w.red[0][tid] = s0;
    w.red[1][tid] = s1;
    w.red[2][tid] = s2;
}

// one level of the tree sum: threads below `half` add the slot `half` above
TP_HD void step_reduce(Work& w, int half, int tid)
{
    if (tid < half)
        for (int q = 0; q < 3; ++q) w.red[q][tid] = f2add(w.red[q][tid], w.red[q][tid + half]);
}

// thread 0: the round's coefficients and its challenge
TP_HD void step_head(Work& w, const Frame& f, const Shape& sh, int rd)
{
    fp2 c[3];
    vole::interpolate_quadratic(f2mul(w.red[0][0], w.beta), f2mul(w.red[1][0], w.beta),
                                f2mul(w.red[2][0], w.beta), c);
    for (int q = 0; q < 3; ++q) f.coefs[3 * rd + q] = c[q];
    fp2 r;
    if (f.chal) {
        r = f.chal[rd];
    } else {
        const fs::Label label = vole::sc_label(sh.layer, sh.round0 + rd);
        if (!vole::round(w.st, w.vs, c, 3, f.u, f.v, sh.count, label, f.proof ? f.proof + 4 * rd : nullptr,
                         &r))
            w.bad = 1;
    }
    w.r = r;
    w.w[rd] = r;
    f.chal_out[rd] = r;
}

// fold T by the challenge into Tn, update the gates' weights
TP_HD void step_fold(Work& w, const uint32_t* gates, const Shape& sh, int rd, int tid)
{
    const bool ph1 = rd < sh.n;
    const int j = ph1 ? rd : rd - sh.n;
    const int half = (1 << sh.n) >> (j + 1);
    const fp2 r = w.r, one_m_r = f2sub(mk(1, 0), r);
    for (int k = tid; k < half; k += kThreads) w.Tn[k] = f2fold(w.T[2 * k], w.T[2 * k + 1], r);
    for (int g = tid; g < sh.n_gates; g += kThreads) {
        const uint32_t t = gates[g];
        const int idx = ph1 ? (int)((t >> 14) & 0x3FFFu) : (int)(t & 0x3FFFu);
        w.A[g] = f2mul(w.A[g], ((idx >> j) & 1) ? r : one_m_r);
    }
}

TP_HD void step_copy(Work& w, int n_entries, int tid)
{
    for (int k = tid; k < n_entries; k += kThreads) w.T[k] = w.Tn[k];
}

TP_HD void step_restart(Work& w, const Shape& sh, int tid)
{
    for (int k = tid; k < (1 << sh.n); k += kThreads) w.T[k] = w.V[k];
}

// thread 0: the point w1 + t (w2 - w1)
TP_HD void step_line_point(Work& w, const Shape& sh, int t)
{
    for (int j = 0; j < sh.n; ++j) w.pt[j] = f2add(w.w[j], f2scale(f2sub(w.w[sh.n + j], w.w[j]), (u64)t));
}

// fold T by coordinate j of the line point into Tn
TP_HD void step_fold_point(Work& w, const Shape& sh, int j, int tid)
{
    const int half = (1 << sh.n) >> (j + 1);
    const fp2 r = w.pt[j];
    for (int k = tid; k < half; k += kThreads) w.Tn[k] = f2fold(w.T[2 * k], w.T[2 * k + 1], r);
}

// thread 0: coefficients (constant first) of the polynomial through (t, h[t]),
// t = 0..n, by Newton's divided differences on the nodes 0..n
TP_HD void step_interpolate(Work& w, const Frame& f, const Shape& sh)
{
    const int n = sh.n;
    fp2 d[kMaxInBits + 1], c[kMaxInBits + 1];
    for (int i = 0; i <= n; ++i) d[i] = w.h[i];
    for (int lvl = 1; lvl <= n; ++lvl) {
        const u64 inv = finv((u64)lvl);
        for (int i = n; i >= lvl; --i) d[i] = f2scale(f2sub(d[i], d[i - 1]), inv);
    }
    // c(t) = d[n]; then c(t) <- c(t) (t - i) + d[i] for i = n - 1..0
    for (int i = 0; i <= n; ++i) c[i] = f2zero();
    c[0] = d[n];
    int deg = 0;
    for (int i = n - 1; i >= 0; --i) {
        c[deg + 1] = c[deg];
        for (int k = deg; k >= 1; --k) c[k] = f2sub(c[k - 1], f2scale(c[k], (u64)i));
        c[0] = f2add(f2sub(f2zero(), f2scale(c[0], (u64)i)), d[i]);
        ++deg;
    }
    for (int i = 0; i <= n; ++i) f.h[i] = w.hc[i] = c[i];
}

// ---- the layer's closing proofs (circuitnizkvec_vole.py:433-500, one layer) ----

// index of the equality value among the closing values (before it: two
// commitments, n commitments, two proof-of-knowledge values, with zk three mask
// commitments, the product proof's two values and with zk the masks' two)
TP_HD int close_eq_index(const Shape& sh) { return sh.n + 6 + 5 * (sh.zk != 0); }

// thread 0: create_final_prod_pok (:175-218; the zero-knowledge prover's,
// circuitnizkvec_vole_ZK.py:188-247, adds three mask commitments of 1 and their
// product proof) on the line's coefficients
TP_HD void step_close_commit(Work& w, const Frame& f, const Shape& sh)
{
    const int n = sh.n;
    const int zk = sh.zk != 0;
    if (w.vs.bad || w.vs.idx + (unsigned long long)(n + 2 + 3 * zk) > (unsigned long long)sh.count) {
        w.vs.bad = 1;
        w.bad = 1;
        return;
    }
    fp2* out = f.closing;
    fp2 sval = f2zero();
    for (int k = 0; k <= n; ++k) sval = f2add(sval, w.hc[k]);
    const fp2 prod = f2mul(w.hc[0], sval);
    fp2 v1, v3;
    out[0] = vole::commit(w.vs, w.hc[0], f.u, f.v, &v1);
    out[1] = vole::commit(w.vs, prod, f.u, f.v, &v3);
    fs::put_fp2(w.st, out[0].re, out[0].im);
    fs::put_fp2(w.st, out[1].re, out[1].im);
    fp2 rest_sum = f2zero(), rest_v = f2zero();
    w.vv[0] = v1;
    for (int k = 1; k <= n; ++k) {
        out[1 + k] = vole::commit(w.vs, w.hc[k], f.u, f.v, &w.vv[k]);
        fs::put_fp2(w.st, out[1 + k].re, out[1 + k].im);
        rest_sum = f2add(rest_sum, w.hc[k]);
        rest_v = f2add(rest_v, w.vv[k]);
    }
    const fp2 c = fs::rand_fp2(w.st, fs::label_lit("pok-vec"));
    out[n + 2] = f2mul(rest_sum, c);
    out[n + 3] = f2mul(rest_v, c);
    fs::put_fp2(w.st, out[n + 2].re, out[n + 2].im);
    fs::put_fp2(w.st, out[n + 3].re, out[n + 3].im);
    int k = n + 4;
    fp2 mtag[3];
    if (zk) {
        for (int q = 0; q < 3; ++q) {
            out[k] = vole::commit(w.vs, mk(1, 0), f.u, f.v, &mtag[q]);
            fs::put_fp2(w.st, out[k].re, out[k].im);
            ++k;
        }
    }
    fp2 vsum = f2zero();
    for (int q = 0; q <= n; ++q) vsum = f2add(vsum, w.vv[q]);
    // prod_finish on (x, sum, x * sum) with tags (v1, sum of tags, v3)
    out[k] = f2mul(v1, vsum);
    out[k + 1] = f2sub(f2add(f2mul(w.hc[0], vsum), f2mul(sval, v1)), v3);
    fs::put_fp2(w.st, out[k].re, out[k].im);
    fs::put_fp2(w.st, out[k + 1].re, out[k + 1].im);
    if (zk) {   // prod_finish on (1, 1, 1) with the masks' tags
        out[k + 2] = f2mul(mtag[0], mtag[1]);
        out[k + 3] = f2sub(f2add(mtag[1], mtag[0]), mtag[2]);
        fs::put_fp2(w.st, out[k + 2].re, out[k + 2].im);
        fs::put_fp2(w.st, out[k + 3].re, out[k + 3].im);
    }
    w.pr[0] = v1;
    w.pr[1] = vsum;
    w.pr[2] = v3;
}

// per-thread partial sums of the wiring predicates' multilinear extensions times
// the committed gate values (CircuitVerifier.eval_mlext, circuitverifier.py:224-290,
// with GateFunctionsPC): sum over gates of z1eq_g * eq(w1, in0_g) * eq(w2, in1_g)
// * pc_gate(v1, sum, v3)
TP_HD void step_close_sums(Work& w, const Frame& f, const uint32_t* gates, const Shape& sh, int tid)
{
    const int n = sh.n;
    fp2 s = f2zero();
    const fp2 one = mk(1, 0);
    for (int g = tid; g < sh.n_gates; g += kThreads) {
        const uint32_t t = gates[g];
        const int in0 = (int)((t >> 14) & 0x3FFFu), in1 = (int)(t & 0x3FFFu);
        fp2 e = f.zg[g];
        for (int j = 0; j < n; ++j) {
            e = f2mul(e, ((in0 >> j) & 1) ? w.w[j] : f2sub(one, w.w[j]));
            e = f2mul(e, ((in1 >> j) & 1) ? w.w[n + j] : f2sub(one, w.w[n + j]));
        }
        s = f2add(s, f2mul(e, pc_gatefn(t >> 28, w.pr[0], w.pr[1], w.pr[2])));
    }
    w.red[0][tid] = s;
    w.red[1][tid] = f2zero();
    w.red[2][tid] = f2zero();
}

// thread 0: the equality proof against the last round's value, tau, the proof of
// knowledge of all round coefficients, the input point and its value proof
TP_HD void step_close_tail(Work& w, const Frame& f, const Shape& sh)
{
    const int n = sh.n, nb = sh.round0;
    fp2* out = f.closing + (close_eq_index(sh) - (n + 6));   // out[n + 6]: the equality value
    // beta's factor: prod over the early challenges of 2 w z + 1 - (w + z)
    fp2 mz = mk(1, 0);
    for (int k = 0; k < nb; ++k) {
        const fp2 wk = f.w3[k * f.w3_stride], zk = f.z2[k];
        mz = f2mul(mz, f2sub(f2add(f2dbl(f2mul(wk, zk)), mk(1, 0)), f2add(wk, zk)));
    }
    const fp2 tv = f2mul(w.red[0][0], mz);
    const fp2 e = fs::rand_fp2(w.st, fs::label_lit("eq"));
    out[n + 6] = f2mul(f2sub(w.vs.prev, tv), e);
    fs::put_fp2(w.st, out[n + 6].re, out[n + 6].im);
    const fp2 tau = fs::rand_fp2(w.st, vole::tau_label(sh.layer));
    fp2 tag = w.vv[n];
    for (int k = n - 1; k >= 0; --k) tag = f2add(f2mul(tag, tau), w.vv[k]);
    for (int j = 0; j < n; ++j) f.point[j] = f2add(w.w[j], f2mul(f2sub(w.w[n + j], w.w[j]), tau));
    for (int k = 0; k < nb; ++k) f.point[n + k] = f.w3[k * f.w3_stride];
    // create_pok_final
    fp2 osum = f2zero(), vsum = f2zero();
    for (int k = 0; k < 4; ++k) {
        osum = f2add(osum, w.vs.out_elem[k]);
        vsum = f2add(vsum, w.vs.v_elem[k]);
    }
    const fp2 c = fs::rand_fp2(w.st, fs::label_lit("pok-final"));
    out[n + 7] = f2mul(osum, c);
    out[n + 8] = f2mul(vsum, c);
    fs::put_fp2(w.st, out[n + 7].re, out[n + 7].im);
    fs::put_fp2(w.st, out[n + 8].re, out[n + 8].im);
    // put(["gkr_input_point", [[re, im], ...]]): a string, then every coordinate's two ints
    fs::put_label(w.st, fs::label_lit("gkr_input_point"));
    for (int k = 0; k < n + nb; ++k) {
        fs::absorb_byte(w.st, 0x02);
        fs::absorb_le(w.st, f.point[k].re, 8);
        fs::absorb_byte(w.st, 0x02);
        fs::absorb_le(w.st, f.point[k].im, 8);
    }
    // create_input_value_proof
    const fp2 civ = fs::rand_fp2(w.st, fs::label_lit("input-val"));
    out[n + 9] = f2mul(tag, civ);
    fs::put_fp2(w.st, out[n + 9].re, out[n + 9].im);
    w.vs.prev = tag;
    *f.tag = tag;
}

// thread 0: the VOLE state and transcript back to the frame
TP_HD void step_store(Work& w, const Frame& f)
{
    if (!f.chal) {
        *f.st = w.st;
        *f.vs = w.vs;
    }
}

// The whole late phase of one frame. par.all(fn) runs fn(thread index) on every
// thread of the CTA and then waits at a barrier; par.one(fn) runs fn on thread 0
// and waits. Every branch below depends only on values all threads read alike
// after a barrier.
#pragma nv_exec_check_disable
template <class Par>
TP_HD void run_frame(Work& w, const Frame& f, const Shape& sh, const uint32_t* gates, const Par& par)
{
    const int n = sh.n, W = 1 << n;
    par.all([&](int tid) { step_load(w, f, sh, tid); });
    for (int rd = 0; rd < 2 * n; ++rd) {
        par.all([&](int tid) { step_sums(w, gates, sh, rd, tid); });
        for (int half = kThreads / 2; half > 0; half >>= 1) par.all([&](int tid) { step_reduce(w, half, tid); });
        par.one([&] { step_head(w, f, sh, rd); });
        if (w.bad) break;
        par.all([&](int tid) { step_fold(w, gates, sh, rd, tid); });
        const int j = rd < n ? rd : rd - n;
        par.all([&](int tid) { step_copy(w, W >> (j + 1), tid); });
        if (rd == n - 1) {
            par.one([&] { w.v1 = w.h[0] = w.T[0]; });
            par.all([&](int tid) { step_restart(w, sh, tid); });
        }
        if (rd == 2 * n - 1) par.one([&] { w.h[1] = w.T[0]; });
    }
    if (!w.bad) {
        for (int t = 2; t <= n; ++t) {
            par.one([&] { step_line_point(w, sh, t); });
            par.all([&](int tid) { step_restart(w, sh, tid); });
            for (int j = 0; j < n; ++j) {
                par.all([&](int tid) { step_fold_point(w, sh, j, tid); });
                par.all([&](int tid) { step_copy(w, W >> (j + 1), tid); });
            }
            par.one([&] { w.h[t] = w.T[0]; });
        }
        par.one([&] { step_interpolate(w, f, sh); });
        if (f.closing) {
            par.one([&] { step_close_commit(w, f, sh); });
            if (!w.bad) {
                par.all([&](int tid) { step_close_sums(w, f, gates, sh, tid); });
                for (int half = kThreads / 2; half > 0; half >>= 1)
                    par.all([&](int tid) { step_reduce(w, half, tid); });
                par.one([&] { step_close_tail(w, f, sh); });
            }
        }
    }
    par.one([&] { step_store(w, f); });
}

}  // namespace late
}  // namespace tp
