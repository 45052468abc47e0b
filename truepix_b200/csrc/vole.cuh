// VOLE-committed sumcheck rounds of the reference prover
// (TruePix-main/libTruePix/circuitnizkvec_vole.py:396-418 with create_pok_temp
// :112-133 and create_eq_proof :220-233; ExtVOLECommit commit d = m - u, tag v;
// util.interpolate_cubic / interpolate_quadratic :91-136), one frame at a time,
// host and device alike:
//   the round polynomial's coefficients from the prover's values at 0, 1, -1
//   (and 2 in an early round); each coefficient committed with the frame's next
//   correlation (d = c - u put into the transcript, the tag v kept, running sums
//   of tags and coefficients kept for the final proof of knowledge); the
//   equality proof of the tags' value at 0 + 1 against the previous round's
//   (challenge rand_ext("eq"), (prev - now) * e put, or now * e in the first
//   round); the fold challenge rand_ext(label); the next previous value, the
//   tags' polynomial at the challenge (Horner).
#pragma once
#include <stdint.h>

#include "fp2.cuh"
#include "transcript.cuh"

namespace tp {
namespace vole {

struct State {
    unsigned long long idx;   // next correlation
    unsigned has_prev, bad;   // bad: the correlations ran out (nothing done)
    fp2 prev;
    fp2 v_elem[4], out_elem[4];   // running sums of tags / coefficients (the final proof of knowledge)
};
static_assert(sizeof(State) == 160, "vole state layout");

constexpr u64 kHalf = 1ull << 60;                  // 2^-1 mod p
constexpr u64 kThird = 1537228672809129301ull;     // 3^-1 mod p

// util.interpolate_cubic: values at 0, 1, -1, 2 -> c0..c3
TP_HD void interpolate_cubic(fp2 f0, fp2 f1, fp2 fm1, fp2 f2, fp2 c[4])
{
    const fp2 a = f2sub(f2zero(), fm1);
    const fp2 b = f2scale(f2add(f1, fm1), kHalf);
    const fp2 cc = f2scale(f2add(f1, a), kHalf);
    const fp2 d = f2scale(f2add(f2, a), kThird);
    const fp2 c2 = f2sub(b, f0);
    const fp2 c3 = f2scale(f2sub(f2sub(d, cc), c2), kHalf);
    c[0] = f0;
    c[1] = f2sub(cc, c3);
    c[2] = c2;
    c[3] = c3;
}

// util.interpolate_quadratic: values at 0, 1, -1 -> c0..c2
TP_HD void interpolate_quadratic(fp2 f0, fp2 f1, fp2 fm1, fp2 c[3])
{
    const fp2 a = f2sub(f2zero(), f0);
    const fp2 c2 = f2add(f2scale(f2add(f1, fm1), kHalf), a);
    c[0] = f0;
    c[1] = f2add(f2sub(f1, c2), a);
    c[2] = c2;
}

// "sc-<layer>-<round>"
TP_HD fs::Label sc_label(int layer, int round)
{
    fs::Label L = fs::label_lit("sc-");
    fs::label_decimal(L, layer);
    fs::label_push(L, '-');
    fs::label_decimal(L, round);
    return L;
}

// "tau-<layer>"
TP_HD fs::Label tau_label(int layer)
{
    fs::Label L = fs::label_lit("tau-");
    fs::label_decimal(L, layer);
    return L;
}

// ExtVOLECommit.commit with one repetition: the tag v and d = m - u of the next
// correlation (the caller checks that one remains)
TP_HD fp2 commit(State& w, fp2 m, const fp2* u, const fp2* v, fp2* tag)
{
    *tag = v[w.idx];
    const fp2 d = f2sub(m, u[w.idx]);
    ++w.idx;
    return d;
}

// One committed round on the coefficients c[0..n_coef) (n_coef <= 4) with the
// frame's correlations u, v (count entries). Returns false, sets w.bad and
// leaves the transcript untouched when fewer than n_coef correlations remain.
// proof (optional): the n_coef values d, then the equality value.
TP_HD bool round(fs::State& s, State& w, const fp2* c, int n_coef, const fp2* u, const fp2* v, long long count,
                 const fs::Label& label, fp2* proof, fp2* r_out)
{
    if (w.bad || w.idx + (unsigned long long)n_coef > (unsigned long long)count) {
        w.bad = 1;
        *r_out = f2zero();
        return false;
    }
    fp2 tag[4];
    for (int k = 0; k < n_coef; ++k) {
        tag[k] = v[w.idx];
        const fp2 dm = f2sub(c[k], u[w.idx]);
        ++w.idx;
        fs::put_fp2(s, dm.re, dm.im);
        if (proof) proof[k] = dm;
        w.v_elem[k] = f2add(w.v_elem[k], tag[k]);
        w.out_elem[k] = f2add(w.out_elem[k], c[k]);
    }
    fp2 now = tag[0];
    for (int k = 0; k < n_coef; ++k) now = f2add(now, tag[k]);
    const fp2 e = fs::rand_fp2(s, fs::label_lit("eq"));
    const fp2 vz = w.has_prev ? f2mul(f2sub(w.prev, now), e) : f2mul(now, e);
    fs::put_fp2(s, vz.re, vz.im);
    if (proof) proof[n_coef] = vz;
    const fp2 r = fs::rand_fp2(s, label);
    fp2 p = tag[n_coef - 1];
    for (int k = n_coef - 2; k >= 0; --k) p = f2add(f2mul(p, r), tag[k]);
    w.prev = p;
    w.has_prev = 1;
    *r_out = r;
    return true;
}

}  // namespace vole
}  // namespace tp
