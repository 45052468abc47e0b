/*
 * CPU oracle for the GKR Fp2 kernels -- TEST INFRASTRUCTURE ONLY.
 *
 * This file restates, in plain C, the algorithms of the reference CPU library
 * `TruePix-main/native_fp2/native_fp2_core.hpp` (arithmetic from
 * `TruePix-main/native_fp2/fp61.cuh`). It is the checker for the CUDA path:
 * only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg may load
 * it. The shipped library never links or calls it.
 *
 * The restatement is deliberately literal (per-gate evaluation of the 13 gate
 * functions at the four points 0, 1, -1, 2) so that it checks the CUDA path's
 * algebraic re-arrangement of the same sums instead of sharing it.
 *
 * Parity pin: tests/golden/ holds outputs of the reference library itself,
 * compiled from source by oracle/Makefile into oracle/_ref/ and run by
 * tests/golden/gen_golden.py; tests/test_oracle.py checks this file against
 * them.
 *
 * Field: p = 2^61 - 1, Fp2 = Fp[i]/(i^2 + 1), all values canonical in [0, p).
 */
#include <stddef.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef uint64_t u64;
typedef unsigned __int128 u128;

#define P61 ((u64)0x1FFFFFFFFFFFFFFFull)

typedef struct { u64 re, im; } f2;

/* fp61.cuh:36-50 -- canonical add/sub/mul mod 2^61-1 */
static inline u64 canon(u64 x) { return x >= P61 ? x - P61 : x; }
static inline u64 red64(u64 x) { return canon((x & P61) + (x >> 61)); }
static inline u64 fadd(u64 a, u64 b) { return canon(a + b); }
static inline u64 fsub(u64 a, u64 b) { return canon(a + P61 - b); }
static inline u64 fmul(u64 a, u64 b)
{
    u128 t = (u128)a * b;
    u64 lo = (u64)t & P61;
    u64 hi = (u64)(t >> 61);
    return canon(lo + hi);
}

/* fp61.cuh:96-119 -- Fp2 with i^2 = -1 (Karatsuba; any exact product is equal) */
static inline f2 F(u64 re, u64 im) { f2 r; r.re = re; r.im = im; return r; }
static inline f2 f2add(f2 a, f2 b) { return F(fadd(a.re, b.re), fadd(a.im, b.im)); }
static inline f2 f2sub(f2 a, f2 b) { return F(fsub(a.re, b.re), fsub(a.im, b.im)); }
static inline f2 f2mul(f2 a, f2 b)
{
    u64 ac = fmul(a.re, b.re), bd = fmul(a.im, b.im);
    u64 s = fmul(fadd(a.re, a.im), fadd(b.re, b.im));
    return F(fsub(ac, bd), fsub(fsub(s, ac), bd));
}

/* native_fp2_core.hpp:32-51 -- the 13 gate functions (default: x) */
static f2 gatefn(int tp, f2 x, f2 y)
{
    const f2 one = F(1, 0), two = F(2, 0);
    switch (tp) {
    case 0: return f2mul(x, y);
    case 1: return f2add(x, y);
    case 2: return f2sub(x, y);
    case 3: return x;
    case 4: return y;
    case 5: return f2sub(f2add(x, y), f2mul(x, y));
    case 6: return f2sub(f2add(x, y), f2mul(two, f2mul(x, y)));
    case 7: return f2sub(one, x);
    case 8: return f2sub(one, f2mul(x, y));
    case 9: return f2sub(f2add(one, f2mul(x, y)), f2add(x, y));
    case 10: return f2sub(f2add(one, f2mul(two, f2mul(x, y))), f2add(x, y));
    case 11: return f2mul(f2sub(one, x), y);
    default: return x;
    }
}

/* x + r*(y - x): the fold of one pair (native_fp2_core.hpp:53-64) */
static inline f2 fold1(f2 x, f2 y, f2 r) { return f2add(x, f2mul(r, f2sub(y, x))); }
static inline f2 at_m1(f2 a, f2 b) { return f2sub(f2add(a, a), b); }  /* fold at -1 */
static inline f2 at_2(f2 a, f2 b) { return f2sub(f2add(b, b), a); }   /* fold at 2 */

void oracle_fp2_fold(const u64* in_re, const u64* in_im, size_t n_out,
                     u64 r_re, u64 r_im, u64* out_re, u64* out_im)
{
    const f2 r = F(r_re, r_im);
    for (size_t i = 0; i < n_out; ++i) {
        f2 o = fold1(F(in_re[2 * i], in_im[2 * i]), F(in_re[2 * i + 1], in_im[2 * i + 1]), r);
        out_re[i] = o.re;
        out_im[i] = o.im;
    }
}

/* native_fp2_core.hpp:66-80 */
void oracle_fp2_expand(const u64* in_re, const u64* in_im, size_t n_src, size_t ncopies,
                       u64* out_re, u64* out_im)
{
    for (size_t i = 0; i < n_src; ++i)
        for (size_t j = 0; j < ncopies; ++j) {
            out_re[i * ncopies + j] = in_re[i];
            out_im[i * ncopies + j] = in_im[i];
        }
}

/* native_fp2_core.hpp:82-137 -- claim with caller-supplied -1 / 2 tables */
void oracle_fp2_sumcheck_early(int n_gates, const int* type, const int* in0, const int* in1,
                               const u64* z1_re, const u64* z1_im, int n_copies, int n_wires,
                               const u64* v_re, const u64* v_im,
                               const u64* f0_re, const u64* f0_im,
                               const u64* f1_re, const u64* f1_im,
                               const u64* b_re, const u64* b_im,
                               const u64* bf0_re, const u64* bf0_im,
                               const u64* bf1_re, const u64* bf1_im, u64 out8[8])
{
    (void)n_wires;
    const size_t n = (size_t)n_copies, h = n >> 1;
    f2 acc[4] = {F(0, 0), F(0, 0), F(0, 0), F(0, 0)};
    for (size_t c = 0; c < n; c += 2) {
        size_t half = c >> 1;
        f2 v[4] = {F(0, 0), F(0, 0), F(0, 0), F(0, 0)};
        for (int g = 0; g < n_gates; ++g) {
            size_t a = (size_t)in0[g], b = (size_t)in1[g];
            f2 z = F(z1_re[g], z1_im[g]);
            v[0] = f2add(v[0], f2mul(gatefn(type[g], F(v_re[a * n + c], v_im[a * n + c]),
                                                 F(v_re[b * n + c], v_im[b * n + c])), z));
            v[1] = f2add(v[1], f2mul(gatefn(type[g], F(v_re[a * n + c + 1], v_im[a * n + c + 1]),
                                                 F(v_re[b * n + c + 1], v_im[b * n + c + 1])), z));
            v[2] = f2add(v[2], f2mul(gatefn(type[g], F(f0_re[a * h + half], f0_im[a * h + half]),
                                                 F(f0_re[b * h + half], f0_im[b * h + half])), z));
            v[3] = f2add(v[3], f2mul(gatefn(type[g], F(f1_re[a * h + half], f1_im[a * h + half]),
                                                 F(f1_re[b * h + half], f1_im[b * h + half])), z));
        }
        acc[0] = f2add(acc[0], f2mul(v[0], F(b_re[c], b_im[c])));
        acc[1] = f2add(acc[1], f2mul(v[1], F(b_re[c + 1], b_im[c + 1])));
        acc[2] = f2add(acc[2], f2mul(v[2], F(bf0_re[half], bf0_im[half])));
        acc[3] = f2add(acc[3], f2mul(v[3], F(bf1_re[half], bf1_im[half])));
    }
    for (int t = 0; t < 4; ++t) {
        out8[2 * t] = acc[t].re;
        out8[2 * t + 1] = acc[t].im;
    }
}

/* native_fp2_core.hpp:139-161 -- eq table, bit j of the index selects z_j */
void oracle_fp2_compute_beta(const u64* z_re, const u64* z_im, int n_z, u64 init_re, u64 init_im,
                             u64* out_re, u64* out_im)
{
    if (n_z <= 0) return;
    out_re[0] = init_re;
    out_im[0] = init_im;
    size_t cur = 1;
    for (int j = 0; j < n_z; ++j) {
        f2 z = F(z_re[j], z_im[j]);
        f2 omz = f2sub(F(1, 0), z);
        for (size_t i = 0; i < cur; ++i) {
            f2 base = F(out_re[i], out_im[i]);
            f2 lo = f2mul(base, omz), hi = f2mul(base, z);
            out_re[i] = lo.re; out_im[i] = lo.im;
            out_re[i + cur] = hi.re; out_im[i + cur] = hi.im;
        }
        cur <<= 1;
    }
}

/* native_fp2_core.hpp:300-366 -- MLE of a base-field vector at an Fp2 point */
void oracle_fp2_mle_eval_base(const u64* inputs, const u64* z_re, const u64* z_im, int n_z,
                              u64* out_re, u64* out_im)
{
    if (n_z <= 0) {
        *out_re = inputs ? inputs[0] : 0;
        *out_im = 0;
        return;
    }
    /* Straight fold chain over all n_z coordinates, LSB first. */
    size_t n = (size_t)1 << n_z;
    u64* cr = (u64*)malloc(n * sizeof(u64));
    u64* ci = (u64*)malloc(n * sizeof(u64));
    for (size_t i = 0; i < n; ++i) { cr[i] = red64(inputs[i]); ci[i] = 0; }
    for (int b = 0; b < n_z; ++b) {
        f2 z = F(z_re[b], z_im[b]);
        size_t m = n >> 1;
        for (size_t i = 0; i < m; ++i) {
            f2 o = fold1(F(cr[2 * i], ci[2 * i]), F(cr[2 * i + 1], ci[2 * i + 1]), z);
            cr[i] = o.re; ci[i] = o.im;
        }
        n = m;
    }
    *out_re = cr[0];
    *out_im = ci[0];
    free(cr);
    free(ci);
}

/* ---- early-round session (native_fp2_core.hpp:163-298) ---- */
typedef struct {
    int n_gates, n_wires, n_copies;
    int *type, *in0, *in1;
    u64 *z_re, *z_im, *v_re, *v_im, *b_re, *b_im;
} oracle_session;

void* oracle_fp2_early_create(int n_gates, const int* type, const int* in0, const int* in1,
                              const u64* z1_re, const u64* z1_im, int n_copies, int n_wires,
                              const u64* v_re, const u64* v_im, const u64* b_re, const u64* b_im)
{
    if (n_gates <= 0 || n_wires <= 0 || n_copies < 2 || (n_copies & (n_copies - 1)) != 0)
        return NULL;
    oracle_session* s = (oracle_session*)calloc(1, sizeof(oracle_session));
    size_t vn = (size_t)n_wires * (size_t)n_copies;
    s->n_gates = n_gates; s->n_wires = n_wires; s->n_copies = n_copies;
    s->type = (int*)malloc(sizeof(int) * n_gates);
    s->in0 = (int*)malloc(sizeof(int) * n_gates);
    s->in1 = (int*)malloc(sizeof(int) * n_gates);
    s->z_re = (u64*)malloc(8 * n_gates);
    s->z_im = (u64*)malloc(8 * n_gates);
    s->v_re = (u64*)malloc(8 * vn);
    s->v_im = (u64*)malloc(8 * vn);
    s->b_re = (u64*)malloc(8 * (size_t)n_copies);
    s->b_im = (u64*)malloc(8 * (size_t)n_copies);
    memcpy(s->type, type, sizeof(int) * n_gates);
    memcpy(s->in0, in0, sizeof(int) * n_gates);
    memcpy(s->in1, in1, sizeof(int) * n_gates);
    memcpy(s->z_re, z1_re, 8 * n_gates);
    memcpy(s->z_im, z1_im, 8 * n_gates);
    memcpy(s->v_re, v_re, 8 * vn);
    memcpy(s->v_im, v_im, 8 * vn);
    memcpy(s->b_re, b_re, 8 * (size_t)n_copies);
    memcpy(s->b_im, b_im, 8 * (size_t)n_copies);
    return s;
}

int oracle_fp2_early_claim(void* h, u64 out8[8])
{
    oracle_session* s = (oracle_session*)h;
    if (!s) return -1;
    const size_t n = (size_t)s->n_copies;
    f2 acc[4] = {F(0, 0), F(0, 0), F(0, 0), F(0, 0)};
    for (size_t c = 0; c + 1 < n; c += 2) {
        f2 v[4] = {F(0, 0), F(0, 0), F(0, 0), F(0, 0)};
        for (int g = 0; g < s->n_gates; ++g) {
            size_t a = (size_t)s->in0[g], b = (size_t)s->in1[g];
            f2 z = F(s->z_re[g], s->z_im[g]);
            f2 a0 = F(s->v_re[a * n + c], s->v_im[a * n + c]);
            f2 a1 = F(s->v_re[a * n + c + 1], s->v_im[a * n + c + 1]);
            f2 b0 = F(s->v_re[b * n + c], s->v_im[b * n + c]);
            f2 b1 = F(s->v_re[b * n + c + 1], s->v_im[b * n + c + 1]);
            int tp = s->type[g];
            v[0] = f2add(v[0], f2mul(gatefn(tp, a0, b0), z));
            v[1] = f2add(v[1], f2mul(gatefn(tp, a1, b1), z));
            v[2] = f2add(v[2], f2mul(gatefn(tp, at_m1(a0, a1), at_m1(b0, b1)), z));
            v[3] = f2add(v[3], f2mul(gatefn(tp, at_2(a0, a1), at_2(b0, b1)), z));
        }
        f2 be0 = F(s->b_re[c], s->b_im[c]), be1 = F(s->b_re[c + 1], s->b_im[c + 1]);
        acc[0] = f2add(acc[0], f2mul(v[0], be0));
        acc[1] = f2add(acc[1], f2mul(v[1], be1));
        acc[2] = f2add(acc[2], f2mul(v[2], at_m1(be0, be1)));
        acc[3] = f2add(acc[3], f2mul(v[3], at_2(be0, be1)));
    }
    for (int t = 0; t < 4; ++t) {
        out8[2 * t] = acc[t].re;
        out8[2 * t + 1] = acc[t].im;
    }
    return 0;
}

int oracle_fp2_early_fold(void* h, u64 r_re, u64 r_im)
{
    oracle_session* s = (oracle_session*)h;
    if (!s) return -1;
    size_t n = (size_t)s->n_copies, m = n >> 1;
    if (m < 1) return 0;
    f2 r = F(r_re, r_im);
    for (size_t w = 0; w < (size_t)s->n_wires; ++w)
        for (size_t i = 0; i < m; ++i) {
            f2 o = fold1(F(s->v_re[w * n + 2 * i], s->v_im[w * n + 2 * i]),
                         F(s->v_re[w * n + 2 * i + 1], s->v_im[w * n + 2 * i + 1]), r);
            /* output index w*m+i never exceeds any input index still to be read */
            s->v_re[w * m + i] = o.re;
            s->v_im[w * m + i] = o.im;
        }
    for (size_t i = 0; i < m; ++i) {
        f2 o = fold1(F(s->b_re[2 * i], s->b_im[2 * i]), F(s->b_re[2 * i + 1], s->b_im[2 * i + 1]), r);
        s->b_re[i] = o.re;
        s->b_im[i] = o.im;
    }
    s->n_copies = (int)m;
    return 0;
}

int oracle_fp2_early_finish(void* h, u64* w_re, u64* w_im, u64* b_re, u64* b_im)
{
    oracle_session* s = (oracle_session*)h;
    if (!s) return -1;
    for (size_t w = 0; w < (size_t)s->n_wires; ++w) {
        w_re[w] = s->v_re[w * (size_t)s->n_copies];
        w_im[w] = s->v_im[w * (size_t)s->n_copies];
    }
    *b_re = s->b_re[0];
    *b_im = s->b_im[0];
    return 0;
}

int oracle_fp2_early_n_copies(void* h) { return h ? ((oracle_session*)h)->n_copies : 0; }
int oracle_fp2_early_n_wires(void* h) { return h ? ((oracle_session*)h)->n_wires : 0; }

void oracle_fp2_early_destroy(void* h)
{
    oracle_session* s = (oracle_session*)h;
    if (!s) return;
    free(s->type); free(s->in0); free(s->in1);
    free(s->z_re); free(s->z_im);
    free(s->v_re); free(s->v_im);
    free(s->b_re); free(s->b_im);
    free(s);
}

/* ---- circuit evaluation (the prover's output vector) ----------------------
 * arithcircuit.py:20-110: the C gates on base-field values, each result reduced
 * like Python's % (non-negative); types by the native index (native_fp2_bridge.py
 * :450-472), with 3 / 4 the left / right multiplexer input as in
 * native_fp2_core.hpp:38-39. */
static u64 modp(__int128 v)
{
    __int128 r = v % (__int128)P61;
    return (u64)(r < 0 ? r + (__int128)P61 : r);
}

static u64 cgate(int tp, u64 a, u64 b)
{
    const __int128 x = (__int128)a, y = (__int128)b;
    switch (tp) {
    case 0: return modp(x * y);
    case 1: return modp(x + y);
    case 2: return modp(x - y);
    case 3: return a;
    case 4: return b;
    case 5: return modp(x + y - x * y);
    case 6: return modp(x + y - 2 * x * y);
    case 7: return modp(1 - x);
    case 8: return modp(1 - x * y);
    case 9: return modp(1 + x * y - x - y);
    case 10: return modp(1 + 2 * x * y - x - y);
    case 11: return modp((1 - x) * y);
    default: return a;
    }
}

/* ArithCircuitBuilder.run over the copies of a frame (arithcircuitbuilder.py:36-46,
 * arithcircuit.py:121-131, 160-181) and the output vector of circuitnizkvec_vole.py
 * :351-355: copy c's input layer is its copy_size bytes, const_val at const_idx
 * (-1: none), zeros up to n_wires; its outputs are the gate values padded with
 * zeros to 2^ceil(log2 n_gates); the copies are concatenated and padded with zeros
 * to n_copies_padded copies. out: n_copies_padded << ceil(log2 n_gates) values. */
int oracle_circuit_outputs(const unsigned char* pix, int n_copies, int n_copies_padded, int copy_size,
                           int n_wires, int const_idx, u64 const_val, int n_gates, const int* type,
                           const int* in0, const int* in1, u64* out)
{
    int bits = 0;
    if (n_copies < 1 || n_copies_padded < n_copies || copy_size > n_wires || n_gates < 1) return -1;
    while ((1 << bits) < n_gates) ++bits;
    const size_t opc = (size_t)1 << bits;
    u64* in = (u64*)calloc((size_t)n_wires, sizeof(u64));
    if (!in) return -1;
    memset(out, 0, (size_t)n_copies_padded * opc * sizeof(u64));
    for (int c = 0; c < n_copies; ++c) {
        for (int w = 0; w < n_wires; ++w)
            in[w] = w < copy_size ? (u64)pix[(size_t)c * copy_size + w] : (w == const_idx ? const_val : 0);
        for (int g = 0; g < n_gates; ++g) {
            if (in0[g] < 0 || in0[g] >= n_wires || in1[g] < 0 || in1[g] >= n_wires) {
                free(in);
                return -1;
            }
            out[(size_t)c * opc + g] = cgate(type[g], in[in0[g]], in[in1[g]]);
        }
    }
    free(in);
    return 0;
}
