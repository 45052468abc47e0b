// One round of the Virgo (linear GKR) sumcheck over the three linear_poly tables
// of a layer: zk_prover::sumcheck_phase1_update / sumcheck_phase2_update
// (TruePix-main/Orion/Orion_nonzk/src/linear_gkr/prover.cpp:576-644, 935-1006;
// the two are the same computation on the tables).
//
// Tables are arrays of linear_poly {a, b} (32 bytes: two {img, real} elements).
// For i < n / 2, with X in {V_mult_add, addV_array, add_mult_sum}:
//   bit 0:  X'[i].b = X[2i].b,            X'[i].a = X[2i+1].b - X'[i].b
//   else:   X'[i].b = X[2i].a r + X[2i].b, X'[i].a = X[2i+1].a r + X[2i+1].b - X'[i].b
// and the round polynomial, over the folded tables M = add_mult_sum',
// V = V_mult_add', A = addV_array':
//   a = sum M.a V.a,  b = sum M.a V.b + M.b V.a + A.a,  c = sum M.b V.b + A.b.
// One thread per folded entry, CTA sums in shared memory, the last CTA (ticket)
// adds the CTA partials.
#include <algorithm>
#include <type_traits>
#include <vector>

#include "fp2.cuh"
#include "runtime.h"
#include "virgo.h"

namespace tp {
namespace virgo {

namespace {

constexpr int kThreads = 256;

struct LP {
    fp2 a, b;
};

__device__ __forceinline__ fp2 ld_fe(const ulonglong2* p) { const ulonglong2 v = __ldg(p); return mk(v.y, v.x); }
__device__ __forceinline__ LP ld_lp(const ulonglong2* t, long long i) { return LP{ld_fe(t + 2 * i), ld_fe(t + 2 * i + 1)}; }
__device__ __forceinline__ void st_lp(ulonglong2* t, long long i, LP v)
{
    const fp2 a = l2canon(v.a), b = l2canon(v.b);
    t[2 * i] = make_ulonglong2(a.im, a.re);
    t[2 * i + 1] = make_ulonglong2(b.im, b.re);
}

__device__ __forceinline__ LP fold(const ulonglong2* t, long long i, fp2 r, bool bit)
{
    const LP x0 = ld_lp(t, 2 * i), x1 = ld_lp(t, 2 * i + 1);
    LP y;
    if (!bit) {
        y.b = x0.b;
        y.a = l2sub(x1.b, y.b);
    } else {
        y.b = l2add(l2mul(x0.a, r), x0.b);
        y.a = l2sub(l2add(l2mul(x1.a, r), x1.b), y.b);
    }
    return y;
}

__device__ __forceinline__ fp2 shfl_down2(fp2 v, int o)
{
    fp2 w;
    w.re = __shfl_down_sync(0xffffffffu, v.re, o);
    w.im = __shfl_down_sync(0xffffffffu, v.im, o);
    return w;
}

__global__ void __launch_bounds__(kThreads) update_kernel(const ulonglong2* __restrict__ vma,
                                                          const ulonglong2* __restrict__ addv,
                                                          const ulonglong2* __restrict__ ams, long long half,
                                                          fp2 r, int bit, ulonglong2* __restrict__ vma_out,
                                                          ulonglong2* __restrict__ addv_out,
                                                          ulonglong2* __restrict__ ams_out, fp2* __restrict__ part,
                                                          unsigned* __restrict__ ticket,
                                                          ulonglong2* __restrict__ ret)
{
    __shared__ fp2 red[3][kThreads / 32];
    __shared__ bool last;
    fp2 qa = f2zero(), qb = f2zero(), qc = f2zero();
    const long long stride = (long long)gridDim.x * kThreads;
    for (long long i = (long long)blockIdx.x * kThreads + threadIdx.x; i < half; i += stride) {
        const LP v = fold(vma, i, r, bit), a = fold(addv, i, r, bit), m = fold(ams, i, r, bit);
        st_lp(vma_out, i, v);
        st_lp(addv_out, i, a);
        st_lp(ams_out, i, m);
        qa = l2add(qa, l2mul(m.a, v.a));
        qb = l2add(qb, l2add(l2add(l2mul(m.a, v.b), l2mul(m.b, v.a)), a.a));
        qc = l2add(qc, l2add(l2mul(m.b, v.b), a.b));
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        qa = l2add(qa, shfl_down2(qa, o));
        qb = l2add(qb, shfl_down2(qb, o));
        qc = l2add(qc, shfl_down2(qc, o));
    }
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) {
        red[0][w] = qa;
        red[1][w] = qb;
        red[2][w] = qc;
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        fp2 s = f2zero();
        for (int k = 0; k < kThreads / 32; ++k) s = l2add(s, red[threadIdx.x][k]);
        part[3 * blockIdx.x + threadIdx.x] = s;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (last && threadIdx.x < 3) {
        __threadfence();
        const volatile u64* pv = reinterpret_cast<const volatile u64*>(part);
        fp2 s = f2zero();
        for (unsigned b = 0; b < gridDim.x; ++b)
            s = l2add(s, mk(pv[2 * (3 * b + threadIdx.x)], pv[2 * (3 * b + threadIdx.x) + 1]));
        s = l2canon(s);
        ret[threadIdx.x] = make_ulonglong2(s.im, s.re);
        if (threadIdx.x == 0) *ticket = 0;
    }
}

}  // namespace

bool update(const ulonglong2* vma, const ulonglong2* addv, const ulonglong2* ams, long long n, fp2 r, int bit,
            ulonglong2* vma_out, ulonglong2* addv_out, ulonglong2* ams_out, ulonglong2* ret, cudaStream_t s)
{
    Ctx* c = ctx();
    if (!c) return false;
    if (n < 2 || (n & 1)) {
        set_error(TP_ERR_ARG, "virgo update: total_uv %lld must be even and >= 2", n);
        return false;
    }
    if (r.re >= P61 || r.im >= P61) {
        set_error(TP_ERR_ARG, "virgo update: previous_random is not canonical");
        return false;
    }
    const long long half = n / 2;
    const long long want = (half + kThreads - 1) / kThreads;
    const unsigned blocks = (unsigned)std::min<long long>(want, (long long)c->n_sm * 8);
    fp2* part = static_cast<fp2*>(dev_alloc(sizeof(fp2) * 3 * blocks + 256, s));
    if (!part) return false;
    unsigned* ticket = reinterpret_cast<unsigned*>(part + 3 * blocks);
    bool ok = !cuda_failed(cudaMemsetAsync(ticket, 0, sizeof(unsigned), s), "virgo ticket");
    if (ok) {
        timer_begin(s, 9300);
        update_kernel<<<blocks, kThreads, 0, s>>>(vma, addv, ams, half, r, bit ? 1 : 0, vma_out, addv_out, ams_out,
                                                  part, ticket, ret);
        timer_end(s);
        ok = !cuda_failed(cudaGetLastError(), "virgo update");
    }
    dev_free(part, s);
    return ok;
}

// ---- layer inits: zk_prover::sumcheck_phase1_init / sumcheck_phase2_init ----
// (prover.cpp:246-570, 645-930). The reference computes per-gate intermediates
// and scatters them into the tables serially; field addition is exact, so the
// sum at each table entry does not depend on the order. The layer's gates are
// turned once, on the host, into terms grouped by the table entry they add to
// (a counting sort), and one thread per entry sums its terms. The terms of
// sum / exp-sum / custom-comb gates that phase 2 adds to addV_array[0] form a
// separate list, reduced by a grid sum.

namespace {

struct HalfEq {   // eq(r, i) = f[i & mask] * s[i >> h] (scaled by the f table)
    const fp2* f;
    const fp2* s;
    long long mask;
    int h;
};

__device__ __forceinline__ fp2 eq_at(const HalfEq& e, long long i) { return l2mul(e.f[i & e.mask], e.s[i >> e.h]); }

__device__ __forceinline__ fp2 ldv(const ulonglong2* t, long long i) { return ld_fe(t + i); }
__device__ __forceinline__ void st_b(ulonglong2* t, long long i, fp2 b)
{
    b = l2canon(b);
    t[2 * i] = make_ulonglong2(0, 0);
    t[2 * i + 1] = make_ulonglong2(b.im, b.re);
}
// x * 2^k (k < 64 here; ranges are bounded by the table size)
__device__ __forceinline__ fp2 times_pow2(fp2 x, int k)
{
    for (; k > 0; --k) x = l2add(x, x);
    return x;
}

__global__ void __launch_bounds__(kThreads) phase1_kernel(Layer L, const ulonglong2* __restrict__ values, HalfEq g0,
                                                          HalfEq g1, ulonglong2* __restrict__ vma,
                                                          ulonglong2* __restrict__ addv, ulonglong2* __restrict__ ams)
{
    const long long t = (long long)blockIdx.x * kThreads + threadIdx.x;
    if (t >= L.total_uv) return;
    fp2 A = f2zero(), M = f2zero();
    for (unsigned e = L.d_p1_ptr[t]; e < L.d_p1_ptr[t + 1]; ++e) {
        const Term q = L.d_p1[e];
        const long long g = q.gate;
        const long long at = q.type == 4 ? L.d_u[g] : g;
        const fp2 tmp = l2add(eq_at(g0, at), eq_at(g1, at));
        switch (q.type) {
        case 0: A = l2add(A, l2mul(ldv(values, L.d_v[g]), tmp)); M = l2add(M, tmp); break;
        case 1: M = l2add(M, l2mul(ldv(values, L.d_v[g]), tmp)); break;
        case 4: case 5: case 10: M = l2add(M, tmp); break;
        case 12: M = l2add(M, times_pow2(tmp, q.k)); break;
        case 14: M = l2add(M, l2mul(ld_fe(L.d_w + q.k), tmp)); break;
        case 6: M = l2sub(M, tmp); A = l2add(A, tmp); break;
        case 7: A = l2sub(A, l2mul(ldv(values, L.d_v[g]), tmp)); M = l2add(M, tmp); break;
        case 8: {
            const fp2 tv = l2mul(tmp, ldv(values, L.d_v[g]));
            A = l2add(A, tv);
            M = l2sub(l2add(M, tmp), l2add(tv, tv));
            break;
        }
        case 13: M = l2sub(l2add(M, tmp), l2mul(tmp, ldv(values, L.d_v[g]))); break;
        case 9: {
            const fp2 tv = l2mul(tmp, ldv(values, L.d_v[g]));
            A = l2add(A, tv);
            M = l2sub(M, tv);
            break;
        }
        default: break;
        }
    }
    const fp2 val = ldv(values, t);
    vma[2 * t] = make_ulonglong2(0, 0);
    vma[2 * t + 1] = make_ulonglong2(val.im, val.re);
    st_b(addv, t, A);
    st_b(ams, t, M);
}

__device__ __forceinline__ fp2 v_u_of(const ulonglong2* vma0, fp2 prev_r)
{
    return l2add(l2mul(ld_fe(vma0), prev_r), ld_fe(vma0 + 1));
}

__global__ void __launch_bounds__(kThreads) phase2_kernel(Layer L, const ulonglong2* __restrict__ values, HalfEq g0,
                                                          HalfEq g1, HalfEq gu, const ulonglong2* __restrict__ vma0,
                                                          fp2 prev_r, ulonglong2* __restrict__ vma,
                                                          ulonglong2* __restrict__ addv, ulonglong2* __restrict__ ams)
{
    const long long t = (long long)blockIdx.x * kThreads + threadIdx.x;
    if (t >= L.total_uv) return;
    const fp2 v_u = v_u_of(vma0, prev_r);
    fp2 A = f2zero(), M = f2zero();
    for (unsigned e = L.d_p2_ptr[t]; e < L.d_p2_ptr[t + 1]; ++e) {
        const Term q = L.d_p2[e];
        const long long g = q.gate;
        const fp2 tgu = l2mul(l2add(eq_at(g0, g), eq_at(g1, g)), eq_at(gu, L.d_u[g]));
        const fp2 tv = l2mul(tgu, v_u);
        switch (q.type) {
        case 1: M = l2add(M, tv); break;
        case 0: M = l2add(M, tgu); A = l2add(A, tv); break;
        case 6: A = l2add(A, l2sub(tgu, tv)); break;
        case 7: M = l2sub(M, tgu); A = l2add(A, tv); break;
        case 8: M = l2add(M, l2sub(tgu, l2add(tv, tv))); A = l2add(A, tv); break;
        case 13: M = l2sub(M, tv); A = l2add(A, tv); break;
        case 9: M = l2add(M, l2sub(tgu, tv)); break;
        case 10: A = l2add(A, tv); break;
        default: break;
        }
    }
    const fp2 val = ldv(values, t);
    vma[2 * t] = make_ulonglong2(0, 0);
    vma[2 * t + 1] = make_ulonglong2(val.im, val.re);
    st_b(addv, t, A);
    st_b(ams, t, M);
}

// addV_array[0].b += sum over the sum / exp-sum / custom-comb terms of
// tmp_g v_u eq(r_u, j) (x 2^e, x weight); the last CTA (ticket) adds the partials
__global__ void __launch_bounds__(kThreads) phase2_sum_kernel(Layer L, HalfEq g0, HalfEq g1, HalfEq gu,
                                                              const ulonglong2* __restrict__ vma0, fp2 prev_r,
                                                              ulonglong2* __restrict__ addv, fp2* __restrict__ part,
                                                              unsigned* __restrict__ ticket)
{
    __shared__ fp2 red[kThreads / 32];
    __shared__ bool last;
    const fp2 v_u = v_u_of(vma0, prev_r);
    fp2 acc = f2zero();
    for (long long e = (long long)blockIdx.x * kThreads + threadIdx.x; e < L.n_p2s; e += (long long)gridDim.x * kThreads) {
        const Term q = L.d_p2s[e];
        const long long g = q.gate;
        const fp2 x = l2mul(l2add(eq_at(g0, g), eq_at(g1, g)), v_u);
        fp2 y;
        if (q.type == 14)
            y = l2mul(l2mul(x, eq_at(gu, L.d_src[q.k])), ld_fe(L.d_w + q.k));
        else if (q.type == 12)
            y = l2mul(times_pow2(x, q.k), eq_at(gu, L.d_u[g] + q.k));
        else
            y = l2mul(x, eq_at(gu, L.d_u[g] + q.k));
        acc = l2add(acc, y);
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) acc = l2add(acc, shfl_down2(acc, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        fp2 sum = f2zero();
        for (int k = 0; k < kThreads / 32; ++k) sum = l2add(sum, red[k]);
        part[blockIdx.x] = sum;
        __threadfence();
        last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (last && threadIdx.x == 0) {
        __threadfence();
        const volatile u64* pv = reinterpret_cast<const volatile u64*>(part);
        fp2 sum = ld_fe(addv + 1);
        for (unsigned b = 0; b < gridDim.x; ++b) sum = l2add(sum, mk(pv[2 * b], pv[2 * b + 1]));
        sum = l2canon(sum);
        addv[1] = make_ulonglong2(sum.im, sum.re);
        *ticket = 0;
    }
}

bool check_canonical(const uint64_t* w, long long n, const char* what)
{
    for (long long i = 0; i < n; ++i)
        if (w[i] >= P61) {
            set_error(TP_ERR_ARG, "virgo init: %s element %lld is not canonical", what, i / 2);
            return false;
        }
    return true;
}

// host half tables of eq(r, .) (bit k of the index <-> r[k]) for len bits, the
// low table scaled by `scale`: f[2^(len/2)], s[2^(len - len/2)], appended to out
fp2 host_fe(const uint64_t* p) { return mk(p[1], p[0]); }

void half_tables(const uint64_t* r, int len, fp2 scale, std::vector<fp2>& out, long long* f_off, long long* s_off,
                 long long* mask, int* h)
{
    const int h1 = len >> 1, h2 = len - h1;
    *h = h1;
    *mask = (1LL << h1) - 1;
    const fp2 one = mk(1, 0);
    auto build = [&](int off, int n, fp2 init) {
        std::vector<fp2> t((size_t)1 << n);
        t[0] = init;
        for (int k = 0; k < n; ++k) {
            const fp2 rk = host_fe(r + 2 * (off + k)), omr = f2sub(one, rk);
            for (long long j = 0; j < (1LL << k); ++j) {
                t[(size_t)(j | (1LL << k))] = f2mul(t[(size_t)j], rk);
                t[(size_t)j] = f2mul(t[(size_t)j], omr);
            }
        }
        return t;
    };
    const std::vector<fp2> f = build(0, h1, scale), s = build(h1, h2, one);
    *f_off = (long long)out.size();
    out.insert(out.end(), f.begin(), f.end());
    *s_off = (long long)out.size();
    out.insert(out.end(), s.begin(), s.end());
}

}  // namespace

Layer* layer_create(int length_g, int length_u, const int* ty, const long long* u, const long long* v,
                    const int* comb_ptr, const int* comb_src, const uint64_t* comb_w)
{
    Ctx* c = ctx();
    if (!c) return nullptr;
    if (length_g < 0 || length_g > 26 || length_u < 1 || length_u > 26 || !ty || !u || !v) {
        set_error(TP_ERR_ARG, "virgo layer: bit lengths %d, %d outside [0, 26] / [1, 26] or null gates", length_g,
                  length_u);
        return nullptr;
    }
    const long long G = 1LL << length_g, U = 1LL << length_u;
    std::vector<long long> cnt1(U + 1, 0), cnt2(U + 1, 0);
    long long n_p2s = 0, n_w = 0;
    for (long long g = 0; g < G; ++g) {
        const int t = ty[g];
        const bool plain = t == 0 || t == 1 || t == 6 || t == 7 || t == 8 || t == 9 || t == 10 || t == 13;
        bool ok = true;
        if (plain)
            ok = u[g] >= 0 && u[g] < U && v[g] >= 0 && v[g] < U;
        else if (t == 4)
            ok = u[g] >= 0 && u[g] < G && u[g] < U && v[g] >= 0 && v[g] < U;
        else if (t == 5)
            ok = u[g] >= 0 && v[g] <= U && u[g] <= v[g] && v[g] - u[g] <= 62;
        else if (t == 12)
            ok = u[g] >= 0 && v[g] < U && u[g] <= v[g] + 1 && v[g] - u[g] < 62;
        else if (t == 14) {
            ok = comb_ptr && comb_src && comb_w && comb_ptr[g] >= 0 && comb_ptr[g] <= comb_ptr[g + 1];
            for (int k = ok ? comb_ptr[g] : 0; ok && k < comb_ptr[g + 1]; ++k)
                ok = comb_src[k] >= 0 && comb_src[k] < U;
            if (ok) n_w = std::max<long long>(n_w, comb_ptr[g + 1]);
        }
        if (!ok) {
            set_error(TP_ERR_ARG, "virgo layer: gate %lld (type %d, u %lld, v %lld) indexes outside the layer", g, t,
                      u[g], v[g]);
            return nullptr;
        }
        if (plain || t == 4) ++cnt1[u[g]];
        if (plain) ++cnt2[v[g]];
        if (t == 5) {
            for (long long j = u[g]; j < v[g]; ++j) ++cnt1[j];
            n_p2s += v[g] - u[g];
        } else if (t == 12) {
            for (long long j = u[g]; j <= v[g]; ++j) ++cnt1[j];
            n_p2s += v[g] - u[g] + 1;
        } else if (t == 14) {
            for (int k = comb_ptr[g]; k < comb_ptr[g + 1]; ++k) ++cnt1[comb_src[k]];
            n_p2s += comb_ptr[g + 1] - comb_ptr[g];
        }
    }
    if (comb_w && !check_canonical(comb_w, 2 * n_w, "custom-comb weight")) return nullptr;
    // exclusive prefix sums -> CSR pointers; fill
    std::vector<unsigned> p1(U + 1), p2(U + 1);
    long long a1 = 0, a2 = 0;
    for (long long t = 0; t < U; ++t) {
        p1[t] = (unsigned)a1;
        p2[t] = (unsigned)a2;
        a1 += cnt1[t];
        a2 += cnt2[t];
    }
    p1[U] = (unsigned)a1;
    p2[U] = (unsigned)a2;
    if (a1 >= (1LL << 32) || a2 >= (1LL << 32)) {
        set_error(TP_ERR_ARG, "virgo layer: too many terms");
        return nullptr;
    }
    std::vector<Term> t1((size_t)std::max<long long>(1, a1)), t2((size_t)std::max<long long>(1, a2)),
        ts((size_t)std::max<long long>(1, n_p2s));
    std::vector<unsigned> f1(p1.begin(), p1.end() - 1), f2(p2.begin(), p2.end() - 1);
    long long fs = 0;
    for (long long g = 0; g < G; ++g) {
        const int t = ty[g];
        const bool plain = t == 0 || t == 1 || t == 6 || t == 7 || t == 8 || t == 9 || t == 10 || t == 13;
        if (plain || t == 4) t1[f1[u[g]]++] = Term{(int)g, t, 0};
        if (plain) t2[f2[v[g]]++] = Term{(int)g, t, 0};
        if (t == 5) {
            for (long long j = u[g]; j < v[g]; ++j) {
                t1[f1[j]++] = Term{(int)g, 5, 0};
                ts[fs++] = Term{(int)g, 5, (int)(j - u[g])};
            }
        } else if (t == 12) {
            for (long long j = u[g]; j <= v[g]; ++j) {
                t1[f1[j]++] = Term{(int)g, 12, (int)(j - u[g])};
                ts[fs++] = Term{(int)g, 12, (int)(j - u[g])};
            }
        } else if (t == 14) {
            for (int k = comb_ptr[g]; k < comb_ptr[g + 1]; ++k) {
                t1[f1[comb_src[k]]++] = Term{(int)g, 14, k};
                ts[fs++] = Term{(int)g, 14, k};
            }
        }
    }
    Layer* L = new Layer();
    L->length_g = length_g;
    L->length_u = length_u;
    L->n_gates = G;
    L->total_uv = U;
    L->n_p2s = n_p2s;
    std::vector<fp2> w((size_t)std::max<long long>(1, n_w));
    std::vector<int> src((size_t)std::max<long long>(1, n_w), 0);
    for (long long k = 0; k < n_w; ++k) {
        w[(size_t)k] = host_fe(comb_w + 2 * k);
        src[(size_t)k] = comb_src[k];
    }
    std::vector<ulonglong2> w2(w.size());
    for (size_t k = 0; k < w.size(); ++k) w2[k] = make_ulonglong2(w[k].im, w[k].re);
    cudaStream_t s = c->stream;
    bool ok = true;
    auto put = [&](auto*& d, const auto& h) {
        using T = typename std::remove_reference<decltype(h)>::type::value_type;
        d = static_cast<std::remove_reference_t<decltype(d)>>(dev_alloc(sizeof(T) * h.size(), s));
        ok = ok && d && host_to_device(d, h.data(), sizeof(T) * h.size(), s);
    };
    std::vector<long long> hu(u, u + G), hv(v, v + G);
    put(L->d_u, hu);
    put(L->d_v, hv);
    put(L->d_p1_ptr, p1);
    put(L->d_p1, t1);
    put(L->d_p2_ptr, p2);
    put(L->d_p2, t2);
    put(L->d_p2s, ts);
    put(L->d_w, w2);
    put(L->d_src, src);
    L->max_blocks = (unsigned)std::max<long long>(1, std::min<long long>((n_p2s + kThreads - 1) / kThreads,
                                                                         (long long)c->n_sm * 8));
    L->d_part = static_cast<fp2*>(dev_alloc(sizeof(fp2) * L->max_blocks + 256, s));
    ok = ok && L->d_part && !cuda_failed(cudaMemsetAsync(L->d_part + L->max_blocks, 0, sizeof(unsigned), s), "ticket") &&
         !cuda_failed(cudaStreamSynchronize(s), "virgo layer upload");
    if (!ok) {
        layer_destroy(L);
        return nullptr;
    }
    return L;
}

void layer_destroy(Layer* L)
{
    if (!L) return;
    Ctx* c = ctx();
    if (c) {
        for (void* p : {(void*)L->d_u, (void*)L->d_v, (void*)L->d_p1_ptr, (void*)L->d_p1, (void*)L->d_p2_ptr,
                        (void*)L->d_p2, (void*)L->d_p2s, (void*)L->d_w, (void*)L->d_src, (void*)L->d_part})
            if (p) dev_free(p, c->stream);
        cudaStreamSynchronize(c->stream);
    }
    delete L;
}

namespace {

struct Tables {
    std::vector<fp2> h;
    HalfEq g0, g1, gu;
    long long off[6];
};

// half tables for g (alpha r0, beta r1) and, when r_u is set, u; uploaded into d
bool eq_tables(const Layer& L, const uint64_t* r0, const uint64_t* r1, const uint64_t* alpha, const uint64_t* beta,
               const uint64_t* r_u, fp2** d, Tables* T, cudaStream_t s)
{
    long long mask;
    int h;
    half_tables(r0, L.length_g, host_fe(alpha), T->h, &T->off[0], &T->off[1], &mask, &h);
    T->g0.mask = mask;
    T->g0.h = h;
    half_tables(r1, L.length_g, host_fe(beta), T->h, &T->off[2], &T->off[3], &mask, &h);
    T->g1.mask = mask;
    T->g1.h = h;
    if (r_u) {
        half_tables(r_u, L.length_u, mk(1, 0), T->h, &T->off[4], &T->off[5], &mask, &h);
        T->gu.mask = mask;
        T->gu.h = h;
    }
    *d = static_cast<fp2*>(dev_alloc(sizeof(fp2) * T->h.size(), s));
    if (!*d || !host_to_device(*d, T->h.data(), sizeof(fp2) * T->h.size(), s)) return false;
    T->g0.f = *d + T->off[0];
    T->g0.s = *d + T->off[1];
    T->g1.f = *d + T->off[2];
    T->g1.s = *d + T->off[3];
    if (r_u) {
        T->gu.f = *d + T->off[4];
        T->gu.s = *d + T->off[5];
    }
    return true;
}

bool randoms_ok(const Layer& L, const uint64_t* r0, const uint64_t* r1, const uint64_t* alpha, const uint64_t* beta)
{
    if ((L.length_g && (!r0 || !r1)) || !alpha || !beta) {
        set_error(TP_ERR_ARG, "virgo init: null randoms");
        return false;
    }
    return check_canonical(r0, 2 * L.length_g, "r_0") && check_canonical(r1, 2 * L.length_g, "r_1") &&
           check_canonical(alpha, 2, "alpha") && check_canonical(beta, 2, "beta");
}

}  // namespace

bool phase1_init(const Layer& L, const ulonglong2* values, const uint64_t* r0, const uint64_t* r1,
                 const uint64_t* alpha, const uint64_t* beta, ulonglong2* vma, ulonglong2* addv, ulonglong2* ams,
                 cudaStream_t s)
{
    if (!randoms_ok(L, r0, r1, alpha, beta)) return false;
    Tables T;
    fp2* d = nullptr;
    bool ok = eq_tables(L, r0, r1, alpha, beta, nullptr, &d, &T, s);
    if (ok) {
        timer_begin(s, 9301);
        phase1_kernel<<<(unsigned)((L.total_uv + kThreads - 1) / kThreads), kThreads, 0, s>>>(L, values, T.g0, T.g1,
                                                                                                vma, addv, ams);
        timer_end(s);
        ok = !cuda_failed(cudaGetLastError(), "virgo phase1 init");
    }
    if (d) dev_free(d, s);
    return ok;
}

bool phase2_init(const Layer& L, const ulonglong2* values, const uint64_t* r0, const uint64_t* r1,
                 const uint64_t* alpha, const uint64_t* beta, const ulonglong2* vma0, const uint64_t* prev_r,
                 const uint64_t* r_u, ulonglong2* vma, ulonglong2* addv, ulonglong2* ams, cudaStream_t s)
{
    if (!randoms_ok(L, r0, r1, alpha, beta)) return false;
    if (!prev_r || !r_u || !vma0) {
        set_error(TP_ERR_ARG, "virgo phase2 init: null previous random, r_u or V_mult_add");
        return false;
    }
    if (!check_canonical(prev_r, 2, "previous_random") || !check_canonical(r_u, 2 * L.length_u, "r_u")) return false;
    Tables T;
    fp2* d = nullptr;
    bool ok = eq_tables(L, r0, r1, alpha, beta, r_u, &d, &T, s);
    const fp2 pr = host_fe(prev_r);
    if (ok) {
        timer_begin(s, 9302);
        phase2_kernel<<<(unsigned)((L.total_uv + kThreads - 1) / kThreads), kThreads, 0, s>>>(
            L, values, T.g0, T.g1, T.gu, vma0, pr, vma, addv, ams);
        timer_end(s);
        ok = !cuda_failed(cudaGetLastError(), "virgo phase2 init");
    }
    if (ok && L.n_p2s > 0) {
        const unsigned blocks = (unsigned)std::min<long long>((L.n_p2s + kThreads - 1) / kThreads, L.max_blocks);
        timer_begin(s, 9303);
        phase2_sum_kernel<<<blocks, kThreads, 0, s>>>(L, T.g0, T.g1, T.gu, vma0, pr, addv, L.d_part,
                                                      reinterpret_cast<unsigned*>(L.d_part + L.max_blocks));
        timer_end(s);
        ok = !cuda_failed(cudaGetLastError(), "virgo phase2 sums");
    }
    if (d) dev_free(d, s);
    return ok;
}

}  // namespace virgo
}  // namespace tp
