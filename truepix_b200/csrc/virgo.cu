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

}  // namespace virgo
}  // namespace tp
