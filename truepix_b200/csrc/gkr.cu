// GKR input-layer sumcheck kernels for sm_100a.
//
// Reference behaviour: TruePix-main/native_fp2/native_fp2_core.hpp (CPU) and
// TruePix-main/native_fp2/native_fp2.cu:125-390 (its CUDA kernels).
//
// Design (one B200, tables resident in HBM):
//  * The table V[w][c] (wire-major, copies contiguous) is packed Fp2 (16 B per
//    element, {re, im}); every load and store is a 16-byte vector access and a
//    warp touches 1-2 KB contiguous per wire.
//  * The gate sum is rewritten once per layer as K0 + sum_w L[w] V_w + sum c V_a V_b
//    (see GateForm). A claim is then a weighted sum over the table that is linear
//    in the round variable t for the L part, so only t = 0, 1 are computed and
//    t = -1, 2 follow as 2*S0 - S1 and 2*S1 - S0 (exact field identities).
//  * fold(r) is recorded and applied by the next claim in the same pass: one
//    kernel reads V (4 copies per thread per wire), writes the folded table and
//    accumulates the next claim from the folded values still in registers. Each
//    early round therefore moves 48 B per folded element and nothing else.
//  * Work item = (claim pair, wire slice); the slice count is chosen so that the
//    grid fills all SMs even when few pairs remain. Reduction: warp shuffle ->
//    shared memory -> last-block grid reduction (ticket), leaving the 8 u64 claim
//    on the device.
#include "gkr.h"
#include "gkr_internal.cuh"
#include "runtime.h"

#include <algorithm>
#include <cstring>
#include <map>
#include <utility>

namespace tp {

namespace {

constexpr int kThreads = 256;
thread_local int t_launches = 0;

enum { MODE_CLAIM = 0, MODE_FOLD_CLAIM = 1, MODE_EXPLICIT = 2 };

struct ClaimArgs {
    const fp2* A;      // table, row stride n_in
    fp2* Aout;         // folded table, row stride n_in/2 (MODE_FOLD_CLAIM)
    const fp2* beta;
    fp2* beta_out;
    fp2 r;             // pending fold challenge
    int n_in;
    int n_pairs;       // claim pairs
    int W, n_slices, wc, tc;   // W = rows stored; rows >= W are identically zero
    fp2 K0;
    const fp2* L;
    const int2* ab;
    const fp2* cf;
    int n_terms;
    const u64* t[12];  // MODE_EXPLICIT: v, f0, f1, b, bf0, bf1 (re, im each)
    fp2* partials;
    unsigned* ticket;
    u64* out8;
};

template <int MODE>
__device__ __forceinline__ void load_01(const ClaimArgs& a, int w, int p, fp2& x0, fp2& x1,
                                        bool store)
{
    if (w >= a.W) {  // a known-zero row (frame padding wires)
        x0 = x1 = f2zero();
        return;
    }
    const fp2* row = a.A + (size_t)w * (size_t)a.n_in;
    if (MODE == MODE_CLAIM) {
        x0 = ld2(row + 2 * (size_t)p);
        x1 = ld2(row + 2 * (size_t)p + 1);
    } else {
        const fp2* q = row + 4 * (size_t)p;
        const fp2 a0 = ld2(q), a1 = ld2(q + 1), a2 = ld2(q + 2), a3 = ld2(q + 3);
        x0 = l2fold(a0, a1, a.r);
        x1 = l2fold(a2, a3, a.r);
        if (store) {
            fp2* o = a.Aout + (size_t)w * (size_t)(a.n_in >> 1) + 2 * (size_t)p;
            st2(o, x0);
            st2(o + 1, x1);
        }
    }
}

__device__ __forceinline__ void load_explicit(const ClaimArgs& a, int w, int p, fp2 (&x)[4])
{
    const size_t n = (size_t)a.n_in, h = (size_t)a.n_pairs;
    const size_t i0 = (size_t)w * n + 2 * (size_t)p, i2 = (size_t)w * h + (size_t)p;
    x[0] = mk(a.t[0][i0], a.t[1][i0]);
    x[1] = mk(a.t[0][i0 + 1], a.t[1][i0 + 1]);
    x[2] = mk(a.t[2][i2], a.t[3][i2]);
    x[3] = mk(a.t[4][i2], a.t[5][i2]);
}

template <int MODE>
__global__ void __launch_bounds__(kThreads) claim_kernel(const ClaimArgs a)
{
    fp2 acc[4] = {f2zero(), f2zero(), f2zero(), f2zero()};
    const long long item = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long n_items = (long long)a.n_pairs * a.n_slices;
    if (item < n_items) {
        const int p = (int)(item % a.n_pairs);
        const int y = (int)(item / a.n_pairs);
        fp2 bt[4], S[4];
        if (MODE == MODE_CLAIM) {
            bt[0] = ld2(a.beta + 2 * (size_t)p);
            bt[1] = ld2(a.beta + 2 * (size_t)p + 1);
        } else if (MODE == MODE_FOLD_CLAIM) {
            const fp2* q = a.beta + 4 * (size_t)p;
            bt[0] = l2fold(ld2(q), ld2(q + 1), a.r);
            bt[1] = l2fold(ld2(q + 2), ld2(q + 3), a.r);
            if (y == 0) {
                st2(a.beta_out + 2 * (size_t)p, bt[0]);
                st2(a.beta_out + 2 * (size_t)p + 1, bt[1]);
            }
        } else {
            bt[0] = mk(a.t[6][2 * (size_t)p], a.t[7][2 * (size_t)p]);
            bt[1] = mk(a.t[6][2 * (size_t)p + 1], a.t[7][2 * (size_t)p + 1]);
            bt[2] = mk(a.t[8][p], a.t[9][p]);
            bt[3] = mk(a.t[10][p], a.t[11][p]);
        }
        if (MODE != MODE_EXPLICIT) {
            bt[2] = l2at_m1(bt[0], bt[1]);
            bt[3] = l2at_2(bt[0], bt[1]);
        }

        // linear part over this slice's wires. Products are nearly canonical
        // (< 2^61 + 8); raw sums of up to 5 of them stay below 2^64, so the
        // accumulators are folded once every 4 wires.
        const int w0 = y * a.wc, w1 = min(a.W, w0 + a.wc);
        if (MODE != MODE_EXPLICIT) {
            fp2 S0 = f2zero(), S1 = f2zero();
            int pending = 0;
            for (int w = w0; w < w1; ++w) {
                fp2 x0, x1;
                load_01<MODE>(a, w, p, x0, x1, true);
                const fp2 l = ld2(a.L + w);
                if (!f2is0(l)) {
                    const fp2 m0 = l2mul(l, x0), m1 = l2mul(l, x1);
                    S0.re += m0.re; S0.im += m0.im;
                    S1.re += m1.re; S1.im += m1.im;
                    if (++pending == 4) {
                        S0 = mk(fold61(S0.re), fold61(S0.im));
                        S1 = mk(fold61(S1.re), fold61(S1.im));
                        pending = 0;
                    }
                }
            }
            S0 = mk(fold61(S0.re), fold61(S0.im));
            S1 = mk(fold61(S1.re), fold61(S1.im));
            S[0] = S0;
            S[1] = S1;
            S[2] = l2at_m1(S0, S1);
            S[3] = l2at_2(S0, S1);
        } else {
#pragma unroll
            for (int t = 0; t < 4; ++t) S[t] = f2zero();
            for (int w = w0; w < w1; ++w) {
                const fp2 l = ld2(a.L + w);
                if (f2is0(l)) continue;
                fp2 x[4];
                load_explicit(a, w, p, x);
#pragma unroll
                for (int t = 0; t < 4; ++t) S[t] = l2add(S[t], l2mul(l, x[t]));
            }
        }
        if (y == 0)
#pragma unroll
            for (int t = 0; t < 4; ++t) S[t] = l2add(S[t], a.K0);

        // product terms c*V[a]*V[b] of this slice, grouped by b
        const int e0 = y * a.tc, e1 = min(a.n_terms, e0 + a.tc);
        if (e0 < e1) {
            fp2 M[4] = {f2zero(), f2zero(), f2zero(), f2zero()};
            int cur_b = a.ab[e0].y;
            for (int e = e0; e <= e1; ++e) {
                const bool flush = (e == e1) || (a.ab[e].y != cur_b);
                if (flush) {
                    fp2 xb[4];
                    if (MODE != MODE_EXPLICIT) {
                        load_01<MODE>(a, cur_b, p, xb[0], xb[1], false);
                        xb[2] = l2at_m1(xb[0], xb[1]);
                        xb[3] = l2at_2(xb[0], xb[1]);
                        M[2] = l2at_m1(M[0], M[1]);
                        M[3] = l2at_2(M[0], M[1]);
                    } else {
                        load_explicit(a, cur_b, p, xb);
                    }
#pragma unroll
                    for (int t = 0; t < 4; ++t) {
                        S[t] = l2add(S[t], l2mul(xb[t], M[t]));
                        M[t] = f2zero();
                    }
                    if (e == e1) break;
                    cur_b = a.ab[e].y;
                }
                const fp2 c = ld2(a.cf + e);
                if (MODE != MODE_EXPLICIT) {
                    fp2 x0, x1;
                    load_01<MODE>(a, a.ab[e].x, p, x0, x1, false);
                    M[0] = l2add(M[0], l2mul(c, x0));
                    M[1] = l2add(M[1], l2mul(c, x1));
                } else {
                    fp2 x[4];
                    load_explicit(a, a.ab[e].x, p, x);
#pragma unroll
                    for (int t = 0; t < 4; ++t) M[t] = l2add(M[t], l2mul(c, x[t]));
                }
            }
        }
        // canonical before the exact (canonical) grid reduction
#pragma unroll
        for (int t = 0; t < 4; ++t) acc[t] = l2canon(l2mul(bt[t], S[t]));
    }
    grid_reduce<4>(acc, a.partials, a.ticket, a.out8);
}

// Fold every row (and beta as row W) from n_in to n_in/2 copies.
__global__ void __launch_bounds__(kThreads)
    fold_rows_kernel(const fp2* __restrict__ A, int n_in, fp2* __restrict__ Aout, int W,
                     const fp2* __restrict__ beta, fp2* __restrict__ beta_out, fp2 r)
{
    const int n_out = n_in >> 1;
    const long long item = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (item >= (long long)(W + 1) * n_out) return;
    const int i = (int)(item % n_out);
    const int w = (int)(item / n_out);
    const fp2* src = w < W ? A + (size_t)w * n_in : beta;
    fp2* dst = w < W ? Aout + (size_t)w * n_out : beta_out;
    st2(dst + i, l2fold(ld2(src + 2 * (size_t)i), ld2(src + 2 * (size_t)i + 1), r));
}

// One block per 64 copies: stage the copies' copy_size bytes in shared memory,
// then write the wire-major packed table V[w][c] (1 KB contiguous per wire) and
// the copy-major base-field input vector x[c * W + w].
constexpr int kPixCopies = 64;
__global__ void __launch_bounds__(kThreads)
    table_from_pixels_kernel(const unsigned char* __restrict__ pix, int n_real, int n_pad,
                             int copy_size, int W, int const_idx, u64 const_val,
                             fp2* __restrict__ table, u64* __restrict__ inputs)
{
    extern __shared__ unsigned char tile[];  // [kPixCopies][copy_size]
    const int c0 = blockIdx.x * kPixCopies;
    const int nb = kPixCopies * copy_size;
    const size_t g0 = (size_t)c0 * copy_size;
    const size_t gend = (size_t)n_real * copy_size;
    for (int i = threadIdx.x; i < nb; i += blockDim.x)
        tile[i] = (g0 + i < gend) ? pix[g0 + i] : 0;
    __syncthreads();
    auto value = [&](int cl, int w) -> u64 {
        if (c0 + cl >= n_real) return 0;
        if (w < copy_size) return tile[cl * copy_size + w];
        return w == const_idx ? const_val : 0;
    };
    if (table) {
        for (int i = threadIdx.x; i < W * kPixCopies; i += blockDim.x) {
            const int w = i / kPixCopies, cl = i % kPixCopies;
            if (c0 + cl < n_pad) st2(table + (size_t)w * n_pad + c0 + cl, mk(value(cl, w), 0));
        }
    }
    if (inputs) {
        for (int i = threadIdx.x; i < W * kPixCopies; i += blockDim.x) {
            const int cl = i / W, w = i % W;
            if (c0 + cl < n_pad) inputs[(size_t)(c0 + cl) * W + w] = value(cl, w);
        }
    }
}

// (re[i], im[i]) -> packed
__global__ void pack_kernel(const u64* __restrict__ re, const u64* __restrict__ im, size_t n,
                            fp2* __restrict__ out)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) st2(out + i, mk(__ldg(re + i), __ldg(im + i)));
}

__global__ void fold_soa_kernel(const u64* __restrict__ in_re, const u64* __restrict__ in_im,
                                size_t n_out, fp2 r, u64* __restrict__ out_re,
                                u64* __restrict__ out_im)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_out) return;
    const ulonglong2 re = __ldg(reinterpret_cast<const ulonglong2*>(in_re) + i);
    const ulonglong2 im = __ldg(reinterpret_cast<const ulonglong2*>(in_im) + i);
    const fp2 o = f2fold(mk(re.x, im.x), mk(re.y, im.y), r);
    out_re[i] = o.re;
    out_im[i] = o.im;
}

__global__ void fold_aos_kernel(const fp2* __restrict__ in, size_t n_out, fp2 r,
                                fp2* __restrict__ out)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_out) return;
    st2(out + i, f2fold(ld2(in + 2 * i), ld2(in + 2 * i + 1), r));
}

__global__ void expand_soa_kernel(const u64* __restrict__ in_re, const u64* __restrict__ in_im,
                                  size_t n_src, size_t nc, u64* __restrict__ out_re,
                                  u64* __restrict__ out_im)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_src * nc) return;
    const size_t s = i / nc;
    out_re[i] = __ldg(in_re + s);
    out_im[i] = __ldg(in_im + s);
}

// lo[k] = prod_{j<h} eq(bit_j(k), z_j);  hi[m] = init * prod_{j<hb} eq(bit_j(m), z_{h+j})
__global__ void eq_tables_kernel(const fp2* __restrict__ z, int h, int hb, fp2 init,
                                 fp2* __restrict__ lo, fp2* __restrict__ hi)
{
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long nlo = 1ll << h, nhi = 1ll << hb;
    if (idx >= nlo + nhi) return;
    const fp2 one = mk(1, 0);
    if (idx < nlo) {
        fp2 v = one;
        for (int j = 0; j < h; ++j) {
            const fp2 zj = ld2(z + j);
            v = f2mul(v, ((idx >> j) & 1) ? zj : f2sub(one, zj));
        }
        st2(lo + idx, v);
    } else {
        const long long m = idx - nlo;
        fp2 v = init;
        for (int j = 0; j < hb; ++j) {
            const fp2 zj = ld2(z + h + j);
            v = f2mul(v, ((m >> j) & 1) ? zj : f2sub(one, zj));
        }
        st2(hi + m, v);
    }
}

__global__ void beta_expand_kernel(const fp2* __restrict__ lo, const fp2* __restrict__ hi, int h,
                                   size_t n, u64* __restrict__ out_re, u64* __restrict__ out_im,
                                   fp2* __restrict__ out_aos)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const fp2 v = f2mul(ld2(hi + (i >> h)), ld2(lo + (i & (((size_t)1 << h) - 1))));
    if (out_aos) {
        st2(out_aos + i, v);
    } else {
        out_re[i] = v.re;
        out_im[i] = v.im;
    }
}

// Batched eq tables: frame blockIdx.y, z at d_z + frame * z_stride, tables at
// tabs + frame * (2^h + 2^hb) (lo first, then hi with `init` folded in).
__global__ void eq_tables_batch_kernel(const fp2* __restrict__ d_z, int z_stride, int h, int hb,
                                       fp2 init, fp2* __restrict__ tabs)
{
    const long long nlo = 1ll << h, nhi = 1ll << hb;
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= nlo + nhi) return;
    const fp2* z = d_z + (size_t)blockIdx.y * z_stride;
    fp2* t = tabs + (size_t)blockIdx.y * (size_t)(nlo + nhi);
    const fp2 one = mk(1, 0);
    fp2 v = idx < nlo ? one : init;
    const long long bits = idx < nlo ? idx : idx - nlo;
    const int n = idx < nlo ? h : hb, off = idx < nlo ? 0 : h;
    for (int j = 0; j < n; ++j) {
        const fp2 zj = ld2(z + off + j);
        v = f2mul(v, ((bits >> j) & 1) ? zj : f2sub(one, zj));
    }
    st2(t + idx, v);
}

__global__ void beta_expand_batch_kernel(const fp2* __restrict__ tabs, int h, int hb,
                                         fp2* __restrict__ out, size_t out_stride)
{
    const size_t n = (size_t)1 << (h + hb);
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const fp2* t = tabs + (size_t)blockIdx.y * (((size_t)1 << h) + ((size_t)1 << hb));
    const fp2* lo = t;
    const fp2* hi = t + ((size_t)1 << h);
    st2(out + (size_t)blockIdx.y * out_stride + i,
        f2mul(ld2(hi + (i >> h)), ld2(lo + (i & (((size_t)1 << h) - 1)))));
}

// sum_i reduce(x[i]) * hi[i >> h] * lo[i & (2^h - 1)]. For h >= 3 every thread takes
// 8 consecutive inputs of one row (four 16-byte loads) and multiplies the row
// weight once; otherwise one input per step.
__global__ void __launch_bounds__(kThreads)
    mle_kernel(const u64* __restrict__ x, size_t n, int h, const fp2* __restrict__ lo,
               const fp2* __restrict__ hi, fp2* partials, unsigned* ticket, u64* out)
{
    fp2 acc[1] = {f2zero()};
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    const size_t tid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const size_t fmask = ((size_t)1 << h) - 1;
    if (h >= 3) {
        const size_t n8 = n >> 3;
        for (size_t q = tid; q < n8; q += stride) {
            const size_t base = q << 3;
            const ulonglong2* src = reinterpret_cast<const ulonglong2*>(x + base);
            ulonglong2 v[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) v[j] = __ldg(src + j);
            const fp2* l = lo + (base & fmask);
            // 8 products < 2^61 + 8 each: fold the raw sum after four of them
            fp2 s = f2zero();
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const fp2 l0 = ld2(l + 2 * j), l1 = ld2(l + 2 * j + 1);
                const u64 x0 = fold61(v[j].x), x1 = fold61(v[j].y);
                s.re += lmul(l0.re, x0) + lmul(l1.re, x1);
                s.im += lmul(l0.im, x0) + lmul(l1.im, x1);
                if (j & 1) s = mk(fold61(s.re), fold61(s.im));
            }
            acc[0] = l2add(acc[0], l2mul(s, ld2(hi + (base >> h))));
        }
    } else {
        for (size_t i = tid; i < n; i += stride) {
            const fp2 w = l2mul(ld2(hi + (i >> h)), ld2(lo + (i & fmask)));
            const u64 xv = fold61(__ldg(x + i));
            acc[0] = l2add(acc[0], mk(lmul(w.re, xv), lmul(w.im, xv)));
        }
    }
    acc[0] = l2canon(acc[0]);
    grid_reduce<1>(acc, partials, ticket, out);
}

// product-term orientation: put the wire shared by most terms second (group key)
void orient_terms(std::map<std::pair<int, int>, fp2>& terms, GateForm& out)
{
    std::map<int, int> deg;
    for (auto& kv : terms) {
        deg[kv.first.first]++;
        if (kv.first.second != kv.first.first) deg[kv.first.second]++;
    }
    std::map<std::pair<int, int>, fp2> by_b;  // key (b, a)
    for (auto& kv : terms) {
        int a = kv.first.first, b = kv.first.second;
        if (deg[a] > deg[b] || (deg[a] == deg[b] && a > b)) std::swap(a, b);
        auto it = by_b.find({b, a});
        if (it == by_b.end())
            by_b[{b, a}] = kv.second;
        else
            it->second = f2add(it->second, kv.second);
    }
    for (auto& kv : by_b) {
        if (f2is0(kv.second)) continue;
        out.tb.push_back(kv.first.first);
        out.ta.push_back(kv.first.second);
        out.tc.push_back(kv.second);
    }
}

}  // namespace

int last_launch_count() { return t_launches; }

void launch_eq_tables(const fp2* d_z, int h, int hb, fp2 init, fp2* lo, fp2* hi, cudaStream_t s)
{
    const size_t nt = ((size_t)1 << h) + ((size_t)1 << hb);
    eq_tables_kernel<<<blocks_for(nt, kThreads), kThreads, 0, s>>>(d_z, h, hb, init, lo, hi);
}

bool build_gate_form(int n_gates, const int* type, const int* in0, const int* in1,
                     const u64* z_re, const u64* z_im, int n_wires, GateForm& out)
{
    // (k0, k1, k2, k3) of k0 + k1*x + k2*y + k3*x*y for types 0..12
    static const int K[13][4] = {
        {0, 0, 0, 1},    // 0 mul
        {0, 1, 1, 0},    // 1 add
        {0, 1, -1, 0},   // 2 sub
        {0, 1, 0, 0},    // 3 mux, select x
        {0, 0, 1, 0},    // 4 mux, select y
        {0, 1, 1, -1},   // 5 or
        {0, 1, 1, -2},   // 6 xor
        {1, -1, 0, 0},   // 7 not
        {1, 0, 0, -1},   // 8 nand
        {1, -1, -1, 1},  // 9 nor
        {1, -1, -1, 2},  // 10 nxor
        {0, 0, 1, -1},   // 11 naab
        {0, 1, 0, 0},    // 12 pass
    };
    out.K0 = f2zero();
    out.L.assign((size_t)n_wires, f2zero());
    out.ta.clear();
    out.tb.clear();
    out.tc.clear();
    std::map<std::pair<int, int>, fp2> terms;
    for (int g = 0; g < n_gates; ++g) {
        const int tp = type[g];
        const int* k = (tp >= 0 && tp <= 12) ? K[tp] : K[12];  // other types act as pass
        const fp2 z = mk(z_re[g], z_im[g]);
        const int a = in0[g], b = in1[g];
        const bool use_a = k[1] != 0 || k[3] != 0, use_b = k[2] != 0 || k[3] != 0;
        if ((use_a && (a < 0 || a >= n_wires)) || (use_b && (b < 0 || b >= n_wires))) {
            set_error(TP_ERR_ARG, "gate %d reads wire (%d, %d) outside [0, %d)", g, a, b, n_wires);
            return false;
        }
        if (z.re >= P61 || z.im >= P61) {
            set_error(TP_ERR_ARG, "z1[%d] is not a canonical field element", g);
            return false;
        }
        if (k[0]) out.K0 = f2add(out.K0, f2scale(z, from_small(k[0])));
        if (k[1]) out.L[a] = f2add(out.L[a], f2scale(z, from_small(k[1])));
        if (k[2]) out.L[b] = f2add(out.L[b], f2scale(z, from_small(k[2])));
        if (k[3]) {
            const std::pair<int, int> key = a <= b ? std::make_pair(a, b) : std::make_pair(b, a);
            auto it = terms.find(key);
            const fp2 c = f2scale(z, from_small(k[3]));
            if (it == terms.end())
                terms[key] = c;
            else
                it->second = f2add(it->second, c);
        }
    }
    orient_terms(terms, out);
    return true;
}

bool upload_gate_form(const GateForm& g, DevGateForm& d, cudaStream_t s)
{
    d.K0 = g.K0;
    d.n_wires = (int)g.L.size();
    d.n_terms = (int)g.tc.size();
    d.L = (fp2*)dev_alloc(sizeof(fp2) * g.L.size(), s);
    d.ab = (int2*)dev_alloc(sizeof(int2) * std::max<size_t>(1, g.tc.size()), s);
    d.c = (fp2*)dev_alloc(sizeof(fp2) * std::max<size_t>(1, g.tc.size()), s);
    if (!d.L || !d.ab || !d.c) return false;
    if (!upload_async(d.L, g.L.data(), sizeof(fp2) * g.L.size(), s)) return false;
    if (d.n_terms) {
        std::vector<int2> ab((size_t)d.n_terms);
        for (int i = 0; i < d.n_terms; ++i) ab[i] = make_int2(g.ta[i], g.tb[i]);
        if (!upload_async(d.ab, ab.data(), sizeof(int2) * ab.size(), s)) return false;
        if (!upload_async(d.c, g.tc.data(), sizeof(fp2) * g.tc.size(), s)) return false;
    }
    return true;
}

void free_gate_form(DevGateForm& d, cudaStream_t s)
{
    dev_free(d.L, s);
    dev_free(d.ab, s);
    dev_free(d.c, s);
    d.L = nullptr;
    d.ab = nullptr;
    d.c = nullptr;
}

bool workspace_init(ClaimWorkspace& w, size_t blocks, cudaStream_t s)
{
    if (w.ticket && blocks <= w.cap_blocks) return true;
    if (!w.ticket) {
        w.ticket = (unsigned*)dev_alloc(256, s);
        w.out8 = (u64*)dev_alloc(8 * sizeof(u64), s);
        if (!w.ticket || !w.out8) return false;
        TP_CUDA_OK(cudaMemsetAsync(w.ticket, 0, 256, s), "ticket init");
    }
    if (blocks > w.cap_blocks) {
        dev_free(w.partials, s);
        const size_t cap = std::max<size_t>(blocks, 1024);
        w.partials = (fp2*)dev_alloc(cap * 4 * sizeof(fp2), s);
        if (!w.partials) return false;
        w.cap_blocks = cap;
    }
    return true;
}

void workspace_free(ClaimWorkspace& w, cudaStream_t s)
{
    dev_free(w.partials, s);
    dev_free(w.ticket, s);
    dev_free(w.out8, s);
    w = ClaimWorkspace();
}

namespace {

void choose_slices(int n_pairs, int W, int n_terms, int& n_slices, int& wc, int& tc)
{
    Ctx* c = ctx();
    const long long target = (long long)(c ? c->n_sm : 148) * 2048;
    long long s = target / std::max(1, n_pairs);
    s = std::max(1ll, std::min<long long>(s, W));
    wc = (int)((W + s - 1) / s);
    n_slices = (W + wc - 1) / wc;
    tc = n_terms ? (n_terms + n_slices - 1) / n_slices : 0;
}

ClaimArgs base_args(const DevGateForm& g, int W, int n_pairs, ClaimWorkspace& ws)
{
    ClaimArgs a;
    memset(&a, 0, sizeof(a));
    a.W = W;
    a.n_pairs = n_pairs;
    choose_slices(n_pairs, W, g.n_terms, a.n_slices, a.wc, a.tc);
    a.K0 = g.K0;
    a.L = g.L;
    a.ab = g.ab;
    a.cf = g.c;
    a.n_terms = g.n_terms;
    a.ticket = ws.ticket;
    a.out8 = nullptr;
    return a;
}

template <int MODE>
bool launch_claim(ClaimArgs& a, ClaimWorkspace& ws, cudaStream_t s)
{
    const size_t items = (size_t)a.n_pairs * (size_t)a.n_slices;
    const unsigned blocks = blocks_for(items, kThreads);
    if (!workspace_init(ws, blocks, s)) return false;
    a.partials = ws.partials;
    a.ticket = ws.ticket;
    if (!a.out8) a.out8 = ws.out8;
    claim_kernel<MODE><<<blocks, kThreads, 0, s>>>(a);
    ++t_launches;
    return !cuda_failed(cudaGetLastError(), "claim kernel launch");
}

}  // namespace

bool launch_claim_explicit(const DevGateForm& g, int n_copies, const u64* const* t12,
                           ClaimWorkspace& ws, cudaStream_t s)
{
    t_launches = 0;
    ClaimArgs a = base_args(g, g.n_wires, n_copies / 2, ws);
    a.n_in = n_copies;
    for (int i = 0; i < 12; ++i) a.t[i] = t12[i];
    return launch_claim<MODE_EXPLICIT>(a, ws, s);
}

bool launch_pack(const u64* re, const u64* im, size_t n, fp2* out, cudaStream_t s, int* launches)
{
    if (n == 0) return true;
    pack_kernel<<<blocks_for(n, kThreads), kThreads, 0, s>>>(re, im, n, out);
    ++*launches;
    return !cuda_failed(cudaGetLastError(), "pack launch");
}

// ---------------------------------------------------------------------------
// fold without a claim (table source): every row [0, W_rows) and beta

bool launch_fold_rows(const fp2* A, int n_in, fp2* Aout, int W_rows, const fp2* beta,
                      fp2* beta_out, fp2 r, cudaStream_t s, int* launches)
{
    const int n_out = n_in >> 1;
    const size_t items = (size_t)(W_rows + 1) * (size_t)n_out;
    fold_rows_kernel<<<blocks_for(items, kThreads), kThreads, 0, s>>>(A, n_in, Aout, W_rows, beta,
                                                                        beta_out, r);
    ++*launches;
    return !cuda_failed(cudaGetLastError(), "fold kernel launch");
}

// ---------------------------------------------------------------------------
// batch launches

bool launch_fold_soa(const u64* in_re, const u64* in_im, size_t n_out, fp2 r, u64* out_re,
                     u64* out_im, cudaStream_t s)
{
    t_launches = 0;
    if (n_out == 0) return true;
    fold_soa_kernel<<<blocks_for(n_out, kThreads), kThreads, 0, s>>>(in_re, in_im, n_out, r, out_re,
                                                                       out_im);
    t_launches = 1;
    return !cuda_failed(cudaGetLastError(), "fold launch");
}

bool launch_fold_aos(const fp2* in, size_t n_out, fp2 r, fp2* out, cudaStream_t s)
{
    t_launches = 0;
    if (n_out == 0) return true;
    fold_aos_kernel<<<blocks_for(n_out, kThreads), kThreads, 0, s>>>(in, n_out, r, out);
    t_launches = 1;
    return !cuda_failed(cudaGetLastError(), "fold launch");
}

bool launch_expand_soa(const u64* in_re, const u64* in_im, size_t n_src, size_t ncopies,
                       u64* out_re, u64* out_im, cudaStream_t s)
{
    t_launches = 0;
    const size_t n = n_src * ncopies;
    if (n == 0) return true;
    expand_soa_kernel<<<blocks_for(n, kThreads), kThreads, 0, s>>>(in_re, in_im, n_src, ncopies,
                                                                     out_re, out_im);
    t_launches = 1;
    return !cuda_failed(cudaGetLastError(), "expand launch");
}

bool launch_beta(const fp2* d_z, int n_z, fp2 init, u64* out_re, u64* out_im, fp2* out_aos,
                 cudaStream_t s)
{
    t_launches = 0;
    if (n_z <= 0) return true;
    const int h = n_z / 2, hb = n_z - h;
    fp2* tabs = (fp2*)dev_alloc(sizeof(fp2) * (((size_t)1 << h) + ((size_t)1 << hb)), s);
    if (!tabs) return false;
    fp2* lo = tabs;
    fp2* hi = tabs + ((size_t)1 << h);
    const size_t nt = ((size_t)1 << h) + ((size_t)1 << hb);
    eq_tables_kernel<<<blocks_for(nt, kThreads), kThreads, 0, s>>>(d_z, h, hb, init, lo, hi);
    const size_t n = (size_t)1 << n_z;
    beta_expand_kernel<<<blocks_for(n, kThreads), kThreads, 0, s>>>(lo, hi, h, n, out_re, out_im,
                                                                      out_aos);
    t_launches = 2;
    dev_free(tabs, s);
    return !cuda_failed(cudaGetLastError(), "beta launch");
}

bool launch_table_from_pixels(const unsigned char* d_pix, int n_real, int n_pad, int copy_size,
                              int W, int const_idx, u64 const_val, fp2* d_table, u64* d_inputs,
                              cudaStream_t s)
{
    t_launches = 0;
    if (n_real < 0 || n_real > n_pad || copy_size <= 0 || copy_size > W || W <= 0 ||
        const_idx >= W || (const_idx >= 0 && const_idx < copy_size) || const_val >= P61) {
        set_error(TP_ERR_ARG, "table_from_pixels: inconsistent layout (copies %d/%d, copy_size %d, "
                              "wires %d, const %d)", n_real, n_pad, copy_size, W, const_idx);
        return false;
    }
    const unsigned blocks = blocks_for((size_t)n_pad, kPixCopies);
    const size_t smem = (size_t)kPixCopies * copy_size;
    table_from_pixels_kernel<<<blocks, kThreads, smem, s>>>(d_pix, n_real, n_pad, copy_size, W,
                                                            const_idx, const_val, d_table, d_inputs);
    t_launches = 1;
    return !cuda_failed(cudaGetLastError(), "table_from_pixels launch");
}

void launch_eq_tables_batch(const fp2* d_z, int z_stride, int h, int hb, fp2 init, fp2* tabs,
                            int n, cudaStream_t s)
{
    const size_t nt = ((size_t)1 << h) + ((size_t)1 << hb);
    eq_tables_batch_kernel<<<dim3(blocks_for(nt, kThreads), n), kThreads, 0, s>>>(d_z, z_stride, h, hb,
                                                                               init, tabs);
}

bool launch_beta_batch(const fp2* d_z, int n_z, int n, fp2* d_out, cudaStream_t s, int* launches)
{
    if (n <= 0 || n_z <= 0) return true;
    const int h = n_z / 2, hb = n_z - h;
    const size_t nt = ((size_t)1 << h) + ((size_t)1 << hb);
    fp2* tabs = (fp2*)dev_alloc(sizeof(fp2) * nt * n, s);
    if (!tabs) return false;
    launch_eq_tables_batch(d_z, n_z, h, hb, mk(1, 0), tabs, n, s);
    const size_t m = (size_t)1 << n_z;
    beta_expand_batch_kernel<<<dim3(blocks_for(m, kThreads), n), kThreads, 0, s>>>(tabs, h, hb,
                                                                                 d_out, m);
    *launches += 2;
    dev_free(tabs, s);
    return !cuda_failed(cudaGetLastError(), "beta batch launch");
}

bool launch_mle_base_into(const u64* d_in, const fp2* d_z, int n_z, fp2* d_out, fp2* tabs,
                          fp2* partials, unsigned* ticket, unsigned max_blocks, cudaStream_t s)
{
    const int h = std::min(n_z, 12), hb = n_z - h;
    const size_t nt = ((size_t)1 << h) + ((size_t)1 << hb);
    fp2* lo = tabs;
    fp2* hi = tabs + ((size_t)1 << h);
    eq_tables_kernel<<<blocks_for(nt, kThreads), kThreads, 0, s>>>(d_z, h, hb, mk(1, 0), lo, hi);
    const size_t n = (size_t)1 << n_z;
    const size_t work = h >= 3 ? (n >> 3) : n;
    const unsigned blocks = (unsigned)std::max<size_t>(
        1, std::min<size_t>(blocks_for(work, kThreads), (size_t)max_blocks));
    mle_kernel<<<blocks, kThreads, 0, s>>>(d_in, n, h, lo, hi, partials, ticket,
                                           reinterpret_cast<u64*>(d_out));
    return !cuda_failed(cudaGetLastError(), "mle launch");
}

bool launch_mle_base(const u64* d_in, const fp2* d_z, int n_z, fp2* d_out, cudaStream_t s)
{
    t_launches = 0;
    Ctx* c = ctx();
    if (!c) return false;
    const int h = std::min(n_z, 12), hb = n_z - h;
    const size_t nt = ((size_t)1 << h) + ((size_t)1 << hb);
    // eq tables, up to 2048 blocks' partials (four words each), the ticket
    fp2* tabs = (fp2*)dev_alloc(sizeof(fp2) * nt + 4 * sizeof(fp2) * 2048 + 256, s);
    if (!tabs) return false;
    fp2* partials = tabs + nt;
    unsigned* ticket = reinterpret_cast<unsigned*>(partials + 4 * 2048);
    bool ok = !cuda_failed(cudaMemsetAsync(ticket, 0, sizeof(unsigned), s), "mle ticket") &&
              launch_mle_base_into(d_in, d_z, n_z, d_out, tabs, partials, ticket,
                                   (unsigned)std::min(c->n_sm * 8, 2048), s);
    if (ok) t_launches = 2;
    dev_free(tabs, s);
    return ok;
}

}  // namespace tp
