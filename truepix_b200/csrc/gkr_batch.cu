// Batched early-round GKR sumcheck: one launch per round for any number of
// frames (sessions), each with its own table, beta, gate form and challenge.
//
// Work decomposition: every frame contributes a "job" to a launch; a job is
// cut into CTAs = (tile of 32 claim pairs or copies) x (group of table rows).
// The 8 warps of a CTA split the group's rows, each lane owns one claim pair
// (table source) or one copy (byte source, pairs formed with the neighbouring
// lane). The four claim points of each pair are summed across the warps in
// shared memory, then warp 0 multiplies by beta, reduces and writes one
// partial per CTA; the last CTA of each job (ticket) writes the job's 8 u64.
// The same kernels serve a single frame (one job) and the reference ABI session.
//
// Sources (kinds):
//   0  table, claim only              1  table, fold by r then claim
//   2  frame bytes, claim only        3  frame bytes, fold by r then claim
// The byte kinds use the exact IMAD accumulation described in gkr_pixels.cu.
#include "gkr.h"
#include "gkr_internal.cuh"
#include "runtime.h"

#include <algorithm>
#include <cstring>

namespace tp {

namespace {

constexpr int kBT = 256;   // threads per CTA (8 warps)
constexpr int kWarps = kBT / 32;

__device__ __forceinline__ uint4 split4b(fp2 v)
{
    return make_uint4((u32)v.re, (u32)(v.re >> 32), (u32)v.im, (u32)(v.im >> 32));
}
__device__ __forceinline__ u64 combine2(u64 lo, u64 hi)
{
    return fold61(fold61(lo) + (hi >> 29) + ((hi & 0x1FFFFFFFull) << 32));
}
__device__ __forceinline__ void four4(fp2 v0, fp2 v1, fp2 (&o)[4])
{
    o[0] = v0;
    o[1] = v1;
    o[2] = l2at_m1(v0, v1);
    o[3] = l2at_2(v0, v1);
}
__device__ __forceinline__ fp2 partner2(fp2 v)
{
    return mk(__shfl_xor_sync(0xffffffffu, v.re, 1), __shfl_xor_sync(0xffffffffu, v.im, 1));
}
// sum of up to 8 nearly canonical values, lazily
__device__ __forceinline__ fp2 lazy_sum8(const fp2* v, int n, int stride)
{
    u64 re = 0, im = 0;
    for (int i = 0; i < n; ++i) {
        re += v[i * stride].re;
        im += v[i * stride].im;
        if ((i & 3) == 3) {
            re = fold61(re);
            im = fold61(im);
        }
    }
    return mk(fold61(re), fold61(im));
}

__device__ __forceinline__ u32 pbyte(const u32* tile, int pw, int row, int w)
{
    return (tile[row * pw + (w >> 2)] >> (8 * (w & 3))) & 0xFFu;
}

// Stage `rows` copies from copy c0 as words; copies >= n_real read as zero.
// With split_pairs, copy c0 + 2i goes to row i and c0 + 2i + 1 to row rows/2 + i,
// so the two copies a lane folds sit in different banks (pw is odd).
// Byte rows that are a multiple of 16 bytes are loaded as 16-byte vectors, all
// of a thread's loads issued before the first shared-memory store.
__device__ __forceinline__ int row_of(int r, int rows, bool split_pairs)
{
    return split_pairs ? ((r & 1) ? (rows >> 1) + (r >> 1) : (r >> 1)) : r;
}

__device__ void stage_rows(const Job& J, int c0, int rows, int pw, u32* tile, bool split_pairs = false)
{
    const int cs = J.cs;
    if ((cs & 15) == 0 && ((reinterpret_cast<size_t>(J.pix) & 15) == 0) && rows * cs <= 8 * 16 * kBT) {
        const int per = cs >> 4;                       // 16-byte vectors per row
        const int nv = rows * per;
        const uint4* src = reinterpret_cast<const uint4*>(J.pix + (size_t)c0 * cs);
        uint4 v[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const int q = threadIdx.x + k * kBT;
            v[k] = make_uint4(0, 0, 0, 0);
            if (q < nv && c0 + q / per < J.n_real) v[k] = __ldg(src + q);
        }
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const int q = threadIdx.x + k * kBT;
            if (q < nv) {
                const int r = q / per, j = 4 * (q - r * per);
                u32* d = tile + row_of(r, rows, split_pairs) * pw + j;
                d[0] = v[k].x;
                d[1] = v[k].y;
                d[2] = v[k].z;
                d[3] = v[k].w;
            }
        }
        const int wpr = cs >> 2;
        for (int i = threadIdx.x; i < rows * (pw - wpr); i += kBT) {
            const int r = i / (pw - wpr);
            tile[r * pw + wpr + (i - r * (pw - wpr))] = 0u;
        }
        return;
    }
    const long long nbytes = (long long)J.n_real * cs;
    const long long g0 = (long long)c0 * cs;
    unsigned char* tb = reinterpret_cast<unsigned char*>(tile);
    for (int i = threadIdx.x; i < rows * pw * 4; i += blockDim.x) {
        const int r = i / (pw * 4), j = i - r * pw * 4;
        const long long g = g0 + (long long)r * cs + j;
        tb[(size_t)row_of(r, rows, split_pairs) * pw * 4 + j] =
            (j < cs && g < nbytes) ? J.pix[g] : (unsigned char)0;
    }
}

__device__ __forceinline__ u64 bval(const Job& J, const u32* tile, int pw, int row, int c, int w)
{
    if (c >= J.n_real) return 0;
    if (w < J.cs) return pbyte(tile, pw, row, w);
    return w == J.const_idx ? J.const_val : 0;
}

// Job = blockIdx.y; copy its descriptor into shared memory. CTAs past the job's
// own count (jobs of a launch may differ in size) return false and exit.
__device__ __forceinline__ bool load_job(const Job* jobs, Job& sj)
{
    const int* src = reinterpret_cast<const int*>(jobs + blockIdx.y);
    int* dst = reinterpret_cast<int*>(&sj);
    for (int i = threadIdx.x; i < (int)(sizeof(Job) / 4); i += blockDim.x) dst[i] = __ldg(src + i);
    __syncthreads();
    return (int)blockIdx.x < sj.tiles * sj.groups;
}

// CTA epilogue: red[warp][pair][t] holds each warp's 4-point values (nearly
// canonical) for `pairs` pairs. Warp 0 sums them, adds K0 (group 0), multiplies
// by beta and reduces; the job's last CTA writes out8.
__device__ void cta_finish(const Job& J, fp2* red, int pairs, int pair0, int local, int g,
                           bool fold, const fp2* bt_override)
{
    __shared__ bool s_last;
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (warp == 0) {
        fp2 acc[4] = {f2zero(), f2zero(), f2zero(), f2zero()};
        const int p = pair0 + lane;
        if (lane < pairs && p < J.n_pairs) {
            fp2 b4[4];
            if (fold) {
                const fp2* q = J.beta + 4 * (size_t)p;
                const fp2 b0 = l2fold(ld2(q), ld2(q + 1), J.r), b1 = l2fold(ld2(q + 2), ld2(q + 3), J.r);
                if (g == 0) {
                    st2(J.beta_out + 2 * (size_t)p, b0);
                    st2(J.beta_out + 2 * (size_t)p + 1, b1);
                }
                four4(b0, b1, b4);
            } else {
                four4(ld2(J.beta + 2 * (size_t)p), ld2(J.beta + 2 * (size_t)p + 1), b4);
            }
#pragma unroll
            for (int t = 0; t < 4; ++t) {
                fp2 v = lazy_sum8(red + (size_t)lane * 4 + t, kWarps, 32 * 4);
                if (g == 0) v = l2add(v, J.K0);
                acc[t] = l2canon(l2mul(b4[t], v));
            }
        }
#pragma unroll
        for (int t = 0; t < 4; ++t) acc[t] = warp_sum(acc[t]);
        if (lane == 0) {
#pragma unroll
            for (int t = 0; t < 4; ++t) stcg2(J.partials + (size_t)local * 4 + t, acc[t]);
            __threadfence();
            const unsigned prev = atomicAdd(J.ticket, 1u);
            s_last = (prev == (unsigned)(J.tiles * J.groups - 1));
        }
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    const int n = J.tiles * J.groups;
    fp2 tot[4] = {f2zero(), f2zero(), f2zero(), f2zero()};
    for (int i = threadIdx.x; i < n; i += blockDim.x)
#pragma unroll
        for (int t = 0; t < 4; ++t) tot[t] = f2add(tot[t], ldcg2(J.partials + (size_t)i * 4 + t));
#pragma unroll
    for (int t = 0; t < 4; ++t) tot[t] = warp_sum(tot[t]);
    __syncthreads();
    if (lane == 0)
#pragma unroll
        for (int t = 0; t < 4; ++t) red[warp * 4 + t] = tot[t];
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int t = 0; t < 4; ++t) {
            fp2 v = lane < kWarps ? red[lane * 4 + t] : f2zero();
            v = warp_sum(v);
            if (lane == 0) {
                J.out8[2 * t] = v.re;
                J.out8[2 * t + 1] = v.im;
            }
        }
    }
    if (threadIdx.x == 0) *J.ticket = 0u;
}

// Epilogue of one warp: lane = claim pair p with 4-point values V (nearly
// canonical). Adds K0 (group 0), multiplies by beta at the four points (beta is
// folded by r first for fold kinds; group 0 stores the folded pair), sums over
// the warp. CTA level: the 8 warp sums go through shared memory to one partial
// per CTA; the job's last CTA (ticket) writes the job's 8 u64.
__device__ void warp_claim(const Job& J, fp2 (&V)[4], int p, bool live, int g, bool fold,
                           fp2 (&acc)[4])
{
#pragma unroll
    for (int t = 0; t < 4; ++t) acc[t] = f2zero();
    if (live) {
        fp2 b4[4];
        if (fold) {
            const fp2* q = J.beta + 4 * (size_t)p;
            const fp2 b0 = l2fold(ld2(q), ld2(q + 1), J.r), b1 = l2fold(ld2(q + 2), ld2(q + 3), J.r);
            if (g == 0) {
                st2(J.beta_out + 2 * (size_t)p, b0);
                st2(J.beta_out + 2 * (size_t)p + 1, b1);
            }
            four4(b0, b1, b4);
        } else {
            four4(ld2(J.beta + 2 * (size_t)p), ld2(J.beta + 2 * (size_t)p + 1), b4);
        }
#pragma unroll
        for (int t = 0; t < 4; ++t) {
            const fp2 v = g == 0 ? l2add(V[t], J.K0) : V[t];
            acc[t] = l2canon(l2mul(b4[t], v));
        }
    }
#pragma unroll
    for (int t = 0; t < 4; ++t) acc[t] = warp_sum(acc[t]);
}

__device__ void cta_combine(const Job& J, const fp2 (&acc)[4], int local)
{
    __shared__ fp2 ws[kWarps][4];
    __shared__ bool s_last;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0)
#pragma unroll
        for (int t = 0; t < 4; ++t) ws[warp][t] = acc[t];
    __syncthreads();
    if (threadIdx.x == 0) {
        fp2 tot[4];
#pragma unroll
        for (int t = 0; t < 4; ++t) {
            tot[t] = ws[0][t];
            for (int w = 1; w < kWarps; ++w) tot[t] = f2add(tot[t], ws[w][t]);
            stcg2(J.partials + (size_t)local * 4 + t, tot[t]);
        }
        __threadfence();
        const unsigned prev = atomicAdd(J.ticket, 1u);
        s_last = (prev == (unsigned)(J.tiles * J.groups - 1));
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    const int n = J.tiles * J.groups;
    fp2 tot[4] = {f2zero(), f2zero(), f2zero(), f2zero()};
    for (int i = threadIdx.x; i < n; i += blockDim.x)
#pragma unroll
        for (int t = 0; t < 4; ++t) tot[t] = f2add(tot[t], ldcg2(J.partials + (size_t)i * 4 + t));
#pragma unroll
    for (int t = 0; t < 4; ++t) tot[t] = warp_sum(tot[t]);
    __syncthreads();
    if (lane == 0)
#pragma unroll
        for (int t = 0; t < 4; ++t) ws[warp][t] = tot[t];
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
        for (int t = 0; t < 4; ++t) {
            fp2 v = ws[0][t];
            for (int w = 1; w < kWarps; ++w) v = f2add(v, ws[w][t]);
            J.out8[2 * t] = v.re;
            J.out8[2 * t + 1] = v.im;
        }
        *J.ticket = 0u;
    }
}

// ---------------------------------------------------------------------------
// kinds 0/1: table source. lane = claim pair, warp = slice of the group's rows
template <bool FOLD>
__device__ __forceinline__ void trow(const Job& J, int w, int p, fp2& x0, fp2& x1, bool store)
{
    if (w >= J.W_rows) {
        x0 = x1 = f2zero();
        return;
    }
    const fp2* row = J.A + (size_t)w * J.n_in;
    if (!FOLD) {
        x0 = ld2(row + 2 * (size_t)p);
        x1 = ld2(row + 2 * (size_t)p + 1);
    } else {
        const fp2* q = row + 4 * (size_t)p;
        const fp2 a0 = ld2(q), a1 = ld2(q + 1), a2 = ld2(q + 2), a3 = ld2(q + 3);
        x0 = l2fold(a0, a1, J.r);
        x1 = l2fold(a2, a3, J.r);
        if (store) {
            fp2* o = J.Aout + (size_t)w * (J.n_in >> 1) + 2 * (size_t)p;
            st2(o, x0);
            st2(o + 1, x1);
        }
    }
}

template <bool FOLD>
__global__ void __launch_bounds__(kBT, 4) table_round_kernel(const Job* __restrict__ jobs)
{
    __shared__ __align__(16) Job J;
    __shared__ __align__(16) fp2 red[kWarps * 32 * 4];
    if (!load_job(jobs, J)) return;
    const int local = blockIdx.x;
    const int tile = local / J.groups, g = local - tile * J.groups;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int p = tile * 32 + lane;
    const bool live = p < J.n_pairs;
    const int pq = live ? p : 0;   // dead lanes read pair 0 (in bounds) and store nothing

    // rows of this warp: group g is [g*wpg, (g+1)*wpg), split over 8 warps
    const int gr0 = g * J.wpg, gr1 = min(J.W_rows, gr0 + J.wpg);
    const int per = (gr1 - gr0 + kWarps - 1) / kWarps;
    const int r0 = gr0 + warp * per, r1 = min(gr1, r0 + per);
    u64 s0r = 0, s0i = 0, s1r = 0, s1i = 0;
    int w = r0;
    // two rows per step: their eight 16-byte loads are issued before any use
    for (; w + 1 < r1; w += 2) {
        fp2 x0, x1, y0, y1;
        trow<FOLD>(J, w, pq, x0, x1, live);
        trow<FOLD>(J, w + 1, pq, y0, y1, live);
        const fp2 l = ld2(J.L + w), m = ld2(J.L + w + 1);
        const fp2 a0 = l2mul(l, x0), a1 = l2mul(l, x1), b0 = l2mul(m, y0), b1 = l2mul(m, y1);
        s0r = fold61(s0r + a0.re + b0.re);
        s0i = fold61(s0i + a0.im + b0.im);
        s1r = fold61(s1r + a1.re + b1.re);
        s1i = fold61(s1i + a1.im + b1.im);
    }
    if (w < r1) {
        fp2 x0, x1;
        trow<FOLD>(J, w, pq, x0, x1, live);
        const fp2 l = ld2(J.L + w);
        const fp2 a0 = l2mul(l, x0), a1 = l2mul(l, x1);
        s0r = fold61(s0r + a0.re);
        s0i = fold61(s0i + a0.im);
        s1r = fold61(s1r + a1.re);
        s1i = fold61(s1i + a1.im);
    }
    fp2 V[4];
    four4(mk(fold61(s0r), fold61(s0i)), mk(fold61(s1r), fold61(s1i)), V);

    // product terms of (group, warp)
    const int tper = (J.tpg + kWarps - 1) / kWarps;
    const int e0 = min(J.n_terms, g * J.tpg + warp * tper);
    const int e1 = min(J.n_terms, min(g * J.tpg + J.tpg, e0 + tper));
    if (e0 < e1) {
        fp2 M0 = f2zero(), M1 = f2zero();
        int cur_b = J.ab[e0].y;
        for (int e = e0; e <= e1; ++e) {
            if (e == e1 || J.ab[e].y != cur_b) {
                fp2 xb[4], M[4];
                trow<FOLD>(J, cur_b, pq, xb[0], xb[1], false);
                four4(xb[0], xb[1], xb);
                four4(M0, M1, M);
#pragma unroll
                for (int t = 0; t < 4; ++t) V[t] = l2add(V[t], l2mul(xb[t], M[t]));
                M0 = M1 = f2zero();
                if (e == e1) break;
                cur_b = J.ab[e].y;
            }
            const fp2 c = ld2(J.cf + e);
            fp2 x0, x1;
            trow<FOLD>(J, J.ab[e].x, pq, x0, x1, false);
            M0 = l2add(M0, l2mul(c, x0));
            M1 = l2add(M1, l2mul(c, x1));
        }
    }
#pragma unroll
    for (int t = 0; t < 4; ++t) red[((size_t)warp * 32 + lane) * 4 + t] = V[t];
    cta_finish(J, red, 32, tile * 32, local, g, FOLD, nullptr);
}

// ---------------------------------------------------------------------------
// byte rows: the 16 bytes of vector q of copy c (zero past n_real)
__device__ __forceinline__ uint4 prow16(const Job& J, int c, int q)
{
    if (c >= J.n_real) return make_uint4(0, 0, 0, 0);
    return __ldg(reinterpret_cast<const uint4*>(J.pix + (size_t)c * J.cs) + q);
}
__device__ __forceinline__ u32 vbyte(const uint4& v, int k)
{
    const u32 word = k < 8 ? (k < 4 ? v.x : v.y) : (k < 12 ? v.z : v.w);
    return (word >> (8 * (k & 3))) & 0xFFu;
}
__device__ __forceinline__ u64 gval(const Job& J, int c, int w)
{
    if (c >= J.n_real) return 0;
    if (w < J.cs) return J.pix[(size_t)c * J.cs + w];
    return w == J.const_idx ? J.const_val : 0;
}

// kind 2: claim over the frame bytes. CTA = 256 claim pairs x one group of
// 16-wire units; lane = pair (copies 2p, 2p+1 read with 16-byte loads).
__global__ void __launch_bounds__(kBT, 4) pix_claim_kernel(const Job* __restrict__ jobs)
{
    __shared__ __align__(16) Job J;
    __shared__ uint4 Ls[512];
    if (!load_job(jobs, J)) return;
    const int local = blockIdx.x;
    const int tile = local / J.groups, g = local - tile * J.groups;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int cs = J.cs;
    const int w0 = 16 * g * J.wpg, w1 = min(cs, w0 + 16 * J.wpg);
    for (int w = w0 + threadIdx.x; w < w1; w += blockDim.x) Ls[w - w0] = split4b(ld2(J.L + w));
    __syncthreads();
    const int p = tile * kBT + warp * 32 + lane;
    const bool live = p < J.n_pairs;
    const int ca = 2 * p, cb = ca + 1;
    u64 A0 = 0, A1 = 0, A2 = 0, A3 = 0, B0 = 0, B1 = 0, B2 = 0, B3 = 0;
    if (J.vec) {
        for (int q = w0 >> 4; q < (w1 + 15) >> 4; ++q) {
            const uint4 va = prow16(J, live ? ca : J.n_real, q);
            const uint4 vb = prow16(J, live ? cb : J.n_real, q);
#pragma unroll
            for (int k = 0; k < 16; ++k) {
                const u32 xa = vbyte(va, k), xb = vbyte(vb, k);
                const uint4 l = Ls[16 * q + k - w0];
                A0 += (u64)l.x * xa; A1 += (u64)l.y * xa; A2 += (u64)l.z * xa; A3 += (u64)l.w * xa;
                B0 += (u64)l.x * xb; B1 += (u64)l.y * xb; B2 += (u64)l.z * xb; B3 += (u64)l.w * xb;
            }
        }
    } else {
        for (int w = w0; w < w1; ++w) {
            const u32 xa = live ? (u32)gval(J, ca, w) : 0u, xb = live ? (u32)gval(J, cb, w) : 0u;
            const uint4 l = Ls[w - w0];
            A0 += (u64)l.x * xa; A1 += (u64)l.y * xa; A2 += (u64)l.z * xa; A3 += (u64)l.w * xa;
            B0 += (u64)l.x * xb; B1 += (u64)l.y * xb; B2 += (u64)l.z * xb; B3 += (u64)l.w * xb;
        }
    }
    fp2 S0 = mk(combine2(A0, A1), combine2(A2, A3));
    fp2 S1 = mk(combine2(B0, B1), combine2(B2, B3));
    if (g == 0 && J.const_idx >= 0) {
        if (ca < J.n_real) S0 = l2add(S0, J.Lc);
        if (cb < J.n_real) S1 = l2add(S1, J.Lc);
    }
    fp2 V[4];
    four4(S0, S1, V);
    const int e0 = min(J.n_terms, g * J.tpg), e1 = min(J.n_terms, e0 + J.tpg);
    if (e0 < e1 && live) {
        fp2 M0 = f2zero(), M1 = f2zero();
        int cur_b = J.ab[e0].y;
        for (int e = e0; e <= e1; ++e) {
            if (e == e1 || J.ab[e].y != cur_b) {
                const u64 xb0 = gval(J, ca, cur_b), xb1 = gval(J, cb, cur_b);
                fp2 m4[4];
                four4(M0, M1, m4);
                const u64 x4[4] = {xb0, xb1, lsub(xb0 + xb0, xb1), lsub(xb1 + xb1, xb0)};
#pragma unroll
                for (int t = 0; t < 4; ++t)
                    V[t] = l2add(V[t], mk(lmul(m4[t].re, x4[t]), lmul(m4[t].im, x4[t])));
                M0 = M1 = f2zero();
                if (e == e1) break;
                cur_b = J.ab[e].y;
            }
            const fp2 cf = ld2(J.cf + e);
            const int w = J.ab[e].x;
            const u64 xa0 = gval(J, ca, w), xa1 = gval(J, cb, w);
            M0 = l2add(M0, mk(lmul(cf.re, xa0), lmul(cf.im, xa0)));
            M1 = l2add(M1, mk(lmul(cf.re, xa1), lmul(cf.im, xa1)));
        }
    }
    fp2 acc[4];
    warp_claim(J, V, p, live, g, false, acc);
    cta_combine(J, acc, local);
}

// ---------------------------------------------------------------------------
// kind 3: fold the byte table by r, store the folded rows, claim them.
// lane = output copy; 64 input copies staged per CTA.
__global__ void __launch_bounds__(kBT) pix_fold_claim_kernel(const Job* __restrict__ jobs)
{
    __shared__ __align__(16) Job J;
    __shared__ __align__(16) fp2 red[kWarps * 32 * 4];
    extern __shared__ __align__(16) unsigned char dsm[];
    if (!load_job(jobs, J)) return;
    const int local = blockIdx.x;
    const int tile = local / J.groups, g = local - tile * J.groups;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int cs = J.cs, pw = J.pw;
    const int nw = (cs + 3) >> 2;
    const int gw0 = g * J.wpg, gw1 = min(nw, gw0 + J.wpg);
    const int gn = 4 * J.wpg;
    uint4* Lm = reinterpret_cast<uint4*>(dsm);                  // [gn]
    uint4* Lr = Lm + gn;                                        // [gn]
    fp2* rd = reinterpret_cast<fp2*>(Lr + gn);                  // [511]
    u32* tile_w = reinterpret_cast<u32*>(rd + 511);             // [64][pw]
    const fp2 r = J.r;
    for (int i = threadIdx.x; i < 4 * (gw1 - gw0); i += blockDim.x) {
        const int w = 4 * gw0 + i;
        if (w < cs) {
            const fp2 l = ld2(J.L + w);
            const fp2 lr = l2canon(l2mul(l, r));
            Lr[i] = split4b(lr);
            Lm[i] = split4b(l2canon(l2sub(l, lr)));
        } else {
            Lr[i] = Lm[i] = make_uint4(0, 0, 0, 0);
        }
    }
    for (int k = threadIdx.x; k < 511; k += blockDim.x) {
        const int d = k - 255;
        const u64 m = (u64)(d < 0 ? -d : d);
        fp2 v = mk(lmul(r.re, m), lmul(r.im, m));
        if (d < 0) v = l2sub(f2zero(), v);
        rd[k] = l2canon(v);
    }
    const int o0 = tile * 32;
    stage_rows(J, 2 * o0, 64, pw, tile_w, true);
    __syncthreads();

    const int oc = o0 + lane;
    const int n_out = J.n_in >> 1;
    const bool live = oc < n_out;
    const int ra = lane, rb = 32 + lane;   // rows of input copies 2*oc and 2*oc + 1
    const int per = (gw1 - gw0 + kWarps - 1) / kWarps;
    const int j0 = gw0 + warp * per, j1 = min(gw1, j0 + per);
    fp2* out = J.Aout + oc;
    u64 A0 = 0, A1 = 0, A2 = 0, A3 = 0;
    for (int j = j0; j < j1; ++j) {
        const u32 va = tile_w[ra * pw + j], vb = tile_w[rb * pw + j];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int w = 4 * j + k;
            const u32 xa = (va >> (8 * k)) & 0xFFu, xb = (vb >> (8 * k)) & 0xFFu;
            if (live && w < cs) {
                const fp2 t = rd[(int)xb - (int)xa + 255];
                st2(out + (size_t)w * n_out, mk(fold61(t.re + xa), t.im));
            }
            const uint4 m = Lm[4 * (j - gw0) + k], q = Lr[4 * (j - gw0) + k];
            A0 += (u64)m.x * xa + (u64)q.x * xb;
            A1 += (u64)m.y * xa + (u64)q.y * xb;
            A2 += (u64)m.z * xa + (u64)q.z * xb;
            A3 += (u64)m.w * xa + (u64)q.w * xb;
        }
    }
    fp2 S = mk(combine2(A0, A1), combine2(A2, A3));
    if (g == 0 && warp == 0) {
        // the constant row and any zero rows in [cs, W_rows)
        for (int w = cs; w < J.W_rows; ++w) {
            fp2 x = f2zero();
            if (w == J.const_idx) {
                const u64 va = 2 * oc < J.n_real ? J.const_val : 0;
                const u64 vb = 2 * oc + 1 < J.n_real ? J.const_val : 0;
                x = l2fold(mk(va, 0), mk(vb, 0), r);
                S = l2add(S, l2mul(ld2(J.L + w), x));
            }
            if (live) st2(out + (size_t)w * n_out, x);
        }
    }

    auto folded = [&](int w) -> fp2 {
        const u64 va = bval(J, tile_w, pw, ra, 2 * oc, w);
        const u64 vb = bval(J, tile_w, pw, rb, 2 * oc + 1, w);
        if (w < cs) {
            const fp2 t = rd[(int)vb - (int)va + 255];
            return mk(fold61(t.re + va), t.im);
        }
        return l2fold(mk(va, 0), mk(vb, 0), r);
    };
    fp2 P[4] = {f2zero(), f2zero(), f2zero(), f2zero()};
    const int tper = (J.tpg + kWarps - 1) / kWarps;
    const int e0 = min(J.n_terms, g * J.tpg + warp * tper);
    const int e1 = min(J.n_terms, min(g * J.tpg + J.tpg, e0 + tper));
    if (e0 < e1) {
        fp2 M = f2zero();
        int cur_b = J.ab[e0].y;
        for (int e = e0; e <= e1; ++e) {
            if (e == e1 || J.ab[e].y != cur_b) {
                const fp2 xb = folded(cur_b);
                const fp2 Mo = partner2(M), xbo = partner2(xb);
                if ((lane & 1) == 0) {
                    fp2 m4[4], x4[4];
                    four4(M, Mo, m4);
                    four4(xb, xbo, x4);
#pragma unroll
                    for (int t = 0; t < 4; ++t) P[t] = l2add(P[t], l2mul(m4[t], x4[t]));
                }
                M = f2zero();
                if (e == e1) break;
                cur_b = J.ab[e].y;
            }
            M = l2add(M, l2mul(ld2(J.cf + e), folded(J.ab[e].x)));
        }
    }
    const fp2 So = partner2(S);
    if ((lane & 1) == 0) {
        fp2 V[4];
        four4(S, So, V);
#pragma unroll
        for (int t = 0; t < 4; ++t) red[((size_t)warp * 32 + (lane >> 1)) * 4 + t] = l2add(V[t], P[t]);
    } else {
#pragma unroll
        for (int t = 0; t < 4; ++t) red[((size_t)warp * 32 + 16 + (lane >> 1)) * 4 + t] = f2zero();
    }
    cta_finish(J, red, 16, tile * 16, local, g, true, nullptr);
}

// ---------------------------------------------------------------------------
// finish: for every job, the wire values at copy 0 (after an optional pending
// fold of the last two copies) and beta, canonical.
__global__ void __launch_bounds__(kBT) finish_kernel(const Job* __restrict__ jobs)
{
    const Job& J = jobs[blockIdx.y];
    const int w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w > J.W) return;
    const bool fold = J.kind & 1;
    if (w == J.W) {
        const fp2 b = fold ? l2fold(ld2(J.beta), ld2(J.beta + 1), J.r) : ld2(J.beta);
        st2(J.fin_beta, l2canon(b));
        return;
    }
    fp2 v = f2zero();
    if (w < J.W_rows) {
        if (J.pix) {
            auto val = [&](int c) -> u64 {
                if (c >= J.n_real) return 0;
                if (w < J.cs) return J.pix[(size_t)c * J.cs + w];
                return w == J.const_idx ? J.const_val : 0;
            };
            v = fold ? l2fold(mk(val(0), 0), mk(val(1), 0), J.r) : mk(val(0), 0);
        } else {
            const fp2* row = J.A + (size_t)w * J.n_in;
            v = fold ? l2fold(ld2(row), ld2(row + 1), J.r) : ld2(row);
        }
    }
    st2(J.fin + w, l2canon(v));
}

size_t pix_fold_smem(int wpg, int pw)
{
    return 32 * 4 * (size_t)wpg + 16 * 511 + 4 * 64 * (size_t)pw;
}

int pad_words_b(int cs)
{
    const int w = (cs + 3) / 4;
    return (w & 1) ? w : w + 1;
}

bool g_attrs = false;
bool set_attrs()
{
    if (g_attrs) return true;
    const int big = 160 * 1024;
    TP_CUDA_OK(cudaFuncSetAttribute(pix_fold_claim_kernel,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, big), "smem attr");
    g_attrs = true;
    return true;
}

}  // namespace

// ---------------------------------------------------------------------------
// host side

void plan_job(Job& j, int target_ctas)
{
    if (j.kind <= 1) {
        j.tiles = (j.n_pairs + 31) / 32;
        int groups = std::max(1, (target_ctas + j.tiles - 1) / j.tiles);
        groups = std::min(groups, std::max(1, (j.W_rows + kWarps - 1) / kWarps));
        j.wpg = (j.W_rows + groups - 1) / groups;
        j.groups = (j.W_rows + j.wpg - 1) / j.wpg;
    } else if (j.kind == 2) {
        j.tiles = (j.n_pairs + kBT - 1) / kBT;   // 256 claim pairs per CTA
        const int units = (j.cs + 15) / 16;      // 16-wire units
        int groups = std::max(1, (target_ctas + j.tiles - 1) / j.tiles);
        groups = std::min(groups, units);
        j.wpg = (units + groups - 1) / groups;
        j.groups = (units + j.wpg - 1) / j.wpg;
    } else {
        j.tiles = ((j.n_in >> 1) + 31) / 32;     // 32 output copies per CTA
        const int nw = (j.cs + 3) / 4;
        int groups = std::max(1, (target_ctas + j.tiles - 1) / j.tiles);
        groups = std::min(groups, std::max(1, (nw + kWarps - 1) / kWarps));
        j.wpg = (nw + groups - 1) / groups;
        j.groups = (nw + j.wpg - 1) / j.wpg;
    }
    j.pw = pad_words_b(j.cs);
    j.tpg = j.n_terms ? (j.n_terms + j.groups - 1) / j.groups : 0;
    j.vec = (j.kind >= 2 && (j.cs & 15) == 0 && (reinterpret_cast<size_t>(j.pix) & 15) == 0) ? 1 : 0;
}

bool prepare_round_kernels() { return set_attrs(); }

bool launch_round(const Job* d_jobs, const std::vector<Job>& jobs, int kind, cudaStream_t s,
                  int* launches)
{
    if (jobs.empty()) return true;
    if (!set_attrs()) return false;
    unsigned max_ctas = 0;
    for (const Job& j : jobs) max_ctas = std::max(max_ctas, (unsigned)(j.tiles * j.groups));
    const dim3 grid(max_ctas, (unsigned)jobs.size());
    if (kind == 0) {
        table_round_kernel<false><<<grid, kBT, 0, s>>>(d_jobs);
    } else if (kind == 1) {
        table_round_kernel<true><<<grid, kBT, 0, s>>>(d_jobs);
    } else {
        size_t smem = 0;
        for (const Job& j : jobs) smem = std::max(smem, pix_fold_smem(j.wpg, j.pw));
        if (kind == 2) pix_claim_kernel<<<grid, kBT, 0, s>>>(d_jobs);
        else pix_fold_claim_kernel<<<grid, kBT, smem, s>>>(d_jobs);
    }
    ++*launches;
    return !cuda_failed(cudaGetLastError(), "round kernel launch");
}

bool launch_finish(const Job* d_jobs, int n_jobs, int max_w, cudaStream_t s, int* launches)
{
    if (n_jobs == 0) return true;
    dim3 grid(blocks_for((size_t)max_w + 1, kBT), (unsigned)n_jobs);
    finish_kernel<<<grid, kBT, 0, s>>>(d_jobs);
    ++*launches;
    return !cuda_failed(cudaGetLastError(), "finish kernel launch");
}

}  // namespace tp
