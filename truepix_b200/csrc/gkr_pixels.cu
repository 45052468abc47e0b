// GKR input-layer kernels that read the frame's uint8 bytes directly.
//
// In TruePix's input layout (TruePix-main/Orion/Orion_nonzk/include/truepix/
// truepix_gkr.h:11-18) the input-layer table is V[w][c] = byte c*copy_size + w
// for w < copy_size, the circuit constant at w = const_idx, zero on the other
// wires and on padded copies. The first claim and the first fold therefore need
// only the bytes: these kernels stage 64 copies' bytes in shared memory and
// evaluate the round without ever writing the 2^23-entry Fp2 table
// (6 MB read instead of 128 MiB for a 1080p frame).
//
// With pixel values x < 2^8 and a canonical coefficient split as
// L = Lh*2^32 + Ll (Lh < 2^29), sum_w L[w]*x_w is accumulated exactly as two
// 64-bit sums of 32x32->64 products (IMAD.WIDE with accumulate) and reduced
// once per copy. The first fold uses x = a + r*(b - a) with r*k looked up in a
// shared table for k in [-255, 255], and the following claim uses
// L*x = (L - L*r)*a + (L*r)*b, again as unsigned IMAD accumulation.
#include "gkr.h"
#include "gkr_internal.cuh"
#include "runtime.h"

#include <algorithm>

namespace tp {

namespace {

constexpr int kT = 256;
constexpr int kClaimCopies = 64;   // claim over pixels: 64 copies x 4 wire slices
constexpr int kFoldCopies = 32;    // fold over pixels: 32 output copies x 8 wire slices

__device__ __forceinline__ uint4 split4(fp2 v)
{
    return make_uint4((u32)v.re, (u32)(v.re >> 32), (u32)v.im, (u32)(v.im >> 32));
}

// (lo + hi * 2^32) mod p, lo < 2^63, hi < 2^45 (raw IMAD sums) -> nearly canonical
__device__ __forceinline__ u64 combine(u64 lo, u64 hi)
{
    return fold61(fold61(lo) + (hi >> 29) + ((hi & 0x1FFFFFFFull) << 32));
}

// Stage `rows` copies starting at copy c0 into tile[rows][pw] words (zero past n_real).
__device__ void stage_pixels(const PixSrc& px, int c0, int rows, int pw, u32* tile)
{
    const int cs = px.cs;
    const long long nbytes_real = (long long)px.n_real * cs;
    const long long g0 = (long long)c0 * cs;
    if ((cs & 3) == 0 && ((reinterpret_cast<size_t>(px.pix) & 3) == 0)) {
        const int wpr = cs >> 2;
        const u32* src = reinterpret_cast<const u32*>(px.pix) + (g0 >> 2);
        const long long words_real = nbytes_real >> 2;
        for (int i = threadIdx.x; i < rows * wpr; i += blockDim.x) {
            const int r = i / wpr, j = i - r * wpr;
            tile[r * pw + j] = ((g0 >> 2) + i < words_real) ? __ldg(src + i) : 0u;
        }
        // zero the padding word(s) of every row
        for (int i = threadIdx.x; i < rows * (pw - wpr); i += blockDim.x) {
            const int r = i / (pw - wpr), j = wpr + i - r * (pw - wpr);
            tile[r * pw + j] = 0u;
        }
    } else {
        unsigned char* tb = reinterpret_cast<unsigned char*>(tile);
        for (int i = threadIdx.x; i < rows * pw * 4; i += blockDim.x) {
            const int r = i / (pw * 4), j = i - r * pw * 4;
            const long long g = g0 + (long long)r * cs + j;
            tb[i] = (j < cs && g < nbytes_real) ? px.pix[g] : (unsigned char)0;
        }
    }
}

__device__ __forceinline__ u32 pix_at(const u32* tile, int pw, int row, int w)
{
    return (tile[row * pw + (w >> 2)] >> (8 * (w & 3))) & 0xFFu;
}

// field value of wire w of copy `c` (tile row `row`)
__device__ __forceinline__ u64 pixval(const PixSrc& px, const u32* tile, int pw, int row, int c,
                                      int w)
{
    if (c >= px.n_real) return 0;
    if (w < px.cs) return pix_at(tile, pw, row, w);
    return w == px.const_idx ? px.const_val : 0;
}

// Exchange with the partner lane (copies 2p and 2p+1 sit in lanes 2k, 2k+1).
__device__ __forceinline__ fp2 partner(fp2 v)
{
    return mk(__shfl_xor_sync(0xffffffffu, v.re, 1), __shfl_xor_sync(0xffffffffu, v.im, 1));
}

// Four claim points from the values at the two copies of a pair (even lane view)
__device__ __forceinline__ void four(fp2 v0, fp2 v1, fp2 (&o)[4])
{
    o[0] = v0;
    o[1] = v1;
    o[2] = l2at_m1(v0, v1);
    o[3] = l2at_2(v0, v1);
}

// ---------------------------------------------------------------------------
// claim over the pixel table (no fold): one thread per (copy, wire slice)
__global__ void __launch_bounds__(kT) claim_pixels_kernel(const PixClaimArgs a)
{
    extern __shared__ __align__(16) unsigned char smem[];
    uint4* Ls = reinterpret_cast<uint4*>(smem);                       // [cs]
    u32* tile = reinterpret_cast<u32*>(smem + 16 * (size_t)a.px.cs);  // [64][pw]
    const int cs = a.px.cs, pw = a.pw;
    for (int w = threadIdx.x; w < cs; w += blockDim.x) Ls[w] = split4(ld2c(a.L + w));
    const int c0 = blockIdx.x * kClaimCopies;
    stage_pixels(a.px, c0, kClaimCopies, pw, tile);
    __syncthreads();

    const int cl = threadIdx.x % kClaimCopies, y = threadIdx.x / kClaimCopies;
    const int c = c0 + cl;
    const bool live = c < a.n_pad;   // pairs are never split: n_pad is even
    const int nw = (cs + 3) >> 2, ws = (nw + 3) / 4;
    const int j0 = y * ws, j1 = min(nw, j0 + ws);
    u64 A0 = 0, A1 = 0, A2 = 0, A3 = 0;
    for (int j = j0; j < j1; ++j) {
        const u32 v = tile[cl * pw + j];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int w = 4 * j + k;
            if (w < cs) {
                const u32 x = (v >> (8 * k)) & 0xFFu;
                const uint4 l = Ls[w];
                A0 += (u64)l.x * x;
                A1 += (u64)l.y * x;
                A2 += (u64)l.z * x;
                A3 += (u64)l.w * x;
            }
        }
    }
    fp2 S = mk(combine(A0, A1), combine(A2, A3));
    if (y == 0 && c < a.px.n_real && a.px.const_idx >= 0) S = l2add(S, a.Lc);

    // product terms of this slice: c * V[a] * V[b], grouped by b
    fp2 P[4] = {f2zero(), f2zero(), f2zero(), f2zero()};
    const int e0 = y * a.tc, e1 = min(a.n_terms, e0 + a.tc);
    if (e0 < e1) {
        fp2 M = f2zero();
        int cur_b = a.ab[e0].y;
        for (int e = e0; e <= e1; ++e) {
            if (e == e1 || a.ab[e].y != cur_b) {
                const u64 xb = pixval(a.px, tile, pw, cl, c, cur_b);
                const fp2 Mo = partner(M);
                const u64 xbo = __shfl_xor_sync(0xffffffffu, xb, 1);
                if ((cl & 1) == 0) {
                    fp2 m4[4];
                    four(M, Mo, m4);
                    const u64 x4[4] = {xb, xbo, lsub(xb + xb, xbo), lsub(xbo + xbo, xb)};
#pragma unroll
                    for (int t = 0; t < 4; ++t)
                        P[t] = l2add(P[t], mk(lmul(m4[t].re, x4[t]), lmul(m4[t].im, x4[t])));
                }
                M = f2zero();
                if (e == e1) break;
                cur_b = a.ab[e].y;
            }
            const fp2 cf = ld2c(a.cf + e);
            const u64 xa = pixval(a.px, tile, pw, cl, c, a.ab[e].x);
            M = l2add(M, mk(lmul(cf.re, xa), lmul(cf.im, xa)));
        }
    }

    fp2 acc[4] = {f2zero(), f2zero(), f2zero(), f2zero()};
    const fp2 So = partner(S);
    if ((cl & 1) == 0 && live) {
        const int p = c >> 1;
        fp2 s4[4], b4[4];
        four(S, So, s4);
        four(ld2c(a.beta + 2 * (size_t)p), ld2c(a.beta + 2 * (size_t)p + 1), b4);
#pragma unroll
        for (int t = 0; t < 4; ++t) {
            fp2 v = l2add(s4[t], P[t]);
            if (y == 0) v = l2add(v, a.K0);
            acc[t] = l2canon(l2mul(b4[t], v));
        }
    }
    grid_reduce<4>(acc, a.partials, a.ticket, a.out8);
}

// ---------------------------------------------------------------------------
// fold by r over the pixel table, write the folded Fp2 rows, claim the result
__global__ void __launch_bounds__(kT) fold_claim_pixels_kernel(const PixClaimArgs a)
{
    extern __shared__ __align__(16) unsigned char smem[];
    const int cs = a.px.cs, pw = a.pw;
    uint4* Lm = reinterpret_cast<uint4*>(smem);             // (L - L*r) split, [cs]
    uint4* Lr = Lm + cs;                                    // (L*r) split, [cs]
    fp2* rd = reinterpret_cast<fp2*>(Lr + cs);              // r*k, k = -255..255 -> [k + 255]
    u32* tile = reinterpret_cast<u32*>(rd + 511);           // [64][pw]
    const fp2 r = a.r;
    for (int w = threadIdx.x; w < cs; w += blockDim.x) {
        const fp2 l = ld2c(a.L + w);
        const fp2 lr = l2canon(l2mul(l, r));
        Lr[w] = split4(lr);
        Lm[w] = split4(l2canon(l2sub(l, lr)));
    }
    for (int k = threadIdx.x; k < 511; k += blockDim.x) {
        const int d = k - 255;
        const u64 m = (u64)(d < 0 ? -d : d);
        fp2 v = mk(lmul(r.re, m), lmul(r.im, m));
        if (d < 0) v = l2sub(f2zero(), v);
        rd[k] = l2canon(v);
    }
    const int o0 = blockIdx.x * kFoldCopies;  // first output copy of this block
    stage_pixels(a.px, 2 * o0, 2 * kFoldCopies, pw, tile);
    __syncthreads();

    const int ol = threadIdx.x % kFoldCopies, y = threadIdx.x / kFoldCopies;
    const int oc = o0 + ol;                    // output copy
    const bool live = oc < a.n_out;            // n_out is even: pairs are never split
    const int ra = 2 * ol, rb = 2 * ol + 1;    // tile rows of its two input copies
    const int n_out = a.n_out;
    const int nw = (cs + 3) >> 2, ws = (nw + 7) / 8;
    const int j0 = y * ws, j1 = min(nw, j0 + ws);
    fp2* out = a.Aout + oc;
    u64 A0 = 0, A1 = 0, A2 = 0, A3 = 0;
    for (int j = j0; j < j1; ++j) {
        const u32 va = tile[ra * pw + j], vb = tile[rb * pw + j];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int w = 4 * j + k;
            if (w < cs) {
                const u32 xa = (va >> (8 * k)) & 0xFFu, xb = (vb >> (8 * k)) & 0xFFu;
                const fp2 t = rd[(int)xb - (int)xa + 255];
                if (live) st2(out + (size_t)w * n_out, mk(fold61(t.re + xa), t.im));
                const uint4 m = Lm[w], q = Lr[w];
                A0 += (u64)m.x * xa + (u64)q.x * xb;
                A1 += (u64)m.y * xa + (u64)q.y * xb;
                A2 += (u64)m.z * xa + (u64)q.z * xb;
                A3 += (u64)m.w * xa + (u64)q.w * xb;
            }
        }
    }
    fp2 S = mk(combine(A0, A1), combine(A2, A3));
    if (y == 0 && live) {
        // constant wire and any zero rows between copy_size and W_rows
        for (int w = cs; w < a.W_rows; ++w) {
            fp2 x = f2zero();
            if (w == a.px.const_idx) {
                const u64 va = 2 * oc < a.px.n_real ? a.px.const_val : 0;
                const u64 vb = 2 * oc + 1 < a.px.n_real ? a.px.const_val : 0;
                x = l2fold(mk(va, 0), mk(vb, 0), r);
                S = l2add(S, l2mul(ld2c(a.L + w), x));
            }
            st2(out + (size_t)w * n_out, x);
        }
    }

    // product terms c * V[a] * V[b] at the folded copy
    fp2 P[4] = {f2zero(), f2zero(), f2zero(), f2zero()};
    const int e0 = y * a.tc, e1 = min(a.n_terms, e0 + a.tc);
    auto folded = [&](int w) -> fp2 {
        const u64 va = pixval(a.px, tile, pw, ra, 2 * oc, w);
        const u64 vb = pixval(a.px, tile, pw, rb, 2 * oc + 1, w);
        if (w < cs) {
            const fp2 t = rd[(int)vb - (int)va + 255];
            return mk(fold61(t.re + va), t.im);
        }
        return l2fold(mk(va, 0), mk(vb, 0), r);
    };
    if (e0 < e1) {
        fp2 M = f2zero();
        int cur_b = a.ab[e0].y;
        for (int e = e0; e <= e1; ++e) {
            if (e == e1 || a.ab[e].y != cur_b) {
                const fp2 xb = folded(cur_b);
                const fp2 Mo = partner(M), xbo = partner(xb);
                if ((ol & 1) == 0) {
                    fp2 m4[4], x4[4];
                    four(M, Mo, m4);
                    four(xb, xbo, x4);
#pragma unroll
                    for (int t = 0; t < 4; ++t) P[t] = l2add(P[t], l2mul(m4[t], x4[t]));
                }
                M = f2zero();
                if (e == e1) break;
                cur_b = a.ab[e].y;
            }
            M = l2add(M, l2mul(ld2c(a.cf + e), folded(a.ab[e].x)));
        }
    }

    fp2 acc[4] = {f2zero(), f2zero(), f2zero(), f2zero()};
    const fp2 So = partner(S);
    if ((ol & 1) == 0 && live) {
        const int p = oc >> 1;                 // claim pair of the folded table
        const fp2* q = a.beta + 4 * (size_t)p;
        const fp2 b0 = l2fold(ld2c(q), ld2c(q + 1), r), b1 = l2fold(ld2c(q + 2), ld2c(q + 3), r);
        if (y == 0) {
            st2(a.beta_out + 2 * (size_t)p, b0);
            st2(a.beta_out + 2 * (size_t)p + 1, b1);
        }
        fp2 s4[4], b4[4];
        four(S, So, s4);
        four(b0, b1, b4);
#pragma unroll
        for (int t = 0; t < 4; ++t) {
            fp2 v = l2add(s4[t], P[t]);
            if (y == 0) v = l2add(v, a.K0);
            acc[t] = l2canon(l2mul(b4[t], v));
        }
    }
    grid_reduce<4>(acc, a.partials, a.ticket, a.out8);
}

// fold by r over the pixel table without a claim (n_copies 2 -> 1, or two
// folds in a row): one thread per (output copy, row)
__global__ void __launch_bounds__(kT) fold_pixels_kernel(const PixSrc px, int W_rows, int n_out,
                                                         fp2 r, fp2* __restrict__ Aout,
                                                         const fp2* __restrict__ beta,
                                                         fp2* __restrict__ beta_out)
{
    const long long item = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (item >= (long long)(W_rows + 1) * n_out) return;
    const int oc = (int)(item % n_out), w = (int)(item / n_out);
    if (w == W_rows) {
        st2(beta_out + oc, l2fold(ld2c(beta + 2 * (size_t)oc), ld2c(beta + 2 * (size_t)oc + 1), r));
        return;
    }
    auto val = [&](int c) -> u64 {
        if (c >= px.n_real) return 0;
        if (w < px.cs) return px.pix[(size_t)c * px.cs + w];
        return w == px.const_idx ? px.const_val : 0;
    };
    st2(Aout + (size_t)w * n_out + oc, l2fold(mk(val(2 * oc), 0), mk(val(2 * oc + 1), 0), r));
}

// fin[w] = V[w][0] straight from the bytes (a finish before any fold)
__global__ void gather_pixels_kernel(const PixSrc px, int W, const fp2* __restrict__ beta,
                                     fp2* __restrict__ fin, fp2* __restrict__ fin_beta)
{
    const int w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w < W) {
        u64 v = 0;
        if (px.n_real > 0) v = w < px.cs ? px.pix[w] : (w == px.const_idx ? px.const_val : 0);
        st2(fin + w, mk(v, 0));
    }
    if (w == W) st2(fin_beta, l2canon(ld2c(beta)));
}

// ---------------------------------------------------------------------------
// MLE of the copy-major input vector x[c * W + w] at z, from the bytes:
//   sum_c hi[c] * (sum_{w < cs} byte(c, w) * lo[w] + const_val * lo[const_idx])
// one warp per copy, lanes read the copy's bytes as consecutive words.
__global__ void __launch_bounds__(kT)
    mle_pixels_kernel(const PixSrc px, const fp2* __restrict__ lo, const fp2* __restrict__ hi,
                      fp2* partials, unsigned* ticket, u64* out)
{
    __shared__ uint4 los[512];
    const int cs = px.cs;
    fp2 const_term = f2zero();
    if (px.const_idx >= 0) {
        const fp2 l = ld2c(lo + px.const_idx);
        const_term = mk(lmul(l.re, px.const_val), lmul(l.im, px.const_val));
    }
    for (int w = threadIdx.x; w < cs && w < 512; w += blockDim.x) los[w] = split4(l2canon(ld2c(lo + w)));
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int n_warps = (gridDim.x * blockDim.x) >> 5;
    fp2 acc[1] = {f2zero()};
    for (int c = warp; c < px.n_real; c += n_warps) {
        u64 A0 = 0, A1 = 0, A2 = 0, A3 = 0;
        const unsigned char* row = px.pix + (size_t)c * cs;
        for (int w = lane; w < cs; w += 32) {
            const u32 x = __ldg(row + w);
            const uint4 l = los[w];
            A0 += (u64)l.x * x;
            A1 += (u64)l.y * x;
            A2 += (u64)l.z * x;
            A3 += (u64)l.w * x;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            A0 += __shfl_xor_sync(0xffffffffu, A0, o);
            A1 += __shfl_xor_sync(0xffffffffu, A1, o);
            A2 += __shfl_xor_sync(0xffffffffu, A2, o);
            A3 += __shfl_xor_sync(0xffffffffu, A3, o);
        }
        if (lane == 0) {
            const fp2 v = l2add(mk(combine(A0, A1), combine(A2, A3)), const_term);
            acc[0] = l2add(acc[0], l2mul(v, ld2c(hi + c)));
        }
    }
    acc[0] = l2canon(acc[0]);
    grid_reduce<1>(acc, partials, ticket, out);
}

int pad_words(int cs)
{
    const int w = (cs + 3) / 4;
    return (w & 1) ? w : w + 1;  // odd word stride: conflict-free column access
}

size_t claim_smem(int cs) { return 16 * (size_t)cs + 4 * (size_t)kClaimCopies * pad_words(cs); }
size_t fold_smem(int cs)
{
    return 32 * (size_t)cs + 16 * 511 + 4 * (size_t)(2 * kFoldCopies) * pad_words(cs);
}

bool smem_attr_done = false;
bool ensure_smem_attrs()
{
    if (smem_attr_done) return true;
    const int big = 200 * 1024;
    TP_CUDA_OK(cudaFuncSetAttribute(claim_pixels_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, big),
               "smem attr");
    TP_CUDA_OK(cudaFuncSetAttribute(fold_claim_pixels_kernel,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, big), "smem attr");
    smem_attr_done = true;
    return true;
}

}  // namespace

bool pixsrc_valid(const PixSrc& px, int n_pad, int W)
{
    if (!px.pix || px.n_real < 0 || px.n_real > n_pad || px.cs <= 0 || px.cs > W || W > 4096 ||
        px.const_idx >= W || (px.const_idx >= 0 && px.const_idx < px.cs) || px.const_val >= P61) {
        set_error(TP_ERR_ARG, "pixel layout: copies %d/%d, copy_size %d, wires %d, const %d",
                  px.n_real, n_pad, px.cs, W, px.const_idx);
        return false;
    }
    return true;
}

int pixsrc_rows(const PixSrc& px)
{
    return px.const_idx >= 0 ? px.const_idx + 1 : px.cs;
}

bool launch_claim_pixels(PixClaimArgs a, bool fold, cudaStream_t s, int* launches)
{
    if (!ensure_smem_attrs()) return false;
    a.pw = pad_words(a.px.cs);
    if (!fold) {
        const unsigned blocks = blocks_for((size_t)a.n_pad, kClaimCopies);
        a.tc = a.n_terms ? (a.n_terms + 3) / 4 : 0;
        claim_pixels_kernel<<<blocks, kT, claim_smem(a.px.cs), s>>>(a);
    } else {
        const unsigned blocks = blocks_for((size_t)a.n_out, kFoldCopies);
        a.tc = a.n_terms ? (a.n_terms + 7) / 8 : 0;
        fold_claim_pixels_kernel<<<blocks, kT, fold_smem(a.px.cs), s>>>(a);
    }
    ++*launches;
    return !cuda_failed(cudaGetLastError(), "pixel claim launch");
}

unsigned claim_pixels_blocks(int n_pad, int n_out, bool fold)
{
    return fold ? blocks_for((size_t)n_out, kFoldCopies) : blocks_for((size_t)n_pad, kClaimCopies);
}

bool launch_fold_pixels(const PixSrc& px, int W_rows, int n_out, fp2 r, fp2* Aout,
                        const fp2* beta, fp2* beta_out, cudaStream_t s, int* launches)
{
    const size_t items = (size_t)(W_rows + 1) * n_out;
    fold_pixels_kernel<<<blocks_for(items, kT), kT, 0, s>>>(px, W_rows, n_out, r, Aout, beta,
                                                           beta_out);
    ++*launches;
    return !cuda_failed(cudaGetLastError(), "pixel fold launch");
}

bool launch_gather_pixels(const PixSrc& px, int W, const fp2* beta, fp2* fin, fp2* fin_beta,
                          cudaStream_t s, int* launches)
{
    gather_pixels_kernel<<<blocks_for((size_t)W + 1, kT), kT, 0, s>>>(px, W, beta, fin, fin_beta);
    ++*launches;
    return !cuda_failed(cudaGetLastError(), "pixel gather launch");
}

bool launch_mle_pixels(const PixSrc& px, int n_pad, int W, const fp2* d_z, fp2* d_out,
                       cudaStream_t s, int* launches)
{
    Ctx* c = ctx();
    if (!c) return false;
    if (!pixsrc_valid(px, n_pad, W)) return false;
    if ((W & (W - 1)) || (n_pad & (n_pad - 1)) || W > 512) {
        set_error(TP_ERR_ARG, "mle over pixels needs power-of-two wires (<= 512) and copies");
        return false;
    }
    int h = 0, hb = 0;
    while ((1 << h) < W) ++h;
    while ((1 << hb) < n_pad) ++hb;
    const size_t nt = ((size_t)1 << h) + ((size_t)1 << hb);
    fp2* tabs = (fp2*)dev_alloc(sizeof(fp2) * (nt + 2048) + 256, s);
    if (!tabs) return false;
    fp2* lo = tabs;
    fp2* hi = tabs + ((size_t)1 << h);
    fp2* partials = tabs + nt;
    unsigned* ticket = reinterpret_cast<unsigned*>(partials + 2048);
    bool ok = !cuda_failed(cudaMemsetAsync(ticket, 0, sizeof(unsigned), s), "mle ticket");
    launch_eq_tables(d_z, h, hb, mk(1, 0), lo, hi, s);
    ++*launches;
    const unsigned blocks = (unsigned)std::max<size_t>(
        1, std::min<size_t>(std::min<size_t>((size_t)c->n_sm * 4, 2048),
                            blocks_for((size_t)std::max(1, px.n_real), kT / 32)));
    mle_pixels_kernel<<<blocks, kT, 0, s>>>(px, lo, hi, partials, ticket,
                                            reinterpret_cast<u64*>(d_out));
    ++*launches;
    ok = ok && !cuda_failed(cudaGetLastError(), "mle pixels launch");
    dev_free(tabs, s);
    return ok;
}

}  // namespace tp
