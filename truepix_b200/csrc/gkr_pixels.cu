// Kernels over a frame's uint8 bytes outside the batched rounds: the fold
// without a claim (two folds in a row, or 2 -> 1 copies) and the MLE of the
// input vector.
//
// In TruePix's input layout (TruePix-main/Orion/Orion_nonzk/include/truepix/
// truepix_gkr.h:11-18) the input-layer table is V[w][c] = byte c*copy_size + w
// for w < copy_size, the circuit constant at w = const_idx, zero on the other
// wires and on padded copies. With byte values x < 2^8 and a canonical
// coefficient split as L = Lh*2^32 + Ll (Lh < 2^29), sum_w L[w]*x_w is
// accumulated exactly as two 64-bit sums of 32x32->64 products (IMAD.WIDE with
// accumulate) and reduced once per copy; the batched round kernels
// (gkr_batch.cu) use the same identity for the first claim and first fold.
#include "gkr.h"
#include "gkr_internal.cuh"
#include "runtime.h"

#include <algorithm>

namespace tp {

namespace {

constexpr int kT = 256;

__device__ __forceinline__ uint4 split4(fp2 v)
{
    return make_uint4((u32)v.re, (u32)(v.re >> 32), (u32)v.im, (u32)(v.im >> 32));
}

// (lo + hi * 2^32) mod p, lo < 2^63, hi < 2^45 (raw IMAD sums) -> nearly canonical
__device__ __forceinline__ u64 combine(u64 lo, u64 hi)
{
    return fold61(fold61(lo) + (hi >> 29) + ((hi & 0x1FFFFFFFull) << 32));
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

}  // namespace

// Batched MLE: frame blockIdx.y, one thread per copy (16-byte loads of its
// bytes), hi[c] applied per copy, per-frame last-block reduction.
__global__ void __launch_bounds__(kT)
    mle_pixels_batch_kernel(const MleFrame* __restrict__ frames, int cs, int h, int hb,
                            int const_idx, u64 const_val, const fp2* __restrict__ tabs,
                            fp2* __restrict__ partials, unsigned* __restrict__ tickets,
                            fp2* __restrict__ out)
{
    __shared__ uint4 los[512];
    __shared__ fp2 red[kT / 32];
    __shared__ bool s_last;
    const int f = blockIdx.y;
    const MleFrame fr = frames[f];
    const size_t nt = ((size_t)1 << h) + ((size_t)1 << hb);
    const fp2* lo = tabs + (size_t)f * nt;
    const fp2* hi = lo + ((size_t)1 << h);
    for (int w = threadIdx.x; w < cs; w += blockDim.x) los[w] = split4(l2canon(ld2c(lo + w)));
    fp2 const_term = f2zero();
    if (const_idx >= 0) {
        const fp2 l = ld2c(lo + const_idx);
        const_term = mk(lmul(l.re, const_val), lmul(l.im, const_val));
    }
    __syncthreads();
    fp2 acc = f2zero();
    const bool vec = (cs & 15) == 0 && ((reinterpret_cast<size_t>(fr.pix) & 15) == 0);
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < fr.n_real; c += gridDim.x * blockDim.x) {
        const unsigned char* row = fr.pix + (size_t)c * cs;
        u64 A0 = 0, A1 = 0, A2 = 0, A3 = 0;
        if (vec) {
            const uint4* r4 = reinterpret_cast<const uint4*>(row);
            for (int q = 0; q < (cs >> 4); ++q) {
                const uint4 v = __ldg(r4 + q);
                const u32 words[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
                for (int k = 0; k < 16; ++k) {
                    const u32 x = (words[k >> 2] >> (8 * (k & 3))) & 0xFFu;
                    const uint4 l = los[16 * q + k];
                    A0 += (u64)l.x * x;
                    A1 += (u64)l.y * x;
                    A2 += (u64)l.z * x;
                    A3 += (u64)l.w * x;
                }
            }
        } else {
            for (int w = 0; w < cs; ++w) {
                const u32 x = __ldg(row + w);
                const uint4 l = los[w];
                A0 += (u64)l.x * x;
                A1 += (u64)l.y * x;
                A2 += (u64)l.z * x;
                A3 += (u64)l.w * x;
            }
        }
        const fp2 v = l2add(mk(combine(A0, A1), combine(A2, A3)), const_term);
        acc = l2add(acc, l2mul(v, ld2c(hi + c)));
    }
    acc = warp_sum(l2canon(acc));
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) red[warp] = acc;
    __syncthreads();
    if (warp == 0) {
        fp2 v = lane < (int)(blockDim.x >> 5) ? red[lane] : f2zero();
        v = warp_sum(v);
        if (lane == 0) {
            stcg2(partials + (size_t)f * gridDim.x + blockIdx.x, v);
            __threadfence();
            s_last = atomicAdd(tickets + f, 1u) == gridDim.x - 1;
        }
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    fp2 t = f2zero();
    for (unsigned i = threadIdx.x; i < gridDim.x; i += blockDim.x)
        t = f2add(t, ldcg2(partials + (size_t)f * gridDim.x + i));
    t = warp_sum(t);
    __syncthreads();
    if (lane == 0) red[warp] = t;
    __syncthreads();
    if (warp == 0) {
        fp2 v = lane < (int)(blockDim.x >> 5) ? red[lane] : f2zero();
        v = warp_sum(v);
        if (lane == 0) {
            st2(out + f, v);
            tickets[f] = 0u;
        }
    }
}

bool launch_mle_pixels_batch(const MleFrame* h_frames, int n, int n_pad, int cs, int W,
                             int const_idx, u64 const_val, const fp2* d_points, fp2* d_out,
                             cudaStream_t s, int* launches)
{
    if (n <= 0) return true;
    if ((W & (W - 1)) || (n_pad & (n_pad - 1)) || W > 512 || cs <= 0 || cs > W ||
        const_idx >= W || (const_idx >= 0 && const_idx < cs) || const_val >= P61) {
        set_error(TP_ERR_ARG, "mle over bytes: bad layout (wires %d, copies %d, copy_size %d)", W,
                  n_pad, cs);
        return false;
    }
    for (int i = 0; i < n; ++i)
        if (!h_frames[i].pix || h_frames[i].n_real < 0 || h_frames[i].n_real > n_pad) {
            set_error(TP_ERR_ARG, "mle over bytes: frame %d has %d of %d copies", i,
                      h_frames[i].n_real, n_pad);
            return false;
        }
    int h = 0, hb = 0;
    while ((1 << h) < W) ++h;
    while ((1 << hb) < n_pad) ++hb;
    const size_t nt = ((size_t)1 << h) + ((size_t)1 << hb);
    const unsigned blocks = (unsigned)std::max(1, std::min(64, (n_pad + kT - 1) / kT));
    const size_t bytes = sizeof(fp2) * (nt * n + (size_t)blocks * n) + sizeof(MleFrame) * n +
                         sizeof(unsigned) * n + 512;
    unsigned char* ws = (unsigned char*)dev_alloc(bytes, s);
    if (!ws) return false;
    fp2* tabs = reinterpret_cast<fp2*>(ws);
    fp2* partials = tabs + nt * n;
    MleFrame* d_frames = reinterpret_cast<MleFrame*>(partials + (size_t)blocks * n);
    unsigned* tickets = reinterpret_cast<unsigned*>(d_frames + n);
    bool ok = !cuda_failed(cudaMemsetAsync(tickets, 0, sizeof(unsigned) * n, s), "mle tickets") &&
              upload_async(d_frames, h_frames, sizeof(MleFrame) * n, s);
    if (ok) {
        launch_eq_tables_batch(d_points, h + hb, h, hb, mk(1, 0), tabs, n, s);
        mle_pixels_batch_kernel<<<dim3(blocks, n), kT, 0, s>>>(d_frames, cs, h, hb, const_idx,
                                                               const_val, tabs, partials, tickets,
                                                               d_out);
        *launches += 2;
        ok = !cuda_failed(cudaGetLastError(), "mle batch launch");
    }
    dev_free(ws, s);
    return ok;
}

bool pixsrc_valid(const PixSrc& px, int n_pad, int W)
{
    if (!px.pix || px.n_real < 0 || px.n_real > n_pad || px.cs <= 0 || px.cs > W || px.cs > 512 ||
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

bool launch_fold_pixels(const PixSrc& px, int W_rows, int n_out, fp2 r, fp2* Aout,
                        const fp2* beta, fp2* beta_out, cudaStream_t s, int* launches)
{
    const size_t items = (size_t)(W_rows + 1) * n_out;
    fold_pixels_kernel<<<blocks_for(items, kT), kT, 0, s>>>(px, W_rows, n_out, r, Aout, beta,
                                                           beta_out);
    ++*launches;
    return !cuda_failed(cudaGetLastError(), "pixel fold launch");
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
