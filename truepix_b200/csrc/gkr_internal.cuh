// Device helpers shared by the GKR kernel files (16-byte Fp2 loads/stores,
// warp and grid reductions) and the argument blocks of the pixel kernels.
#pragma once
#include <cuda_runtime.h>

#include "fp2.cuh"

namespace tp {

constexpr int kRedThreads = 256;  // block size assumed by grid_reduce's shared buffer

__device__ __forceinline__ fp2 ld2(const fp2* p)
{
    const ulonglong2 v = __ldg(reinterpret_cast<const ulonglong2*>(p));
    return mk(v.x, v.y);
}
// same, for buffers written earlier in the stream (read-only during the kernel)
__device__ __forceinline__ fp2 ld2c(const fp2* p) { return ld2(p); }
__device__ __forceinline__ fp2 ldcg2(const fp2* p)
{
    const ulonglong2 v = __ldcg(reinterpret_cast<const ulonglong2*>(p));
    return mk(v.x, v.y);
}
__device__ __forceinline__ void st2(fp2* p, fp2 v)
{
    *reinterpret_cast<ulonglong2*>(p) = make_ulonglong2(v.re, v.im);
}
__device__ __forceinline__ void stcg2(fp2* p, fp2 v)
{
    __stcg(reinterpret_cast<ulonglong2*>(p), make_ulonglong2(v.re, v.im));
}

__device__ __forceinline__ fp2 warp_sum(fp2 v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const u64 r = __shfl_xor_sync(0xffffffffu, v.re, o);
        const u64 i = __shfl_xor_sync(0xffffffffu, v.im, o);
        v = f2add(v, mk(r, i));
    }
    return v;
}

// Sum NV canonical Fp2 values over the whole grid (blockDim.x <= kRedThreads).
// Every thread of every block must call it. Per-block partials go to
// `partials`; the last block to arrive (ticket) adds them, writes out[2*NV]
// and re-arms the ticket for the next launch on the stream.
template <int NV>
__device__ void grid_reduce(fp2 (&acc)[NV], fp2* partials, unsigned* ticket, u64* out)
{
    __shared__ fp2 sm[kRedThreads / 32][NV];
    __shared__ bool s_last;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int t = 0; t < NV; ++t) acc[t] = warp_sum(acc[t]);
    if (lane == 0)
#pragma unroll
        for (int t = 0; t < NV; ++t) sm[warp][t] = acc[t];
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int t = 0; t < NV; ++t) {
            fp2 v = lane < nw ? sm[lane][t] : f2zero();
            v = warp_sum(v);
            if (lane == 0) stcg2(partials + (size_t)blockIdx.x * NV + t, v);
        }
    }
    if (threadIdx.x == 0) {
        __threadfence();
        const unsigned prev = atomicAdd(ticket, 1u);
        s_last = (prev == gridDim.x - 1);
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    fp2 tot[NV];
#pragma unroll
    for (int t = 0; t < NV; ++t) tot[t] = f2zero();
    for (unsigned i = threadIdx.x; i < gridDim.x; i += blockDim.x)
#pragma unroll
        for (int t = 0; t < NV; ++t) tot[t] = f2add(tot[t], ldcg2(partials + (size_t)i * NV + t));
#pragma unroll
    for (int t = 0; t < NV; ++t) tot[t] = warp_sum(tot[t]);
    __syncthreads();
    if (lane == 0)
#pragma unroll
        for (int t = 0; t < NV; ++t) sm[warp][t] = tot[t];
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int t = 0; t < NV; ++t) {
            fp2 v = lane < nw ? sm[lane][t] : f2zero();
            v = warp_sum(v);
            if (lane == 0) {
                out[2 * t] = v.re;
                out[2 * t + 1] = v.im;
            }
        }
    }
    if (threadIdx.x == 0) *ticket = 0u;
}

// The implicit input-layer table of a uint8 frame: V[w][c] = pix[c * cs + w] for
// w < cs, const_val at w = const_idx, zero elsewhere and for c >= n_real.
struct PixSrc {
    const unsigned char* pix;
    int n_real;
    int cs;
    int const_idx;
    u64 const_val;
};

struct PixClaimArgs {
    PixSrc px;
    int pw;          // padded 32-bit words per staged copy
    int W_rows;      // rows kept in the folded table (private wires + constant)
    int n_pad;       // copies of the implicit table
    int n_out;       // folded copies (fold kernel)
    const fp2* L;    // canonical linear coefficients [n_wires]
    fp2 K0;
    fp2 Lc;          // L[const_idx] * const_val
    const int2* ab;  // product terms, grouped by b
    const fp2* cf;
    int n_terms, tc;
    const fp2* beta;
    fp2* beta_out;
    fp2* Aout;       // folded rows, stride n_out
    fp2 r;
    fp2* partials;
    unsigned* ticket;
    u64* out8;
};

// host-side launchers implemented in gkr_pixels.cu / gkr.cu
bool pixsrc_valid(const PixSrc& px, int n_pad, int W);
int pixsrc_rows(const PixSrc& px);
bool launch_claim_pixels(PixClaimArgs a, bool fold, cudaStream_t s, int* launches);
bool launch_fold_pixels(const PixSrc& px, int W_rows, int n_out, fp2 r, fp2* Aout,
                        const fp2* beta, fp2* beta_out, cudaStream_t s, int* launches);
bool launch_gather_pixels(const PixSrc& px, int W, const fp2* beta, fp2* fin, fp2* fin_beta,
                          cudaStream_t s, int* launches);
bool launch_mle_pixels(const PixSrc& px, int n_pad, int W, const fp2* d_z, fp2* d_out,
                       cudaStream_t s, int* launches);
void launch_eq_tables(const fp2* d_z, int h, int hb, fp2 init, fp2* lo, fp2* hi, cudaStream_t s);

}  // namespace tp
