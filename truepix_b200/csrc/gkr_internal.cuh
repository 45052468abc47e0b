// Device helpers shared by the GKR kernel files (16-byte Fp2 loads/stores,
// warp and grid reductions) and the argument blocks of the pixel kernels.
#pragma once
#include <cuda_runtime.h>

#include <vector>

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


// One frame's work in a batched round launch (device memory). Table source
// when A != nullptr, frame bytes when pix != nullptr.
struct Job {
    const fp2* A;           // table [W_rows][n_in]
    fp2* Aout;              // folded table [W_rows][n_in / 2]
    const unsigned char* pix;
    const fp2* beta;
    fp2* beta_out;
    const fp2* L;           // canonical linear coefficients [W]
    const int2* ab;         // product terms grouped by b
    const fp2* cf;
    fp2* partials;          // [tiles * groups][4]
    unsigned* ticket;
    u64* out8;
    fp2* fin;               // finish: wires [W]
    fp2* fin_beta;          // finish: beta [1]
    fp2 K0, Lc, r;
    u64 const_val;
    int kind;               // 0 table claim, 1 table fold+claim, 2 bytes claim, 3 bytes fold+claim
    int n_in;               // copies of the source
    int n_pairs;            // claim pairs
    int W, W_rows;
    int n_real, cs, const_idx;
    int n_terms, tiles, groups, wpg, tpg, pw, cta0;
    int vec;                // byte rows are whole 16-byte vectors (copy_size % 16 == 0, aligned)
};

void plan_job(Job& j, int target_ctas);
bool launch_round(const Job* d_jobs, const std::vector<Job>& jobs, int kind, cudaStream_t s,
                  int* launches);
bool launch_finish(const Job* d_jobs, int n_jobs, int max_w, cudaStream_t s, int* launches);
// the round kernels' attributes, set once (before a stream capture)
bool prepare_round_kernels();
// one VOLE-committed round of n frames on device transcripts (transcript.cu,
// tp_vole_round_dev's kernel): label at most 32 bytes. d_rounds (device, n
// ints, optional): frame i takes part only while round k < d_rounds[i]
bool launch_vole_round_batch(void* d_states, void* d_vole_states, int n, const void* d_claims, const void* d_u,
                             const void* d_v, long long count, const char* label, void* d_chal, void* d_proof,
                             cudaStream_t s, const int* d_rounds = nullptr, int k = 0);

// host-side launchers implemented in gkr_pixels.cu / gkr.cu
bool pixsrc_valid(const PixSrc& px, int n_pad, int W);
int pixsrc_rows(const PixSrc& px);
bool launch_fold_pixels(const PixSrc& px, int W_rows, int n_out, fp2 r, fp2* Aout,
                        const fp2* beta, fp2* beta_out, cudaStream_t s, int* launches);
bool launch_pack(const u64* re, const u64* im, size_t n, fp2* out, cudaStream_t s, int* launches);
bool launch_fold_rows(const fp2* A, int n_in, fp2* Aout, int W_rows, const fp2* beta,
                      fp2* beta_out, fp2 r, cudaStream_t s, int* launches);
bool launch_mle_pixels(const PixSrc& px, int n_pad, int W, const fp2* d_z, fp2* d_out,
                       cudaStream_t s, int* launches);
void launch_eq_tables(const fp2* d_z, int h, int hb, fp2 init, fp2* lo, fp2* hi, cudaStream_t s);
void launch_eq_tables_batch(const fp2* d_z, int z_stride, int h, int hb, fp2 init, fp2* tabs,
                            int n, cudaStream_t s);
// beta tables of n frames: d_z packed [n][n_z], d_out packed [n][2^n_z]
bool launch_beta_batch(const fp2* d_z, int n_z, int n, fp2* d_out, cudaStream_t s, int* launches);
// MLE of n frames' input vectors (same padded size) from their bytes:
// frames[i] = {pix, n_real}; points packed [n][log2 W + log2 n_pad]; out packed [n]
struct MleFrame {
    const unsigned char* pix;
    int n_real;
    int pad_;
};
bool launch_mle_pixels_batch(const MleFrame* h_frames, int n, int n_pad, int cs, int W,
                             int const_idx, u64 const_val, const fp2* d_points, fp2* d_out,
                             cudaStream_t s, int* launches);

}  // namespace tp
