// Prover-side passes of the Orion tensor-product opening over the row-major
// codeword that commit() leaves in HBM
// (TruePix-main/Orion/Orion_nonzk/src/VPD/linearPC.cpp:480-531, 569-571):
//   combined[t] = sum_j r0[j] * codeword[t][j]        (t < cw_len; the first N/128
//                 entries are combined_message)
//   leaves      = SHA256(combined[i] || 0^48), i < 2 N/128, zero element past
//                 cw_len (merkle_tree.cpp:5-13); tree as in the commit
//   queried     = queried_cols[i][j] = codeword[q_i][j]
//   answer      = sum_{i < N/128} r1[i] * combined[i]
#include <algorithm>

#include "fp2.cuh"
#include "orion.h"
#include "runtime.h"
#include "sha256.cuh"

namespace tp {
namespace orion {

namespace {

constexpr int kTagCombine = 9110, kTagCombineLeaves = 9111;

__device__ __forceinline__ fp2 ld_fe(const ulonglong2* p) { const ulonglong2 v = __ldg(p); return mk(v.y, v.x); }

__device__ __forceinline__ fp2 warp_sum2(fp2 a)
{
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        fp2 b;
        b.re = __shfl_xor_sync(0xffffffffu, a.re, o);
        b.im = __shfl_xor_sync(0xffffffffu, a.im, o);
        a = l2add(a, b);
    }
    return a;
}

// One warp per codeword row (grid-stride): lane l holds r0[l + 32k], k < 4, and
// multiplies the row's four 512-byte column slices by them.
__global__ void __launch_bounds__(256) combine_kernel(const ulonglong2* __restrict__ rows, long long cw_len,
                                                      const ulonglong2* __restrict__ r0,
                                                      ulonglong2* __restrict__ combined)
{
    const int lane = threadIdx.x & 31;
    fp2 r[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) r[k] = ld_fe(r0 + lane + 32 * k);
    const long long warps = (long long)gridDim.x * 8;
    for (long long t = (long long)blockIdx.x * 8 + (threadIdx.x >> 5); t < cw_len; t += warps) {
        const ulonglong2* row = rows + t * kColumns + lane;
        fp2 x[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) x[k] = ld_fe(row + 32 * k);
        fp2 acc = l2add(l2add(l2mul(r[0], x[0]), l2mul(r[1], x[1])), l2add(l2mul(r[2], x[2]), l2mul(r[3], x[3])));
        acc = warp_sum2(acc);
        if (lane == 0) combined[t] = make_ulonglong2(canon61(acc.im), canon61(acc.re));
    }
}

// leaves [0, size): SHA256(element || 0^48) of combined[i] for i < cw_len, of the
// zero element (= SHA256(0^64)) beyond
__global__ void __launch_bounds__(256) single_leaf_kernel(const ulonglong2* __restrict__ combined,
                                                          long long cw_len, long long size,
                                                          unsigned char* __restrict__ tree, uint32_t one)
{
    const long long i = (long long)blockIdx.x * 256 + threadIdx.x;
    if (i >= size) return;
    uint32_t w[16], st[8];
    const ulonglong2 x = i < cw_len ? __ldg(combined + i) : make_ulonglong2(0, 0);
    sha::fe_words(x.x, x.y, w);
#pragma unroll
    for (int k = 4; k < 16; ++k) w[k] = 0;
    sha::hash64(w, st, sha::AddMad{one});
    uint4 a, b;
    a.x = sha::bswap32(st[0]); a.y = sha::bswap32(st[1]); a.z = sha::bswap32(st[2]); a.w = sha::bswap32(st[3]);
    b.x = sha::bswap32(st[4]); b.y = sha::bswap32(st[5]); b.z = sha::bswap32(st[6]); b.w = sha::bswap32(st[7]);
    uint4* p = reinterpret_cast<uint4*>(tree + (size + i) * 32);
    p[0] = a;
    p[1] = b;
}

// out[i] = rows[q[i]] (2 KB each); one CTA of 128 threads per query
__global__ void __launch_bounds__(128) query_kernel(const ulonglong2* __restrict__ rows, long long cw_len,
                                                    const long long* __restrict__ q, int count,
                                                    ulonglong2* __restrict__ out, int* __restrict__ bad)
{
    const int i = blockIdx.x;
    if (i >= count) return;
    const long long r = q[i];
    if (r < 0 || r >= cw_len) {
        if (threadIdx.x == 0) atomicExch(bad, 1);
        return;
    }
    out[(long long)i * kColumns + threadIdx.x] = __ldg(rows + r * kColumns + threadIdx.x);
}

// the same without a host round trip: a row index outside [0, cw_len) gives a
// zero row and raises *bad (when given), which the caller reads later
__global__ void __launch_bounds__(128) query_async_kernel(const ulonglong2* __restrict__ rows, long long cw_len,
                                                          const long long* __restrict__ q, int count,
                                                          ulonglong2* __restrict__ out, int* __restrict__ bad)
{
    const int i = blockIdx.x;
    if (i >= count) return;
    const long long r = q[i];
    const bool in = r >= 0 && r < cw_len;
    if (!in && bad && threadIdx.x == 0) atomicExch(bad, 1);
    out[(long long)i * kColumns + threadIdx.x] = in ? __ldg(rows + r * kColumns + threadIdx.x) : make_ulonglong2(0, 0);
}

// answer = sum_i r1[i] * combined[i], i < n: one CTA per 4096 entries, partial
// sums to `part`, the last CTA (ticket) adds them up
__global__ void __launch_bounds__(256) answer_kernel(const ulonglong2* __restrict__ combined,
                                                     const ulonglong2* __restrict__ r1, long long n,
                                                     fp2* __restrict__ part, unsigned* __restrict__ ticket,
                                                     ulonglong2* __restrict__ answer)
{
    __shared__ fp2 sw[8];
    __shared__ bool last;
    fp2 acc = f2zero();
    const long long base = (long long)blockIdx.x * 4096;
    for (long long i = base + threadIdx.x; i < base + 4096 && i < n; i += 256)
        acc = l2add(acc, l2mul(ld_fe(r1 + i), ld_fe(combined + i)));
    acc = warp_sum2(acc);
    if ((threadIdx.x & 31) == 0) sw[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        fp2 s = f2zero();
        for (int k = 0; k < 8; ++k) s = l2add(s, sw[k]);
        part[blockIdx.x] = s;
        __threadfence();
        last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (last && threadIdx.x == 0) {
        __threadfence();
        fp2 s = f2zero();
        const volatile u64* pv = reinterpret_cast<const volatile u64*>(part);
        for (unsigned b = 0; b < gridDim.x; ++b) s = l2add(s, mk(pv[2 * b], pv[2 * b + 1]));
        *answer = make_ulonglong2(canon61(s.im), canon61(s.re));
        *ticket = 0;
    }
}

bool ok(const char* what) { return !cuda_failed(cudaGetLastError(), what); }

}  // namespace

bool combine(const ulonglong2* rows, long long col_len, long long cw_len, const ulonglong2* r0,
             ulonglong2* combined, unsigned char* tree, cudaStream_t s)
{
    const long long size = tree_leaves(col_len);
    Ctx* c = ctx();
    if (!c) return false;
    const unsigned blocks = (unsigned)std::min<long long>((cw_len + 7) / 8, (long long)c->n_sm * 8);
    timer_begin(s, kTagCombine);
    combine_kernel<<<blocks, 256, 0, s>>>(rows, cw_len, r0, combined);
    timer_end(s);
    if (!ok("orion combine")) return false;
    if (!tree) return true;
    if (cuda_failed(cudaMemsetAsync(tree, 0, 32, s), "orion combined tree clear")) return false;
    timer_begin(s, kTagCombineLeaves);
    single_leaf_kernel<<<(unsigned)((size + 255) / 256), 256, 0, s>>>(combined, cw_len, size, tree, 1u);
    timer_end(s);
    if (!ok("orion combined leaves")) return false;
    return build_tree(tree, size, s);
}

bool query_rows(const ulonglong2* rows, long long cw_len, const long long* q, int count, ulonglong2* out,
                cudaStream_t s)
{
    int* bad = static_cast<int*>(dev_alloc(sizeof(int), s));
    if (!bad) return false;
    int h_bad = 0;
    bool good = !cuda_failed(cudaMemsetAsync(bad, 0, sizeof(int), s), "orion query flag");
    if (good) {
        query_kernel<<<count, 128, 0, s>>>(rows, cw_len, q, count, out, bad);
        good = ok("orion query") &&
               !cuda_failed(cudaMemcpyAsync(&h_bad, bad, sizeof(int), cudaMemcpyDeviceToHost, s), "D2H") &&
               !cuda_failed(cudaStreamSynchronize(s), "synchronize");
    }
    dev_free(bad, s);
    if (good && h_bad) {
        set_error(TP_ERR_ARG, "orion query: a row index is outside [0, %lld)", cw_len);
        return false;
    }
    return good;
}

bool query_rows_async(const ulonglong2* rows, long long cw_len, const long long* q, int count, ulonglong2* out,
                      int* bad, cudaStream_t s)
{
    query_async_kernel<<<count, 128, 0, s>>>(rows, cw_len, q, count, out, bad);
    return ok("orion query");
}

bool answer(const ulonglong2* combined, const ulonglong2* r1, long long n, ulonglong2* out, cudaStream_t s)
{
    const long long blocks = (n + 4095) / 4096;
    fp2* part = static_cast<fp2*>(dev_alloc(sizeof(fp2) * (size_t)blocks + 256, s));
    if (!part) return false;
    unsigned* ticket = reinterpret_cast<unsigned*>(part + blocks);
    bool good = !cuda_failed(cudaMemsetAsync(ticket, 0, sizeof(unsigned), s), "orion answer ticket");
    if (good) {
        answer_kernel<<<(unsigned)blocks, 256, 0, s>>>(combined, r1, n, part, ticket, out);
        good = ok("orion answer");
    }
    dev_free(part, s);
    return good;
}

}  // namespace orion
}  // namespace tp
