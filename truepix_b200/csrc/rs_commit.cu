// Reed-Solomon commit: batched slice transforms, FRI leaf chains, Merkle tree.
#include "fp2.cuh"
#include "ntt.h"
#include "orion.h"
#include "runtime.h"
#include "sha256.cuh"

namespace tp {
namespace rs {

namespace {

constexpr int kSlices = 64;   // 2^log_slice_number (include/infrastructure/constants.h)

// leaf j: h <- SHA256(x || y || h) over the 64 slices (fri.cpp:96-110: the pair
// first, the running digest second -- the opposite order of the Orion row leaves)
__global__ void __launch_bounds__(256) fri_leaf_kernel(const ulonglong2* __restrict__ l_eval, long long slice,
                                                       unsigned char* __restrict__ tree, uint32_t one)
{
    const long long half = slice >> 1;
    const long long j = (long long)blockIdx.x * 256 + threadIdx.x;
    if (j >= half) return;
    uint32_t st[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) st[i] = 0;
#pragma unroll 1
    for (int i = 0; i < kSlices; ++i) {
        const ulonglong2 x = __ldg(l_eval + i * slice + j);
        const ulonglong2 y = __ldg(l_eval + i * slice + j + half);
        uint32_t w[16];
        sha::fe_words(x.x, x.y, w);
        sha::fe_words(y.x, y.y, w + 4);
#pragma unroll
        for (int k = 0; k < 8; ++k) w[8 + k] = st[k];
        sha::hash64(w, st, sha::AddMad{one});
    }
    uint4 a, b;
    a.x = sha::bswap32(st[0]); a.y = sha::bswap32(st[1]); a.z = sha::bswap32(st[2]); a.w = sha::bswap32(st[3]);
    b.x = sha::bswap32(st[4]); b.y = sha::bswap32(st[5]); b.z = sha::bswap32(st[6]); b.w = sha::bswap32(st[7]);
    uint4* p = reinterpret_cast<uint4*>(tree + (half + j) * 32);
    p[0] = a;
    p[1] = b;
}

__device__ __forceinline__ fp2 ld_fe(const ulonglong2* p) { const ulonglong2 v = __ldg(p); return mk(v.y, v.x); }

// v[i][j] = 2^-1 ((x + y) + w_M^-i r (x - y)) into the next interleaved witness;
// one thread per (i, j), j fastest: the 64 pairs of a row are 2 KB contiguous.
__global__ void __launch_bounds__(256) fri_fold_kernel(const ulonglong2* __restrict__ w, long long nxt, fp2 r,
                                                       const fp2* __restrict__ lo, const fp2* __restrict__ hi,
                                                       int h, ulonglong2* __restrict__ next)
{
    const long long t = (long long)blockIdx.x * 256 + threadIdx.x;
    if (t >= nxt * kSlices) return;
    const long long i = t >> 6;
    const int j = (int)(t & 63);
    const fp2 x = ld_fe(w + ((i << 7) | (j << 1))), y = ld_fe(w + ((i << 7) | (j << 1) | 1));
    fp2 inv_mu = lo[i & ((1ll << h) - 1)];
    if (i >> h) inv_mu = l2mul(inv_mu, hi[i >> h]);
    const fp2 d = l2sub(x, y);
    const fp2 v = l2mul(mk(1ull << 60, 0), l2add(l2add(x, y), l2mul(l2mul(inv_mu, r), d)));
    const fp2 c = l2canon(v);
    const long long half = nxt >> 1;
    const long long pos = i < half ? ((i << 7) | (j << 1)) : (((i - half) << 7) | (j << 1) | 1);
    next[pos] = make_ulonglong2(c.im, c.re);
}

// leaf i = chain over the 64 pairs of row i of the interleaved witness:
// h <- SHA256(x || y || h) (fri.cpp:396-410)
__global__ void __launch_bounds__(256) fri_row_leaf_kernel(const ulonglong2* __restrict__ w, long long n_leaves,
                                                           unsigned char* __restrict__ tree, uint32_t one)
{
    const long long i = (long long)blockIdx.x * 256 + threadIdx.x;
    if (i >= n_leaves) return;
    uint32_t st[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) st[k] = 0;
    const ulonglong2* row = w + (i << 7);
#pragma unroll 1
    for (int j = 0; j < kSlices; ++j) {
        const ulonglong2 x = __ldg(row + 2 * j), y = __ldg(row + 2 * j + 1);
        uint32_t m[16];
        sha::fe_words(x.x, x.y, m);
        sha::fe_words(y.x, y.y, m + 4);
#pragma unroll
        for (int k = 0; k < 8; ++k) m[8 + k] = st[k];
        sha::hash64(m, st, sha::AddMad{one});
    }
    uint4 a, b;
    a.x = sha::bswap32(st[0]); a.y = sha::bswap32(st[1]); a.z = sha::bswap32(st[2]); a.w = sha::bswap32(st[3]);
    b.x = sha::bswap32(st[4]); b.y = sha::bswap32(st[5]); b.z = sha::bswap32(st[6]); b.w = sha::bswap32(st[7]);
    uint4* p = reinterpret_cast<uint4*>(tree + (n_leaves + i) * 32);
    p[0] = a;
    p[1] = b;
}

}  // namespace

bool fri_step(const ulonglong2* w, int log_m, fp2 r, ulonglong2* next, unsigned char* tree, cudaStream_t s)
{
    if (log_m < 2 || log_m > 26) {
        set_error(TP_ERR_ARG, "fri step: log2 of the per-slice witness size %d outside [2, 26]", log_m);
        return false;
    }
    if (r.re >= P61 || r.im >= P61) {
        set_error(TP_ERR_ARG, "fri step: the random is not canonical");
        return false;
    }
    const fp2 *lo, *hi;
    int h;
    if (!ntt::power_tables(log_m, true, &lo, &hi, &h)) return false;
    const long long nxt = 1LL << (log_m - 1), n_leaves = nxt / 2;
    timer_begin(s, 9210);
    fri_fold_kernel<<<(unsigned)((nxt * kSlices + 255) / 256), 256, 0, s>>>(w, nxt, r, lo, hi, h, next);
    timer_end(s);
    if (cuda_failed(cudaGetLastError(), "fri fold")) return false;
    if (cuda_failed(cudaMemsetAsync(tree, 0, 32, s), "fri tree clear")) return false;
    timer_begin(s, 9211);
    fri_row_leaf_kernel<<<(unsigned)((n_leaves + 255) / 256), 256, 0, s>>>(next, n_leaves, tree, 1u);
    timer_end(s);
    if (cuda_failed(cudaGetLastError(), "fri leaves")) return false;
    return orion::build_tree(tree, n_leaves, s);
}

bool commit(const ulonglong2* src, int log_len, ulonglong2* l_eval, unsigned char* tree, cudaStream_t s)
{
    if (log_len < kMinLog || log_len > kMaxLog) {
        set_error(TP_ERR_ARG, "rs commit: log_len %d outside [%d, %d]", log_len, kMinLog, kMaxLog);
        return false;
    }
    const long long real_cnt = 1LL << (log_len - 6), slice = 1LL << (log_len - 1);
    // the 64 slices' coefficients (2^log_len elements)
    ulonglong2* coef = static_cast<ulonglong2*>(dev_alloc(sizeof(ulonglong2) * (size_t)(real_cnt * kSlices), s));
    if (!coef) return false;
    bool ok = ntt::inverse(src, real_cnt, real_cnt, coef, kSlices, real_cnt, real_cnt, nullptr, s) &&
              ntt::forward(coef, real_cnt, slice, l_eval, kSlices, real_cnt, slice, nullptr, s);
    dev_free(coef, s);
    if (!ok) return false;
    if (cuda_failed(cudaMemsetAsync(tree, 0, 32, s), "rs tree clear")) return false;
    const long long half = slice >> 1;
    fri_leaf_kernel<<<(unsigned)((half + 255) / 256), 256, 0, s>>>(l_eval, slice, tree, 1u);
    if (cuda_failed(cudaGetLastError(), "rs leaves")) return false;
    return orion::build_tree(tree, half, s);
}

}  // namespace rs
}  // namespace tp
