// Reed-Solomon commit: batched slice transforms, FRI leaf chains, Merkle tree.
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

}  // namespace

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
