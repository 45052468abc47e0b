// Verifier side of the Orion NIZK opening on the device
// (TruePix-main/Orion/Orion_nonzk/src/VPD/linearPC.cpp:733-879 verify_opening_proof,
// src/truepix/orion_proof.cpp:176-200 verify_claim_sparse) and the code of one
// message (the EC(y1) step: Enc(combined_message) at the second batch of
// queried positions, linearPC.cpp:573-605).
//
// Per queried column i (one thread each, all queries at once):
//   column     sum_j r0[j] col_i[j] == combined_codeword[q_i]   (col_i: 128 elements)
//   commitment leaf = the column's SHA-256 chain (as the commit's row leaves),
//              walked up with the proof's sparse siblings to the commitment root
//   combined   leaf = SHA256(combined_codeword[q_i] || 0^48), walked up to the
//              combined root
//   EC(y1)     Enc(combined_message)[q2_i] == combined_codeword[q2_i]
// A sibling is looked up by binary search in the proof's node list, sorted by
// node index on the host (the reference keeps the first entry of an index).
#include <algorithm>

#include "fp2.cuh"
#include "orion.h"
#include "runtime.h"
#include "sha256.cuh"

namespace tp {
namespace orion {

namespace {

// out[dst + t] = sum_e w_e out[src + esrc_e] over the in-edges of target t: the
// gather of one column (the commit's gather_kernel runs 128 at once)
__global__ void __launch_bounds__(256) gather1_kernel(ulonglong2* __restrict__ v, long long src_row,
                                                      long long dst_row, long long n_targets,
                                                      const unsigned* __restrict__ ptr,
                                                      const unsigned* __restrict__ esrc,
                                                      const ulonglong2* __restrict__ ew)
{
    const long long t = (long long)blockIdx.x * 256 + threadIdx.x;
    if (t >= n_targets) return;
    u64 ac = 0, bd = 0, sm = 0;   // Karatsuba parts, nearly canonical
    for (unsigned e = ptr[t]; e < ptr[t + 1]; ++e) {
        const ulonglong2 w = __ldg(ew + e), x = v[src_row + esrc[e]];
        ac = fold61(ac + lmul(x.y, w.y));
        bd = fold61(bd + lmul(x.x, w.x));
        sm = fold61(sm + lmul(x.y + x.x, w.y + w.x));
    }
    const u64 re = fold61(ac + (2 * P61 - bd));
    const u64 im = fold61(sm + (4 * P61 - ac - bd));
    v[dst_row + t] = make_ulonglong2(canon61(im), canon61(re));
}

struct Root {
    uint32_t w[8];   // digest words as the tree stores them after the byte swap
};

__device__ __forceinline__ void digest_words(const unsigned char* d, uint32_t* w)
{
    const uint4* p = reinterpret_cast<const uint4*>(d);
    const uint4 a = p[0], b = p[1];
    w[0] = sha::bswap32(a.x); w[1] = sha::bswap32(a.y); w[2] = sha::bswap32(a.z); w[3] = sha::bswap32(a.w);
    w[4] = sha::bswap32(b.x); w[5] = sha::bswap32(b.y); w[6] = sha::bswap32(b.z); w[7] = sha::bswap32(b.w);
}

// node index -> position in the sorted list, or -1
__device__ __forceinline__ int find(const unsigned* idx, int n, unsigned key)
{
    int lo = 0, hi = n - 1;
    while (lo <= hi) {
        const int mid = (lo + hi) >> 1;
        const unsigned m = idx[mid];
        if (m == key) return mid;
        if (m < key) lo = mid + 1; else hi = mid - 1;
    }
    return -1;
}

// walks from leaf `h` at position pos up to node 1 with the listed siblings
__device__ bool walk(uint32_t h[8], long long pos, long long leaves, const unsigned* idx, const unsigned char* dig,
                     int n, const Root& root, uint32_t one)
{
    long long node = pos + leaves;
    while (node != 1) {
        const int k = find(idx, n, (unsigned)(node ^ 1));
        if (k < 0) return false;
        uint32_t w[16], s[8];
        uint32_t* mine = w + ((node & 1) ? 8 : 0);
        uint32_t* sib = w + ((node & 1) ? 0 : 8);
#pragma unroll
        for (int i = 0; i < 8; ++i) mine[i] = h[i];
        digest_words(dig + 32LL * k, sib);
        sha::hash64(w, s, sha::AddMad{one});
#pragma unroll
        for (int i = 0; i < 8; ++i) h[i] = s[i];
        node >>= 1;
    }
    bool eq = true;
#pragma unroll
    for (int i = 0; i < 8; ++i) eq &= h[i] == root.w[i];
    return eq;
}

__global__ void __launch_bounds__(128) verify_kernel(const long long* __restrict__ q, const long long* __restrict__ q2,
                                                     int count, long long leaves, long long cw_len,
                                                     const ulonglong2* __restrict__ col_sums,
                                                     const unsigned char* __restrict__ col_digests,
                                                     const ulonglong2* __restrict__ combined,
                                                     const ulonglong2* __restrict__ enc,
                                                     const unsigned* __restrict__ com_idx,
                                                     const unsigned char* __restrict__ com_dig, int n_com,
                                                     const unsigned* __restrict__ cmb_idx,
                                                     const unsigned char* __restrict__ cmb_dig, int n_cmb,
                                                     Root com_root, Root cmb_root, uint32_t one,
                                                     int* __restrict__ flags)
{
    const int i = blockIdx.x * 128 + threadIdx.x;
    if (i >= count) return;
    const long long p = q[i], p2 = q2 ? q2[i] : 0;
    if (p < 0 || p >= cw_len || p2 < 0 || p2 >= cw_len) {
        flags[i] = 16;
        return;
    }
    int f = 0;
    const ulonglong2 a = col_sums[i], b = combined[p];
    if (a.x != b.x || a.y != b.y) f |= 1;
    uint32_t h[8];
    digest_words(col_digests + 32LL * i, h);
    if (!walk(h, p, leaves, com_idx, com_dig, n_com, com_root, one)) f |= 2;
    uint32_t w[16];
    sha::fe_words(b.x, b.y, w);
#pragma unroll
    for (int k = 4; k < 16; ++k) w[k] = 0;
    sha::hash64(w, h, sha::AddMad{one});
    if (!walk(h, p, leaves, cmb_idx, cmb_dig, n_cmb, cmb_root, one)) f |= 4;
    if (q2) {
        const ulonglong2 e = enc[p2], c = combined[p2];
        if (e.x != c.x || e.y != c.y) f |= 8;
    }
    flags[i] = f;
}

Root root_of(const unsigned char* r32)
{
    Root r;
    for (int i = 0; i < 8; ++i)
        r.w[i] = ((uint32_t)r32[4 * i] << 24) | ((uint32_t)r32[4 * i + 1] << 16) | ((uint32_t)r32[4 * i + 2] << 8) |
                 (uint32_t)r32[4 * i + 3];
    return r;
}

}  // namespace

bool encode_vector(const Encoder& enc, const ulonglong2* msg, ulonglong2* out, cudaStream_t s)
{
    if (cuda_failed(cudaMemcpyAsync(out, msg, sizeof(ulonglong2) * enc.col_len, cudaMemcpyDeviceToDevice, s),
                    "orion encode message"))
        return false;
    for (const Level& lv : enc.levels) {
        if (lv.R == 0) continue;
        gather1_kernel<<<(unsigned)((lv.R + 255) / 256), 256, 0, s>>>(out, lv.off, lv.off + lv.n, lv.R,
                                                                      enc.d_ptr + lv.c_ptr, enc.d_src + lv.c_edge,
                                                                      enc.d_w + lv.c_edge);
        if (cuda_failed(cudaGetLastError(), "orion encode C")) return false;
    }
    for (auto it = enc.levels.rbegin(); it != enc.levels.rend(); ++it) {
        const Level& lv = *it;
        if (lv.RD == 0) continue;
        const long long next = lv.off + lv.n;
        gather1_kernel<<<(unsigned)((lv.RD + 255) / 256), 256, 0, s>>>(out, next, next + lv.L, lv.RD,
                                                                       enc.d_ptr + lv.d_ptr, enc.d_src + lv.d_edge,
                                                                       enc.d_w + lv.d_edge);
        if (cuda_failed(cudaGetLastError(), "orion encode D")) return false;
    }
    return true;
}

bool verify_opening(long long msg_len, long long cw_len, const ulonglong2* r0, const long long* q,
                    const long long* q2, int count, const ulonglong2* cols, const ulonglong2* combined,
                    const ulonglong2* enc, const unsigned* com_idx, const unsigned char* com_dig, int n_com,
                    const unsigned* cmb_idx, const unsigned char* cmb_dig, int n_cmb, const unsigned char* com_root,
                    const unsigned char* cmb_root, int* flags, cudaStream_t s)
{
    // the column sums (the commit's combine pass over the queried columns) and
    // the columns' leaf chains, in one scratch block
    const size_t sums_bytes = sizeof(ulonglong2) * count, dig_bytes = 32 * (size_t)count;
    unsigned char* scratch = static_cast<unsigned char*>(dev_alloc(sums_bytes + dig_bytes, s));
    if (!scratch) return false;
    ulonglong2* sums = reinterpret_cast<ulonglong2*>(scratch);
    unsigned char* digs = scratch + sums_bytes;
    bool ok = combine(cols, msg_len, count, r0, sums, nullptr, s) && leaf_digests(cols, count, digs, s);
    if (ok) {
        verify_kernel<<<(unsigned)((count + 127) / 128), 128, 0, s>>>(
            q, q2, count, tree_leaves(msg_len), cw_len, sums, digs, combined, enc, com_idx, com_dig, n_com, cmb_idx,
            cmb_dig, n_cmb, root_of(com_root), root_of(cmb_root), 1u, flags);
        ok = !cuda_failed(cudaGetLastError(), "orion verify");
    }
    dev_free(scratch, s);
    return ok;
}

}  // namespace orion
}  // namespace tp
