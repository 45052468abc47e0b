// Helpers of the Orion opening proof for a prover that proves many frames at
// once (truepix_b200/pipeline.py): the eq tables of the opening point on the
// host (the row weights r1 also enter the opening's host transcript), the list of
// Merkle nodes an opening file carries (collect_merkle_siblings,
// TruePix-main/Orion/Orion_nonzk/src/truepix/orion_proof.cpp:153-174), and a
// device gather of those nodes, so that only the digests the file needs leave
// the GPU instead of the whole trees.
#include <stdint.h>
#include <string.h>

#include <vector>

#include "fp2.cuh"
#include "runtime.h"
#include "../../include/orion_gpu.h"

namespace {

using tp::fp2;

// out[i] = tree[nodes[i]] (32-byte digests); a node outside the tree gives zeros
__global__ void gather_nodes_kernel(const uint4* __restrict__ tree, long long tree_nodes,
                                    const int* __restrict__ nodes, int n, uint4* __restrict__ out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;   // one 16-byte half of a digest
    if (i >= 2 * n) return;
    const long long node = nodes[i >> 1];
    out[i] = node >= 0 && node < tree_nodes ? tree[2 * node + (i & 1)] : make_uint4(0, 0, 0, 0);
}

}  // namespace

extern "C" {

int tp_eq_table_host(const uint64_t* z, int k, uint64_t* out)
{
    tp::clear_error();
    if (!z || !out || k < 0 || k > 26) {
        tp::set_error(tp::TP_ERR_ARG, "tp_eq_table_host: bad arguments");
        return -1;
    }
    for (int j = 0; j < k; ++j)
        if (z[2 * j] >= tp::P61 || z[2 * j + 1] >= tp::P61) {
            tp::set_error(tp::TP_ERR_ARG, "tp_eq_table_host: coordinate %d is not canonical", j);
            return -1;
        }
    fp2* t = reinterpret_cast<fp2*>(out);
    t[0] = tp::mk(1, 0);
    for (int j = 0; j < k; ++j) {
        const fp2 zj = tp::mk(z[2 * j], z[2 * j + 1]);
        const fp2 one_m = tp::f2sub(tp::mk(1, 0), zj);
        const long long half = 1ll << j;
        for (long long i = 0; i < half; ++i) {
            const fp2 v = t[i];
            t[i + half] = tp::f2mul(v, zj);
            t[i] = tp::f2mul(v, one_m);
        }
    }
    return 0;
}

int tp_orion_path_nodes(long long n_leaves, const long long* positions, int count, int* out_nodes, int cap)
{
    tp::clear_error();
    if (n_leaves < 2 || (n_leaves & (n_leaves - 1)) != 0 || n_leaves > (1ll << 30) || !positions || count < 0 ||
        !out_nodes || cap < 0) {
        tp::set_error(tp::TP_ERR_ARG, "tp_orion_path_nodes: bad arguments");
        return -1;
    }
    std::vector<uint8_t> seen((size_t)(2 * n_leaves), 0);
    int n = 0;
    for (int q = 0; q < count; ++q) {
        if (positions[q] < 0 || positions[q] >= n_leaves) {
            tp::set_error(tp::TP_ERR_ARG, "tp_orion_path_nodes: position %d out of range", q);
            return -1;
        }
        for (long long node = positions[q] + n_leaves; node != 1; node >>= 1) {
            const long long sib = node ^ 1;
            if (seen[(size_t)sib]) continue;
            seen[(size_t)sib] = 1;
            if (n == cap) {
                tp::set_error(tp::TP_ERR_ARG, "tp_orion_path_nodes: more than %d nodes", cap);
                return -1;
            }
            out_nodes[n++] = (int)sib;
        }
    }
    return n;
}

long long tp_orion_opening_file_size(long long msg_len, long long cw_len, int n_queries, int n_com_nodes,
                                     int n_comb_nodes)
{
    if (msg_len < 0 || cw_len < 0 || n_queries < 0 || n_com_nodes < 0 || n_comb_nodes < 0) return -1;
    return 8 + 44 + 16 + 32 + 32 + 8ll * n_queries + 16ll * 128 * n_queries + 16 * cw_len + 16 * msg_len +
           8 + 36ll * n_com_nodes + 8 + 36ll * n_comb_nodes;
}

long long tp_orion_opening_file(long long N, long long msg_len, long long cw_len, const uint64_t* answer,
                                const unsigned char* com_root, const unsigned char* comb_root, const long long* col_q,
                                int n_queries, const uint64_t* cols, const uint64_t* combined, const int* com_idx,
                                const unsigned char* com_nodes, int n_com_nodes, const int* comb_idx,
                                const unsigned char* comb_nodes, int n_comb_nodes, int use_group1, unsigned char* out,
                                long long cap)
{
    tp::clear_error();
    const long long size = tp_orion_opening_file_size(msg_len, cw_len, n_queries, n_com_nodes, n_comb_nodes);
    if (size < 0 || !answer || !com_root || !comb_root || (n_queries && (!col_q || !cols)) || !combined || !out ||
        msg_len > cw_len || (n_com_nodes && (!com_idx || !com_nodes)) || (n_comb_nodes && (!comb_idx || !comb_nodes))) {
        tp::set_error(tp::TP_ERR_ARG, "tp_orion_opening_file: bad arguments");
        return -1;
    }
    if (cap < size) {
        tp::set_error(tp::TP_ERR_ARG, "tp_orion_opening_file: %lld bytes needed, %lld given", size, cap);
        return -1;
    }
    unsigned char* o = out;
    auto put = [&](const void* p, size_t n) {
        memcpy(o, p, n);
        o += n;
    };
    auto u32 = [&](uint32_t v) { put(&v, 4); };
    auto u64 = [&](uint64_t v) { put(&v, 8); };
    put("ORIONPV1", 8);
    u32(2);
    u32((uint32_t)use_group1);
    u64((uint64_t)N);
    u64(128);
    u64((uint64_t)msg_len);
    u64((uint64_t)cw_len);
    u32((uint32_t)n_queries);
    put(answer, 16);
    put(com_root, 32);
    put(comb_root, 32);
    put(col_q, 8 * (size_t)n_queries);
    put(cols, 16 * 128 * (size_t)n_queries);
    put(combined, 16 * (size_t)cw_len);
    put(combined, 16 * (size_t)msg_len);
    for (int t = 0; t < 2; ++t) {
        const int n = t ? n_comb_nodes : n_com_nodes;
        const int* idx = t ? comb_idx : com_idx;
        const unsigned char* dig = t ? comb_nodes : com_nodes;
        u64((uint64_t)n);
        for (int i = 0; i < n; ++i) {
            u32((uint32_t)idx[i]);
            put(dig + 32 * (size_t)i, 32);
        }
    }
    return (long long)(o - out);
}

int tp_orion_gather_nodes_dev(const void* d_tree, long long n_nodes_tree, const void* d_nodes, int n, void* d_out,
                              void* stream)
{
    tp::clear_error();
    if (!tp::ctx()) return -1;
    if (!d_tree || n_nodes_tree < 2 || n < 0 || (n > 0 && (!d_nodes || !d_out))) {
        tp::set_error(tp::TP_ERR_ARG, "tp_orion_gather_nodes_dev: bad arguments");
        return -1;
    }
    if (n == 0) return 0;
    const int threads = 256;
    gather_nodes_kernel<<<(2 * n + threads - 1) / threads, threads, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
        static_cast<const uint4*>(d_tree), n_nodes_tree, static_cast<const int*>(d_nodes), n,
        static_cast<uint4*>(d_out));
    return tp::cuda_failed(cudaGetLastError(), "gather nodes") ? -1 : 0;
}

}  // extern "C"
