// C ABI of the Orion commitment (include/orion_gpu.h).
#include <stdint.h>
#include <string.h>

#include <algorithm>

#include "fp2.cuh"
#include "orion.h"
#include "runtime.h"
#include "../../include/orion_gpu.h"

namespace {

constexpr long long kMaxColLen = 1LL << 22;

bool check_n(long long N, const char* who)
{
    if (N <= 0 || N % tp::orion::kColumns != 0 || N / tp::orion::kColumns > kMaxColLen) {
        tp::set_error(tp::TP_ERR_ARG, "%s: N = %lld must be a positive multiple of 128 with N/128 <= 2^22",
                      who, N);
        return false;
    }
    return true;
}

struct DevBuf {
    void* p = nullptr;
    cudaStream_t s;
    explicit DevBuf(size_t bytes, cudaStream_t st) : s(st) { p = tp::dev_alloc(bytes, st); }
    ~DevBuf()
    {
        if (p) tp::dev_free(p, s);
    }
};

// checks a frame layout (the TruePix layout of truepix_gkr.h:107-206) and fills px and N
bool pixel_layout(const void* d_pixels, int n_copies, int n_copies_padded, int copy_size, int n_wires,
                  int const_idx, uint64_t const_val, const char* who, tp::orion::PixelInput& px, long long& N)
{
    if (!d_pixels || n_copies < 0 || n_copies > n_copies_padded || copy_size <= 0 || copy_size > n_wires ||
        n_wires <= 0 || (n_wires & (n_wires - 1)) || n_copies_padded <= 0 || const_idx >= n_wires ||
        (const_idx >= 0 && const_idx < copy_size) || const_val >= tp::P61) {
        tp::set_error(tp::TP_ERR_ARG, "%s: layout copies %d/%d, copy_size %d, wires %d, const %d", who, n_copies,
                      n_copies_padded, copy_size, n_wires, const_idx);
        return false;
    }
    N = (long long)n_copies_padded * n_wires;
    if (!check_n(N, who)) return false;
    px.pix = static_cast<const unsigned char*>(d_pixels);
    px.copies = n_copies;
    px.cs = copy_size;
    px.W = n_wires;
    px.const_idx = const_idx;
    px.const_val = const_val;
    return true;
}

// *first = min(*first, i) over words w[i] >= p (non-canonical limbs)
__global__ void __launch_bounds__(256) noncanonical_kernel(const uint64_t* __restrict__ w, long long n,
                                                           unsigned long long* __restrict__ first)
{
    for (long long i = (long long)blockIdx.x * 256 + threadIdx.x; i < n; i += (long long)gridDim.x * 256)
        if (w[i] >= tp::P61) atomicMin(first, (unsigned long long)i);
}

// the index of the first non-canonical limb of d_words (n words) or -1; false
// on a CUDA error. Synchronises s.
bool first_noncanonical(const void* d_words, long long n, cudaStream_t s, long long* first)
{
    DevBuf flag(8, s);
    if (!flag.p) return false;
    unsigned long long h = ~0ull;
    if (tp::cuda_failed(cudaMemsetAsync(flag.p, 0xFF, 8, s), "canonical check")) return false;
    const tp::Ctx* c = tp::ctx();
    const long long blocks = std::min<long long>((n + 255) / 256, (long long)c->n_sm * 16);
    noncanonical_kernel<<<(unsigned)std::max<long long>(1, blocks), 256, 0, s>>>(
        static_cast<const uint64_t*>(d_words), n, static_cast<unsigned long long*>(flag.p));
    if (tp::cuda_failed(cudaGetLastError(), "canonical check") ||
        tp::cuda_failed(cudaMemcpyAsync(&h, flag.p, 8, cudaMemcpyDeviceToHost, s), "D2H") ||
        tp::cuda_failed(cudaStreamSynchronize(s), "synchronize"))
        return false;
    *first = h == ~0ull ? -1 : (long long)h;
    return true;
}

// a host-buffer commit of N elements {img, real}: the tree to tree_out, the
// column-major codeword to codeword_out when it is set
int commit_host(const uint64_t* src, long long N, unsigned char* tree_out, uint64_t* codeword_out, const char* who)
{
    tp::Ctx* c = tp::ctx();
    if (!c) return -1;
    if (!check_n(N, who)) return -1;
    if (!src || !tree_out) {
        tp::set_error(tp::TP_ERR_ARG, "%s: null buffer", who);
        return -1;
    }
    const long long col_len = N / tp::orion::kColumns;
    const tp::orion::Encoder* e = tp::orion::encoder(col_len);
    if (!e) return -1;
    const long long cw_len = e->cw_len, leaves = tp::orion::tree_leaves(col_len);
    cudaStream_t s = c->stream;
    DevBuf d_src(16 * (size_t)N, s), d_rows(16 * (size_t)cw_len * tp::orion::kColumns, s),
        d_tree(64 * (size_t)leaves, s);
    if (!d_src.p || !d_rows.p || !d_tree.p) return -1;
    if (!tp::host_to_device(d_src.p, src, 16 * (size_t)N, s)) return -1;
    long long bad = -1;
    if (!first_noncanonical(d_src.p, 2 * N, s, &bad)) return -1;
    if (bad >= 0) {
        tp::set_error(tp::TP_ERR_ARG, "%s: element %lld is not canonical", who, bad / 2);
        return -1;
    }
    if (!tp::orion::commit(*e, static_cast<const ulonglong2*>(d_src.p), nullptr, static_cast<ulonglong2*>(d_rows.p),
                           static_cast<unsigned char*>(d_tree.p), s))
        return -1;
    if (!tp::device_to_host(tree_out, d_tree.p, 64 * (size_t)leaves, s)) return -1;
    if (codeword_out) {
        DevBuf d_cols(16 * (size_t)cw_len * tp::orion::kColumns, s);
        if (!d_cols.p) return -1;
        if (!tp::orion::rows_to_columns(static_cast<const ulonglong2*>(d_rows.p), cw_len,
                                        static_cast<ulonglong2*>(d_cols.p), s))
            return -1;
        if (!tp::device_to_host(codeword_out, d_cols.p, 16 * (size_t)cw_len * tp::orion::kColumns, s)) return -1;
    }
    return tp::cuda_failed(cudaStreamSynchronize(s), "synchronize") ? -1 : 0;
}

}  // namespace

extern "C" {

long long tp_orion_codeword_len(long long col_len)
{
    if (col_len <= 0) return 0;
    return tp::orion::codeword_len(col_len);
}

long long tp_orion_tree_leaves(long long N)
{
    if (N <= 0 || N % tp::orion::kColumns) return 0;
    return tp::orion::tree_leaves(N / tp::orion::kColumns);
}

int tp_orion_commit_dev(const void* d_src, long long N, void* d_rows, void* d_tree, void* stream)
{
    tp::clear_error();
    if (!tp::ctx()) return -1;
    if (!check_n(N, "tp_orion_commit_dev")) return -1;
    if (!d_src || !d_rows || !d_tree) {
        tp::set_error(tp::TP_ERR_ARG, "tp_orion_commit_dev: null buffer");
        return -1;
    }
    const tp::orion::Encoder* e = tp::orion::encoder(N / tp::orion::kColumns);
    if (!e) return -1;
    return tp::orion::commit(*e, static_cast<const ulonglong2*>(d_src), nullptr, static_cast<ulonglong2*>(d_rows),
                             static_cast<unsigned char*>(d_tree), reinterpret_cast<cudaStream_t>(stream))
               ? 0
               : -1;
}

int tp_orion_commit_pixels_dev(const void* d_pixels, int n_copies, int n_copies_padded, int copy_size,
                               int n_wires, int const_idx, uint64_t const_val, void* d_rows, void* d_tree,
                               void* stream)
{
    tp::clear_error();
    if (!tp::ctx()) return -1;
    tp::orion::PixelInput px;
    long long N = 0;
    if (!pixel_layout(d_pixels, n_copies, n_copies_padded, copy_size, n_wires, const_idx, const_val,
                      "tp_orion_commit_pixels_dev", px, N))
        return -1;
    if (!d_rows || !d_tree) {
        tp::set_error(tp::TP_ERR_ARG, "tp_orion_commit_pixels_dev: null buffer");
        return -1;
    }
    const tp::orion::Encoder* e = tp::orion::encoder(N / tp::orion::kColumns);
    if (!e) return -1;
    return tp::orion::commit(*e, nullptr, &px, static_cast<ulonglong2*>(d_rows),
                             static_cast<unsigned char*>(d_tree), reinterpret_cast<cudaStream_t>(stream))
               ? 0
               : -1;
}

int tp_orion_commit_zk_pixels_dev(const void* d_pixels, int n_copies, int n_copies_padded, int copy_size,
                                  int n_wires, int const_idx, uint64_t const_val, uint64_t mask_seed,
                                  void* d_rows_masked, void* d_tree_masked, void* d_rows_mask, void* d_tree_mask,
                                  void* stream)
{
    tp::clear_error();
    if (!tp::ctx()) return -1;
    tp::orion::PixelInput px;
    long long N = 0;
    if (!pixel_layout(d_pixels, n_copies, n_copies_padded, copy_size, n_wires, const_idx, const_val,
                      "tp_orion_commit_zk_pixels_dev", px, N))
        return -1;
    if (!d_rows_masked || !d_tree_masked || !d_rows_mask || !d_tree_mask) {
        tp::set_error(tp::TP_ERR_ARG, "tp_orion_commit_zk_pixels_dev: null buffer");
        return -1;
    }
    const tp::orion::Encoder* e = tp::orion::encoder(N / tp::orion::kColumns);
    if (!e) return -1;
    const cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    px.mask_seed = mask_seed;
    px.mask_mode = tp::orion::kMaskMasked;
    if (!tp::orion::commit(*e, nullptr, &px, static_cast<ulonglong2*>(d_rows_masked),
                           static_cast<unsigned char*>(d_tree_masked), s))
        return -1;
    const int first = tp::orion::last_launches();
    px.mask_mode = tp::orion::kMaskOnly;
    if (!tp::orion::commit(*e, nullptr, &px, static_cast<ulonglong2*>(d_rows_mask),
                           static_cast<unsigned char*>(d_tree_mask), s))
        return -1;
    tp::orion::add_launches(first);
    return 0;
}

int tp_orion_pixel_vector_dev(const void* d_pixels, int n_copies, int n_copies_padded, int copy_size, int n_wires,
                              int const_idx, uint64_t const_val, uint64_t mask_seed, int mask_mode, void* d_out,
                              void* stream)
{
    tp::clear_error();
    if (!tp::ctx()) return -1;
    tp::orion::PixelInput px;
    long long N = 0;
    if (!pixel_layout(d_pixels, n_copies, n_copies_padded, copy_size, n_wires, const_idx, const_val,
                      "tp_orion_pixel_vector_dev", px, N))
        return -1;
    if (!d_out || mask_mode < tp::orion::kMaskNone || mask_mode > tp::orion::kMaskOnly) {
        tp::set_error(tp::TP_ERR_ARG, "tp_orion_pixel_vector_dev: null output or mask mode %d", mask_mode);
        return -1;
    }
    px.mask_seed = mask_seed;
    px.mask_mode = mask_mode;
    return tp::orion::pixel_vector(px, N, static_cast<uint64_t*>(d_out), reinterpret_cast<cudaStream_t>(stream))
               ? 0
               : -1;
}

int tp_orion_last_launches(void) { return tp::orion::last_launches(); }

int tp_orion_set_leaf_chunks(int n)
{
    tp::clear_error();
    return tp::orion::set_leaf_chunks(n) ? 0 : -1;
}

int tp_orion_set_gather_lanes(int columns_per_lane)
{
    tp::clear_error();
    return tp::orion::set_gather_lanes(columns_per_lane) ? 0 : -1;
}

int tp_orion_combine_dev(const void* d_rows, long long N, const void* d_r0, void* d_combined, void* d_ctree,
                         void* stream)
{
    tp::clear_error();
    if (!tp::ctx()) return -1;
    if (!check_n(N, "tp_orion_combine_dev")) return -1;
    if (!d_rows || !d_r0 || !d_combined) {
        tp::set_error(tp::TP_ERR_ARG, "tp_orion_combine_dev: null buffer");
        return -1;
    }
    const long long col_len = N / tp::orion::kColumns;
    return tp::orion::combine(static_cast<const ulonglong2*>(d_rows), col_len, tp::orion::codeword_len(col_len),
                              static_cast<const ulonglong2*>(d_r0), static_cast<ulonglong2*>(d_combined),
                              static_cast<unsigned char*>(d_ctree), reinterpret_cast<cudaStream_t>(stream))
               ? 0
               : -1;
}

int tp_orion_query_columns_dev(const void* d_rows, long long N, const void* d_q, int count, void* d_out,
                               void* stream)
{
    tp::clear_error();
    if (!tp::ctx()) return -1;
    if (!check_n(N, "tp_orion_query_columns_dev")) return -1;
    if (!d_rows || !d_q || !d_out || count <= 0) {
        tp::set_error(tp::TP_ERR_ARG, "tp_orion_query_columns_dev: bad arguments");
        return -1;
    }
    const long long col_len = N / tp::orion::kColumns;
    return tp::orion::query_rows(static_cast<const ulonglong2*>(d_rows), tp::orion::codeword_len(col_len),
                                 static_cast<const long long*>(d_q), count, static_cast<ulonglong2*>(d_out),
                                 reinterpret_cast<cudaStream_t>(stream))
               ? 0
               : -1;
}

int tp_orion_query_columns_async_dev(const void* d_rows, long long N, const void* d_q, int count, void* d_out,
                                     int* d_bad, void* stream)
{
    tp::clear_error();
    if (!tp::ctx()) return -1;
    if (!check_n(N, "tp_orion_query_columns_async_dev")) return -1;
    if (!d_rows || !d_q || !d_out || count <= 0) {
        tp::set_error(tp::TP_ERR_ARG, "tp_orion_query_columns_async_dev: bad arguments");
        return -1;
    }
    const long long col_len = N / tp::orion::kColumns;
    return tp::orion::query_rows_async(static_cast<const ulonglong2*>(d_rows), tp::orion::codeword_len(col_len),
                                       static_cast<const long long*>(d_q), count, static_cast<ulonglong2*>(d_out),
                                       d_bad, reinterpret_cast<cudaStream_t>(stream))
               ? 0
               : -1;
}

int tp_orion_answer_dev(const void* d_combined, long long msg_len, const void* d_r1, void* d_answer, void* stream)
{
    tp::clear_error();
    if (!tp::ctx()) return -1;
    if (!d_combined || !d_r1 || !d_answer || msg_len <= 0) {
        tp::set_error(tp::TP_ERR_ARG, "tp_orion_answer_dev: bad arguments");
        return -1;
    }
    return tp::orion::answer(static_cast<const ulonglong2*>(d_combined), static_cast<const ulonglong2*>(d_r1),
                             msg_len, static_cast<ulonglong2*>(d_answer), reinterpret_cast<cudaStream_t>(stream))
               ? 0
               : -1;
}

int tp_orion_encode_dev(const void* d_msg, long long col_len, void* d_out, void* stream)
{
    tp::clear_error();
    if (!tp::ctx()) return -1;
    if (!d_msg || !d_out || col_len <= 0 || col_len > (1LL << 22)) {
        tp::set_error(tp::TP_ERR_ARG, "tp_orion_encode_dev: bad arguments");
        return -1;
    }
    const tp::orion::Encoder* e = tp::orion::encoder(col_len);
    if (!e) return -1;
    return tp::orion::encode_vector(*e, static_cast<const ulonglong2*>(d_msg), static_cast<ulonglong2*>(d_out),
                                    reinterpret_cast<cudaStream_t>(stream))
               ? 0
               : -1;
}

int tp_orion_verify_opening_dev(long long msg_len, long long cw_len, const void* d_r0, const void* d_q,
                                const void* d_q2, int count, const void* d_cols, const void* d_combined,
                                const void* d_enc, const void* d_com_idx, const void* d_com_nodes, int n_com,
                                const void* d_cmb_idx, const void* d_cmb_nodes, int n_cmb,
                                const unsigned char* com_root, const unsigned char* comb_root, int* d_flags,
                                void* stream)
{
    tp::clear_error();
    if (!tp::ctx()) return -1;
    if (msg_len <= 0 || (msg_len & (msg_len - 1)) || cw_len != tp::orion::codeword_len(msg_len) || !d_r0 || !d_q ||
        count <= 0 || !d_cols || !d_combined || (d_q2 && !d_enc) || !d_com_idx || !d_com_nodes || n_com <= 0 ||
        !d_cmb_idx || !d_cmb_nodes || n_cmb <= 0 || !com_root || !comb_root || !d_flags) {
        tp::set_error(tp::TP_ERR_ARG, "tp_orion_verify_opening_dev: bad arguments");
        return -1;
    }
    return tp::orion::verify_opening(msg_len, cw_len, static_cast<const ulonglong2*>(d_r0),
                                     static_cast<const long long*>(d_q), static_cast<const long long*>(d_q2), count,
                                     static_cast<const ulonglong2*>(d_cols), static_cast<const ulonglong2*>(d_combined),
                                     static_cast<const ulonglong2*>(d_enc), static_cast<const unsigned*>(d_com_idx),
                                     static_cast<const unsigned char*>(d_com_nodes), n_com,
                                     static_cast<const unsigned*>(d_cmb_idx),
                                     static_cast<const unsigned char*>(d_cmb_nodes), n_cmb, com_root, comb_root,
                                     d_flags, reinterpret_cast<cudaStream_t>(stream))
               ? 0
               : -1;
}

int tp_sha256_peak_dev(int blocks, int iters, void* d_out, void* stream)
{
    tp::clear_error();
    if (!tp::ctx()) return -1;
    if (blocks <= 0 || iters <= 0 || !d_out) {
        tp::set_error(tp::TP_ERR_ARG, "tp_sha256_peak_dev: bad arguments");
        return -1;
    }
    return tp::orion::sha_peak(blocks, iters, static_cast<uint32_t*>(d_out), reinterpret_cast<cudaStream_t>(stream))
               ? 0
               : -1;
}

int tp_orion_rows_to_columns_dev(const void* d_rows, long long cw_len, void* d_cols, void* stream)
{
    tp::clear_error();
    if (!tp::ctx()) return -1;
    if (!d_rows || !d_cols || cw_len <= 0) {
        tp::set_error(tp::TP_ERR_ARG, "tp_orion_rows_to_columns_dev: bad arguments");
        return -1;
    }
    return tp::orion::rows_to_columns(static_cast<const ulonglong2*>(d_rows), cw_len,
                                      static_cast<ulonglong2*>(d_cols), reinterpret_cast<cudaStream_t>(stream))
               ? 0
               : -1;
}

int tp_orion_commit(const uint64_t* src, long long N, unsigned char* tree_out, uint64_t* codeword_out)
{
    tp::clear_error();
    return commit_host(src, N, tree_out, codeword_out, "tp_orion_commit");
}

int tp_orion_commit_pair(const uint64_t* masked, const uint64_t* mask, long long N, unsigned char* tree_masked,
                         unsigned char* tree_mask)
{
    tp::clear_error();
    if (commit_host(masked, N, tree_masked, nullptr, "tp_orion_commit_pair (masked)")) return -1;
    return commit_host(mask, N, tree_mask, nullptr, "tp_orion_commit_pair (mask)");
}

}  // extern "C"
