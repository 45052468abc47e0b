// Orion input-layer commitment on the device: expander encode of 128 columns
// and the SHA-256 Merkle tree over the codeword rows.
//
// Reference: TruePix-main/Orion/Orion_nonzk -- commit() src/VPD/linearPC.cpp:97-197,
// encode() include/linear_code/linear_code_encode.h:17-72, graphs
// include/linear_code/expanders.h:19-60, tree src/infrastructure/merkle_tree.cpp:28-84.
//
// Device layout (ours): the codeword of all 128 columns is one row-major matrix
// rows[r][c] of 16-byte field elements {u64 img, u64 real} (the reference's element
// memory order), r < cw_len. A row is 2 KB: the expander gathers of one row and
// the leaf hash of one row both read it contiguously. The encoder's levels live
// in that one matrix: level k's message starts at row off_k, its codeword is
// [message | codeword of level k+1 | D-part], and level k+1's message starts at
// off_k + n_k, so no level needs a copy.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

namespace tp {
namespace orion {

constexpr int kColumns = 128;     // column_size (include/linear_code/parameter.h)
constexpr int kThreshold = 13;    // distance_threshold = (int)(1 / 0.07) - 1
constexpr int kCDegree = 10;      // cn
constexpr int kDDegree = 20;      // dn

struct Level {
    long long n;     // message length at this depth
    long long R;     // C targets  = (long long)(0.238 * n)
    long long L;     // codeword length of the next depth
    long long RD;    // D targets  = (long long)(n * 0.72 - L)
    long long off;   // first row of this depth's message in the codeword matrix
    long long c_ptr, c_edge;   // offsets of this depth's C graph in the CSR arrays
    long long d_ptr, d_edge;   // same for the D graph
};

// Graphs of one column length, transposed to CSR by target on the host and kept
// on the device (the reference draws them from glibc rand() in its default seed
// state; the same draws are replayed here).
struct Encoder {
    int device = -1;
    long long col_len = 0;
    long long cw_len = 0;
    std::vector<Level> levels;         // depths with n > kThreshold, outermost first
    long long n_ptr = 0, n_edges = 0;
    unsigned max_c0_in_degree = 0;     // largest in-degree of the depth-0 C graph
    unsigned* d_ptr = nullptr;         // [n_ptr] first edge of each target (per graph, + 1 end)
    unsigned* d_src = nullptr;         // [n_edges] source row within the graph's source range
    ulonglong2* d_w = nullptr;         // [n_edges] weights {img, real}, canonical
    // The reference draws each weight limb as rand() % p (prime_field::random,
    // src/linear_gkr/prime_field.cpp:35-40), so both limbs are below 2^31; when
    // every weight is, they are also kept as {real, img} 32-bit pairs and the
    // gathers multiply 61 x 31 bits (d_w32 non-null).
    uint2* d_w32 = nullptr;            // [n_edges]
};

// cached per (device, col_len); nullptr and the error set on failure
const Encoder* encoder(long long col_len);
// encode_output_len(col_len), computed without building graphs
long long codeword_len(long long col_len);
// power of two >= 2 * col_len (the Merkle tree has 2 * leaves() digests)
long long tree_leaves(long long col_len);

// Host-side SHA-256 constants of the commit: the chain of a row of zeros and
// SHA-256 of 64 zero bytes (padded tree leaves), as digest bytes.
void zero_row_leaf(unsigned char out[32]);
void zero_block_hash(unsigned char out[32]);

// Frame bytes as the commit's input vector (TruePix layout, truepix_gkr.h:107-206):
// element f = copy * W + wire is pixel[copy * cs + wire] for wire < cs and copy < copies,
// const_val at wire == const_idx (copy < copies), zero elsewhere (real part; img 0).
//
// ZK commits (TruePix-main/Orion/Orion_zk/include/truepix/truepix_gkr.h:286-384)
// replace that vector by the masked polynomial (mask_mode kMaskMasked: element +
// mask) or the mask alone (kMaskOnly). The mask is zero except at the private
// wires (wire < cs, copy < copies), where the k-th private wire in flat order,
// k = copy * cs + wire, holds splitmix64 output number k + 1 of the state
// mask_seed, reduced mod 2^61 - 1 (real part; img 0).
enum MaskMode { kMaskNone = 0, kMaskMasked = 1, kMaskOnly = 2 };

struct PixelInput {
    const unsigned char* pix;
    int copies, cs, W, const_idx;
    uint64_t const_val;
    uint64_t mask_seed = 0;
    int mask_mode = kMaskNone;
};

// the polynomial a PixelInput stands for, as base-field values out[f], f < copies_padded * W
bool pixel_vector(const PixelInput& px, long long n, uint64_t* out, cudaStream_t s);

// Full commit into caller buffers: rows (cw_len x 128 elements) and tree
// (2 * tree_leaves digests of 32 bytes, heap order, root at index 1).
// src is the reference's column-major input (column c = src[c * col_len ..]),
// or pixels when src == nullptr.
bool commit(const Encoder& enc, const ulonglong2* src, const PixelInput* px, ulonglong2* rows,
            unsigned char* tree, cudaStream_t s);

// Merkle tree over `leaves` (a power of two) digests already stored at heap
// positions [leaves, 2 leaves) of `tree`: node k = SHA256(node 2k || node 2k + 1)
// (src/infrastructure/merkle_tree.cpp:64-83), root at 1.
bool build_tree(unsigned char* tree, long long leaves, cudaStream_t s);

// rows -> column-major codeword (the reference's encoded_codeword[c][r])
bool rows_to_columns(const ulonglong2* rows, long long cw_len, ulonglong2* cols, cudaStream_t s);

// Opening passes (orion_open.cu, src/VPD/linearPC.cpp:480-531,569-571) over the
// rows written by commit(): combined[t] = sum_j r0[j] rows[t][j] (t < cw_len);
// when tree != nullptr also the combined codeword's tree (leaves SHA256(x || 0^48),
// 2 * tree_leaves(col_len) digests).
bool combine(const ulonglong2* rows, long long col_len, long long cw_len, const ulonglong2* r0,
             ulonglong2* combined, unsigned char* tree, cudaStream_t s);
// out[i][.] = rows[q[i]][.] (the queried columns of the reference); synchronises
// to report indices outside [0, cw_len)
bool query_rows(const ulonglong2* rows, long long cw_len, const long long* q, int count, ulonglong2* out,
                cudaStream_t s);
// query_rows without the host round trip: bad rows give zeros and raise *bad
bool query_rows_async(const ulonglong2* rows, long long cw_len, const long long* q, int count, ulonglong2* out,
                      int* bad, cudaStream_t s);
// *out = sum_{i < n} r1[i] combined[i]
bool answer(const ulonglong2* combined, const ulonglong2* r1, long long n, ulonglong2* out, cudaStream_t s);

// The row-leaf chains of `count` rows of 128 elements (the commit's leaves)
// into digests[0 .. count) (32 bytes each).
bool leaf_digests(const ulonglong2* rows, long long count, unsigned char* digests, cudaStream_t s);

// Enc(msg) of one column (orion_verify.cu): out[0, cw_len) from msg[0, col_len)
// with the encoder's graphs, level by level as commit() does for 128 columns.
bool encode_vector(const Encoder& enc, const ulonglong2* msg, ulonglong2* out, cudaStream_t s);

// The verifier's per-query checks of an opening proof (orion_verify.cu): flags[i]
// bit 0 column sum != combined[q[i]], bit 1 commitment path, bit 2 combined
// path, bit 3 enc[q2[i]] != combined[q2[i]] (q2 may be null), 16 an index
// outside the codeword. Sibling lists sorted by node index.
bool verify_opening(long long msg_len, long long cw_len, const ulonglong2* r0, const long long* q,
                    const long long* q2, int count, const ulonglong2* cols, const ulonglong2* combined,
                    const ulonglong2* enc, const unsigned* com_idx, const unsigned char* com_dig, int n_com,
                    const unsigned* cmb_idx, const unsigned char* cmb_dig, int n_cmb, const unsigned char* com_root,
                    const unsigned char* cmb_root, int* flags, cudaStream_t s);

// `blocks` CTAs of 128 threads, each thread chaining `iters` SHA-256 of 64 bytes
// in registers (2 compressions each); XORs its last digest into *out
bool sha_peak(int blocks, int iters, uint32_t* out, cudaStream_t s);

// The row-leaf chains of later commits run as n launches of 64 / n column pairs
// each (n in 1, 2, 4, 8, 16; default 1): shorter launches release SMs sooner to
// kernels of other streams (latency of a serving loop's rounds), at the cost of
// n - 1 launches and 64 bytes per row of extra traffic. Same digests for any n.
bool set_leaf_chunks(int n);

// columns per lane (1, 2, 4; default 2) of the 61 x 31-bit gathers of graphs
// with 8192 targets or more: 4 warps, 2 or 1 per target; same codewords
bool set_gather_lanes(int columns_per_lane);

// launches issued by commit() / build_tree() on this thread since the last commit()
int last_launches();
// adds n to that count (entry points that run several commits)
void add_launches(int n);

}  // namespace orion
}  // namespace tp
