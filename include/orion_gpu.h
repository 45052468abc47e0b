/*
 * Orion input-layer commitment, Fp2 NTT and Reed-Solomon commit on the GPU
 * (libnative_fp2_gpu.so).
 *
 * The reference runs these steps on the CPU inside its Orion binaries
 * (TruePix-main/Orion/Orion_nonzk, driven by examples/multivariate_PC_test_*.cpp
 * through `linearPC_multi_{commit,prove,open}`); a rebuilt driver calls the
 * entry points below instead. Field elements are 16 bytes in the reference's
 * memory order (u64 img, then u64 real; include/linear_gkr/prime_field.h),
 * canonical in [0, 2^61 - 1). Digests are 32 bytes exactly as __hhash_digest
 * stores them (the SHA-256 output bytes).
 *
 * Return value: 0 on success, -1 on failure with tp_last_error_code() /
 * tp_last_error() set (native_fp2.h). Host-buffer entry points run on the
 * library stream and return when their outputs are written; *_dev entry points
 * take device pointers and a cudaStream_t (NULL = the CUDA default stream) and
 * return once the work is queued.
 */
#ifndef TRUEPIX_B200_ORION_GPU_H
#define TRUEPIX_B200_ORION_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* encode_output_len(col_len): codeword length of one column
 * (include/linear_code/linear_code_encode.h:8-15 after expander_init(col_len),
 * include/linear_code/expanders.h:47-60). */
long long tp_orion_codeword_len(long long col_len);

/* Merkle leaves after padding for an N-element commit: the power of two >=
 * 2 * N / 128 (merkle_tree.cpp:30-32); the tree holds 2 * leaves digests. */
long long tp_orion_tree_leaves(long long N);

/* Replaces commit(src, N) (src/VPD/linearPC.cpp:97-197) with the encoder state of
 * expander_init(N / 128) drawn from glibc rand() in its unseeded state, as the
 * reference's drivers do. src: N elements, column c = src[c * N/128 ...].
 * tree_out: 2 * tp_orion_tree_leaves(N) digests, heap order (root at index 1,
 * index 0 zero) -- the array commit() returns. codeword_out: NULL, or
 * 128 * tp_orion_codeword_len(N/128) elements, column-major like the reference's
 * encoded_codeword[c][r] when set_retain_encoded_codeword(true). N % 128 == 0,
 * N / 128 <= 2^22. */
int tp_orion_commit(const uint64_t* src, long long N, unsigned char* tree_out, uint64_t* codeword_out);

/* Device form of tp_orion_commit. d_src: N elements, column-major as above.
 * d_rows: scratch and output, cw_len x 128 elements, ROW-major (row r holds
 * element r of every column). d_tree: 2 * tp_orion_tree_leaves(N) digests. */
int tp_orion_commit_dev(const void* d_src, long long N, void* d_rows, void* d_tree, void* stream);

/* Commit of a frame read from its uint8 bytes in TruePix's layout
 * (include/truepix/truepix_gkr.h:107-206: element copy * n_wires + wire is
 * pixel[copy * copy_size + wire] for wire < copy_size, const_val at const_idx,
 * zero elsewhere and for copies >= n_copies). N = n_copies_padded * n_wires.
 * No N-element input vector is materialised. */
int tp_orion_commit_pixels_dev(const void* d_pixels, int n_copies, int n_copies_padded, int copy_size,
                               int n_wires, int const_idx, uint64_t const_val, void* d_rows,
                               void* d_tree, void* stream);

/* No counterpart in the reference. The SHA-256 row-leaf chains of later commits
 * (of every kind) run as n launches of 64 / n column pairs each, n in {1, 2, 4,
 * 8, 16}, default 1 (process-wide). Shorter launches release SMs sooner to
 * kernels of other streams, e.g. the rounds a serving loop waits on; the
 * digests do not depend on n. 0, or -1 for another n. */
int tp_orion_set_leaf_chunks(int n);

/* No counterpart in the reference. The expander gathers of later commits
 * multiply 61 x 31 bits when every weight limb is below 2^31 (the reference's
 * weights are rand() % p per limb); for graphs of 8192 targets or more each
 * lane handles 1, 2 (default) or 4 of the 128 columns (4, 2 or 1 warps per
 * target). Process-wide; the codewords do not depend on it. 0, or -1 otherwise. */
int tp_orion_set_gather_lanes(int columns_per_lane);

/* Zero-knowledge commits (TruePix-main/Orion/Orion_zk). Replaces
 * commit_pair(masked, mask, N) of src/VPD/linearPC.cpp:253-460: two Orion
 * commits, each byte-identical to commit() of its polynomial, trees returned
 * (tree_masked, tree_mask: 2 * tp_orion_tree_leaves(N) digests each; roots at
 * digest 1). Host buffers, N elements {img, real} each, canonical. */
int tp_orion_commit_pair(const uint64_t* masked, const uint64_t* mask, long long N, unsigned char* tree_masked,
                         unsigned char* tree_mask);

/* The ZK commit of a frame from its bytes and the mask seed: the masked
 * polynomial (frame + mask) and the mask, as alloc_masked_from_seed /
 * alloc_mask_from_seed build them (include/truepix/truepix_gkr.h:286-384: the
 * mask is zero except at the private wires, wire < copy_size and copy <
 * n_copies, where the k-th one in flat order holds the (k+1)-th splitmix64
 * output of the seed mod 2^61 - 1), committed into two row-major codewords
 * and two trees as by tp_orion_commit_pixels_dev. Neither polynomial is
 * materialised. Replaces the commit phase of
 * examples/multivariate_PC_test_commit.cpp:280-340 (linearPC_multi_commit_zk). */
int tp_orion_commit_zk_pixels_dev(const void* d_pixels, int n_copies, int n_copies_padded, int copy_size,
                                  int n_wires, int const_idx, uint64_t const_val, uint64_t mask_seed,
                                  void* d_rows_masked, void* d_tree_masked, void* d_rows_mask, void* d_tree_mask,
                                  void* stream);

/* The polynomial a frame stands for, as N = n_copies_padded * n_wires base-field
 * values (u64, imaginary parts are zero): mask_mode 0 the frame
 * (truepix::load_coefs), 1 the masked polynomial, 2 the mask (as above). For
 * the MLE evaluations of the ZK opening (tp_mle_eval_base_dev on d_out). */
int tp_orion_pixel_vector_dev(const void* d_pixels, int n_copies, int n_copies_padded, int copy_size, int n_wires,
                              int const_idx, uint64_t const_val, uint64_t mask_seed, int mask_mode, void* d_out,
                              void* stream);

/* Prover-side passes of tensor_product_protocol (src/VPD/linearPC.cpp:480-531,
 * 569-571) over the ROW-major codeword d_rows that a commit above left on the
 * device. d_r0: 128 elements (the column weights r0). d_combined: cw_len
 * elements, combined_codeword (its first N/128 entries are combined_message).
 * d_ctree: NULL, or 2 * tp_orion_tree_leaves(N) digests: combined_codeword_mt,
 * leaves merkle_tree::hash_single_field_element(combined[i]) (zero element past
 * cw_len), root at 1. */
int tp_orion_combine_dev(const void* d_rows, long long N, const void* d_r0, void* d_combined, void* d_ctree,
                         void* stream);

/* queried_cols[i][j] = encoded_codeword[j][col_q[i]] for i < count: d_q holds
 * count int64 row indices (< cw_len, checked), d_out count * 128 elements.
 * Synchronises the stream. */
int tp_orion_query_columns_dev(const void* d_rows, long long N, const void* d_q, int count, void* d_out,
                               void* stream);
/* tp_orion_query_columns_dev without waiting for the device: an index outside
 * the codeword gives a zero column and sets *d_bad (device int, optional; the
 * caller clears it and reads it back later). Async on `stream`. */
int tp_orion_query_columns_async_dev(const void* d_rows, long long N, const void* d_q, int count, void* d_out,
                                     int* d_bad, void* stream);

/* answer = sum_{i < msg_len} r1[i] * combined_message[i] (linearPC.cpp:569-571);
 * d_answer: one element. */
int tp_orion_answer_dev(const void* d_combined, long long msg_len, const void* d_r1, void* d_answer,
                        void* stream);

/* Replaces encode(src, dst, n) of one message (include/linear_code/linear_code_encode.h:17-72)
 * with the graphs of expander_init(col_len): d_out (tp_orion_codeword_len(col_len)
 * elements) receives the codeword of d_msg (col_len elements). The EC(y1) step of
 * the opening (linearPC.cpp:585-605: the GKR circuit generate_circuit builds
 * computes this code at the queried positions). Async. */
int tp_orion_encode_dev(const void* d_msg, long long col_len, void* d_out, void* stream);

/* The per-query checks of verify_opening_proof (src/VPD/linearPC.cpp:733-879) on
 * the device, all queries at once: for i < count,
 *   d_flags[i] bit 0  sum_j r0[j] cols[i][j] != combined[q[i]]   (column linear combo)
 *              bit 1  the column's leaf chain does not reach com_root along the
 *                     commitment's sparse siblings (verify_claim_sparse,
 *                     src/truepix/orion_proof.cpp:176-200)
 *              bit 2  SHA256(combined[q[i]] || 0^48) does not reach comb_root
 *              bit 3  enc[q2[i]] != combined[q2[i]] (EC(y1); d_q2 may be NULL)
 *              16     an index outside [0, cw_len)
 * d_r0: 128 elements; d_q, d_q2: count int64; d_cols: count x 128 elements;
 * d_combined, d_enc: cw_len elements; sibling lists: n node indices (uint32,
 * ascending) and n 32-byte digests on the device; roots: 32 host bytes. msg_len a
 * power of two, cw_len = tp_orion_codeword_len(msg_len). Async. */
int tp_orion_verify_opening_dev(long long msg_len, long long cw_len, const void* d_r0, const void* d_q,
                                const void* d_q2, int count, const void* d_cols, const void* d_combined,
                                const void* d_enc, const void* d_com_idx, const void* d_com_nodes, int n_com,
                                const void* d_cmb_idx, const void* d_cmb_nodes, int n_cmb,
                                const unsigned char* com_root, const unsigned char* comb_root, int* d_flags,
                                void* stream);

/* Kernels launched by the calling thread's last commit (any of the three forms). */
int tp_orion_last_launches(void);

/* Row-major codeword (as written by the commits above) -> column-major
 * (encoded_codeword[c][r]); d_cols holds 128 * cw_len elements. */
int tp_orion_rows_to_columns_dev(const void* d_rows, long long cw_len, void* d_cols, void* stream);

/* Measurement entry point, no counterpart in the reference: the register-only
 * throughput of the library's SHA-256 code. blocks x 128 threads each chain
 * `iters` SHA-256 of a 64-byte message (2 compressions each) and XOR their last
 * digest word into *d_out (4 bytes, device). Used as the compute roof of the
 * Merkle leaf kernels. */
int tp_sha256_peak_dev(int blocks, int iters, void* d_out, void* stream);

/* ---- Fp2 NTT (src/infrastructure/RS_polynomial.cpp) ------------------------ */

/* Replaces fast_fourier_transform(coef, coef_len, order, root, result)
 * (RS_polynomial.cpp:46-130) with root = get_root_of_unity(log2 order)
 * (src/linear_gkr/prime_field.cpp:60-73): result[i] = P(w^i), i < order, for the
 * coef_len coefficients of P. Powers of two, coef_len <= order <= 2^28. */
int tp_fft(const uint64_t* coef, int coef_len, int order, uint64_t* result);

/* Replaces inverse_fast_fourier_transform(evals, coef_len, order, root, result)
 * (RS_polynomial.cpp:132-206): the coef_len coefficients whose values on the
 * coef_len-th roots of unity are evals[i * (order / coef_len)]. */
int tp_ifft(const uint64_t* evals, int coef_len, int order, uint64_t* result);

/* Device forms; `batch` transforms, transform b reading d_in + b * in_stride and
 * writing d_out + b * out_stride (strides in elements). d_in == d_out only for
 * batch 1. */
int tp_fft_dev(const void* d_coef, long long coef_len, long long order, void* d_out, int batch,
               long long in_stride, long long out_stride, void* stream);
int tp_ifft_dev(const void* d_evals, long long coef_len, long long order, void* d_out, int batch,
                long long in_stride, long long out_stride, void* stream);

/* Autotuner for the transforms above (no counterpart in the reference, whose
 * FFT is one fixed radix-2 loop): times every split of a 2^log_n-point transform
 * into shared-memory passes (radix 2^3 .. 2^10 each) on the current device, with
 * `batch` transforms per launch, and keeps the fastest for every later transform
 * of that size on that device. digits_out (3 ints) receives the chosen radix
 * bits per pass, *ms_out its time per batch. Returns the number of passes, or -1.
 * Allocates 3 * 2^log_n * batch elements while it runs. */
int tp_ntt_autotune(int log_n, int batch, int* digits_out, float* ms_out);

/* Replaces poly_commit_prover::commit_private_array(src, log_len)
 * (include/poly_commitment/poly_commit.h:42-96) together with the
 * fri::request_init_commit(log_len, 0) it ends in (src/VPD/fri.cpp:36-123):
 * Reed-Solomon code at rate 2^-5 over 64 slices and the Merkle tree of the
 * interleaved codeword. src: 2^log_len elements, 6 <= log_len <= 25.
 * l_eval_out: NULL or 2^(log_len+5) elements (poly_commit::l_eval, slice-major).
 * tree_out: 2^(log_len-1) digests (fri::witness_merkle[0]); the root (the
 * function's return value in the reference) is tree_out[1]. */
int tp_rs_commit(const uint64_t* src, int log_len, uint64_t* l_eval_out, unsigned char* tree_out);
int tp_rs_commit_dev(const void* d_src, int log_len, void* d_l_eval, void* d_tree, void* stream);

/* Replaces fri::commit_phase_step(r) (src/VPD/fri.cpp:316-420) for the steps
 * after the first oracle: d_witness holds the current witness in the
 * interleaved layout of request_init_commit, w[(k << 7) | (j << 1) | h] = slice
 * j's value at point k + h * M/2 (M = 2^log_m points per slice, 2 <= log_m <=
 * 26; the reference's rs_codeword[step - 1] with its mapping applied). d_next
 * (M/2 * 64 elements) receives the folded witness 2^-1((x + y) + w_M^-i r (x - y))
 * in the same layout (rs_codeword[step]); d_tree (M/2 digests) its Merkle tree
 * (merkle[step], root at 1). r canonical (real, imag). */
int tp_fri_commit_step_dev(const void* d_witness, int log_m, uint64_t r_real, uint64_t r_imag, void* d_next,
                           void* d_tree, void* stream);

/* ---- ./fft_gkr (src/VPD/fft_circuit_GKR.cpp) ---------------------------------
 * Replaces the program that poly_commit_verifier::verify_poly_commitment runs as
 * system("./fft_gkr <lg> log_fftgkr.txt") (src/VPD/vpd_verifier.cpp:80-89): the
 * GKR proof, with its verifier's checks, of the circuit build_circuit(lg)
 * (:22-112: tensor expansion of lg points, inverse FFT of size 2^lg, scaling,
 * 64 polynomial evaluations and their sums) over the sumcheck of engage_gkr
 * (:770-825). The prover runs on the device; the verifier's randomness is the
 * reference's (glibc rand() in its unseeded state, drawn in its order), so the
 * claims are the reference's. Outputs what main (:827-845) writes: v_time
 * (seconds of the closed-form layer checks), proof_size (bytes, the reference's
 * count) and p_time (seconds of the whole proof, checks included); *accepted = 1
 * when every check passed. trace_path: NULL, or a file receiving the layers (lg
 * <= 6), the claim after each layer group, the last sumcheck tables and the
 * result (the fixture format of tests/golden/gen_fft_gkr_golden.py). 0 <= lg <= 20. */
int tp_fft_gkr(int lg, double* v_time, long long* proof_size, double* p_time, int* accepted, const char* trace_path);

/* ---- Virgo (linear GKR) sumcheck (src/linear_gkr/prover.cpp) --------------- */

/* Replaces zk_prover::sumcheck_phase1_update and sumcheck_phase2_update
 * (prover.cpp:576-644, 935-1006; one computation): the tables V_mult_add,
 * addV_array, add_mult_sum (total_uv linear_poly entries {a, b} each, 32 bytes)
 * are folded with previous_random (or, for current_bit == 0, without it) into
 * d_*_out (total_uv / 2 entries each; the reference swaps them in), and d_ret gets
 * the returned quadratic_poly {a, b, c} (48 bytes). total_uv even and >= 2;
 * tables and previous_random canonical. */
int tp_virgo_sumcheck_update_dev(const void* d_vma, const void* d_addv, const void* d_ams, long long total_uv,
                                 uint64_t r_real, uint64_t r_imag, int current_bit, void* d_vma_out,
                                 void* d_addv_out, void* d_ams_out, void* d_ret, void* stream);

/* Layer inits of the Virgo sumcheck: zk_prover::sumcheck_phase1_init and
 * sumcheck_phase2_init (prover.cpp:246-570, 645-930) for layer
 * sumcheck_layer_id of a layered circuit. The layer is given once: 2^length_g
 * gates (ty[g], u[g], v[g] as in circuit_fast_track.h's gate; type-14 gates take
 * the (src, weight) pairs comb_src / comb_w[comb_ptr[g] .. comb_ptr[g + 1]),
 * weights {img, real}; comb_* may be NULL without type-14 gates) over a previous
 * layer of 2^length_u values. Indices outside the layer are rejected (NULL);
 * unknown gate types contribute nothing, as in the reference. */
void* tp_virgo_layer_create(int length_g, int length_u, const int* ty, const long long* u, const long long* v,
                            const int* comb_ptr, const int* comb_src, const uint64_t* comb_w);
void tp_virgo_layer_destroy(void* layer);

/* Phase 1: d_values = circuit_value[layer - 1] (2^length_u elements, device);
 * r0, r1: length_g host elements, alpha, beta: one each (sumcheck_init's
 * arguments). Writes the linear_poly tables V_mult_add, addV_array,
 * add_mult_sum (2^length_u entries of 32 bytes each, device) that
 * tp_virgo_sumcheck_update_dev folds. */
int tp_virgo_phase1_init_dev(void* layer, const void* d_values, const uint64_t* r0, const uint64_t* r1,
                             const uint64_t* alpha, const uint64_t* beta, void* d_vma, void* d_addv, void* d_ams,
                             void* stream);

/* Phase 2: as phase 1 plus d_vma0 (device: the one-entry V_mult_add that phase
 * 1's rounds leave, whose value at prev_r is v_u), prev_r (one host element)
 * and r_u (length_u host elements). */
int tp_virgo_phase2_init_dev(void* layer, const void* d_values, const uint64_t* r0, const uint64_t* r1,
                             const uint64_t* alpha, const uint64_t* beta, const void* d_vma0, const uint64_t* prev_r,
                             const uint64_t* r_u, void* d_vma, void* d_addv, void* d_ams, void* stream);

/* ---- opening helpers for a prover of many frames ----
 * eq(z, i) for i < 2^k, bit j of i <-> z_j (LSB first), as native_fp2_compute_beta
 * with init 1 (native_fp2_core.hpp:139-161) but on the host: z: k (re, im)
 * pairs, canonical; out: 2^k (re, im) pairs. The opening's column and row
 * weights (linearPC.cpp:693-731 dfs over the reversed point halves). k <= 26. */
int tp_eq_table_host(const uint64_t* z, int k, uint64_t* out);
/* collect_merkle_siblings (orion_proof.cpp:153-174): for each position in order,
 * the siblings on its path to the root (heap order, root 1) not listed before;
 * writes their node indices to out_nodes (cap entries) and returns how many
 * (-1 on bad arguments or when more than cap). */
int tp_orion_path_nodes(long long n_leaves, const long long* positions, int count, int* out_nodes, int cap);
/* The bytes of an opening proof file (OpeningProof::write_file, orion_proof.cpp:67-95):
 * "ORIONPV1", version 2, use_group1, N, the column size 128, msg_len, cw_len, the
 * query count; the answer; both roots; the queried column indices; the queried
 * columns (n_queries x 128 elements); the combined codeword (cw_len elements) and
 * its first msg_len again (the combined message); then per tree the node count and
 * (u32 index, 32-byte digest) per node. Elements are (img, real) u64 pairs. Writes
 * into out (cap bytes; tp_orion_opening_file_size tells how many) on the host and
 * returns the size, or -1. */
long long tp_orion_opening_file_size(long long msg_len, long long cw_len, int n_queries, int n_com_nodes,
                                     int n_comb_nodes);
long long tp_orion_opening_file(long long N, long long msg_len, long long cw_len, const uint64_t* answer,
                                const unsigned char* com_root, const unsigned char* comb_root, const long long* col_q,
                                int n_queries, const uint64_t* cols, const uint64_t* combined, const int* com_idx,
                                const unsigned char* com_nodes, int n_com_nodes, const int* comb_idx,
                                const unsigned char* comb_nodes, int n_comb_nodes, int use_group1, unsigned char* out,
                                long long cap);
/* d_out[i] = the 32-byte node d_nodes[i] of a heap-ordered tree of n_nodes_tree
 * digests (device; a node index outside the tree gives 32 zero bytes). Async. */
int tp_orion_gather_nodes_dev(const void* d_tree, long long n_nodes_tree, const void* d_nodes, int n, void* d_out,
                              void* stream);

#ifdef __cplusplus
}
#endif

#endif