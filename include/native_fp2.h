/*
 * libnative_fp2_gpu.so -- B200 (sm_100a) GKR Fp2 prover core, C ABI.
 *
 * Drop-in for the reference library loaded by
 * TruePix-main/libTruePix/native_fp2_bridge.py:116-183 from
 * TruePix-main/native_fp2/lib/. The first 14 declarations keep the reference
 * prototypes (TruePix-main/native_fp2/native_fp2.cpp:11-160,
 * TruePix-main/native_fp2/native_fp2.cu:824-1022) and meaning:
 *   - field p = 2^61 - 1, Fp2 = Fp[i]/(i^2+1), canonical limbs in [0, p);
 *   - host arrays are caller-owned SoA real[]/imag[]; inputs are consumed and
 *     outputs written before the call returns;
 *   - session handles are opaque and freed by native_fp2_early_destroy.
 * Differences: there is no host fallback. A void entry point that fails leaves
 * its outputs untouched and sets tp_last_error_code() != 0; session calls
 * return -1 / NULL as the reference does. Wire indices used by a gate must lie
 * in [0, n_wires) and challenges must be canonical, else the call fails.
 *
 * The tp_* entry points are extensions: error reporting and device-buffer
 * variants whose Fp2 buffers are packed {re, im} pairs of uint64 (16 bytes per
 * element, 16-byte aligned) in device memory, asynchronous on `stream`
 * (a cudaStream_t; NULL is the CUDA default stream).
 */
#ifndef TRUEPIX_NATIVE_FP2_H
#define TRUEPIX_NATIVE_FP2_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* native_fp2.cu:826-829 -- initialise; 0 = ok (also without a device) */
int native_fp2_init(void);
/* native_fp2.cu:831-834 -- 1 when a CUDA device is usable */
int native_fp2_cuda_available(void);

/* native_fp2.cu:836-848 (core.hpp:53-64): out[i] = in[2i] + r (in[2i+1] - in[2i]) */
void native_fp2_fold(const uint64_t* in_real, const uint64_t* in_imag, size_t n_out,
                     uint64_t r_real, uint64_t r_imag, uint64_t* out_real, uint64_t* out_imag);

/* native_fp2.cu:850-862 (core.hpp:66-80): out[i*ncopies + j] = in[i] */
void native_fp2_expand(const uint64_t* in_real, const uint64_t* in_imag, size_t n_src,
                       size_t ncopies, uint64_t* out_real, uint64_t* out_imag);

/* native_fp2.cu:864-893 (core.hpp:82-137): early-round claim at t = 0, 1, -1, 2 with
 * caller-supplied -1/2 tables; out8 = [re0, im0, re1, im1, re-1, im-1, re2, im2] */
void native_fp2_sumcheck_early(int n_gates, const int* gate_type, const int* in0, const int* in1,
                               const uint64_t* z1_real, const uint64_t* z1_imag, int n_copies,
                               int n_wires, const uint64_t* values_real,
                               const uint64_t* values_imag, const uint64_t* fact0_real,
                               const uint64_t* fact0_imag, const uint64_t* fact1_real,
                               const uint64_t* fact1_imag, const uint64_t* beta_real,
                               const uint64_t* beta_imag, const uint64_t* beta_f0_real,
                               const uint64_t* beta_f0_imag, const uint64_t* beta_f1_real,
                               const uint64_t* beta_f1_imag, uint64_t out8[8]);

/* native_fp2.cu:895-907 (core.hpp:139-161): out[i] = init * prod_j (bit_j(i) ? z_j : 1 - z_j) */
void native_fp2_compute_beta(const uint64_t* z_real, const uint64_t* z_imag, int n_z,
                             uint64_t init_real, uint64_t init_imag, uint64_t* out_real,
                             uint64_t* out_imag);

/* native_fp2.cu:909-921 (core.hpp:300-366): MLE of 2^n_z base-field inputs at z (LSB first) */
void native_fp2_mle_eval_base(const uint64_t* inputs, const uint64_t* z_real,
                              const uint64_t* z_imag, int n_z, uint64_t* out_real,
                              uint64_t* out_imag);

/* native_fp2.cu:923-952 (core.hpp:173-198): resident early-round session; NULL on failure.
 * values: n_wires x n_copies, wire-major; n_copies a power of two >= 2. */
void* native_fp2_early_create(int n_gates, const int* gate_type, const int* in0, const int* in1,
                              const uint64_t* z1_real, const uint64_t* z1_imag, int n_copies,
                              int n_wires, const uint64_t* values_real,
                              const uint64_t* values_imag, const uint64_t* beta_real,
                              const uint64_t* beta_imag);
/* native_fp2.cu:954-963 (core.hpp:200-248): claim of the current round; 0 ok, -1 error */
int native_fp2_early_claim(void* handle, uint64_t out8[8]);
/* native_fp2.cu:965-974 (core.hpp:250-279): fold every wire and beta by r; 0 ok, -1 error */
int native_fp2_early_fold(void* handle, uint64_t r_real, uint64_t r_imag);
/* native_fp2.cu:976-989 (core.hpp:281-296): wire[w] = V[w][0], beta = beta[0] */
int native_fp2_early_finish(void* handle, uint64_t* wire_real, uint64_t* wire_imag,
                            uint64_t* beta_real, uint64_t* beta_imag);
/* native_fp2.cu:991-1005 */
int native_fp2_early_n_copies(void* handle);
int native_fp2_early_n_wires(void* handle);
/* native_fp2.cu:1007-1020 */
void native_fp2_early_destroy(void* handle);

/* ---- extensions (no counterpart in the reference) ---- */

/* error state of the calling thread: 0 = ok; text describes the last failure */
int tp_last_error_code(void);
const char* tp_last_error(void);
void tp_clear_error(void);
/* kernels launched by the last batch entry point */
int tp_last_launch_count(void);

/* Host-only: the per-layer linear form the claim kernels use,
 *   sum_g z1[g] gate_g(V[in0], V[in1]) = K0 + sum_w L[w] V[w] + sum_t c_t V[a_t] V[b_t].
 * Writes k0[2], lin[2*n_wires] (re, im pairs) and up to max_terms product terms
 * (term_ab[2i] = a, term_ab[2i+1] = b, term_c[2i..2i+1] = c); returns the number of
 * terms, or -1 on a bad wire index. Needs no GPU. */
int tp_gate_form(int n_gates, const int* gate_type, const int* in0, const int* in1,
                 const uint64_t* z1_real, const uint64_t* z1_imag, int n_wires, uint64_t* k0,
                 uint64_t* lin, int max_terms, int* term_ab, uint64_t* term_c);

/* Session over a packed device table d_values (n_wires x n_copies Fp2) and packed
 * d_beta (n_copies Fp2). borrow != 0 adopts d_values as working storage (the caller
 * keeps it alive until destroy; its contents are overwritten); otherwise it is copied. */
void* tp_early_create_dev(int n_gates, const int* gate_type, const int* in0, const int* in1,
                          const uint64_t* z1_real, const uint64_t* z1_imag, int n_copies,
                          int n_wires, const void* d_values, const void* d_beta, int borrow,
                          void* stream);
/* claim into 8 x uint64 of device memory, without synchronising */
int tp_early_claim_dev(void* handle, void* d_out8);
/* wires into n_wires packed Fp2 and beta[0] into one packed Fp2, device memory, async */
int tp_early_finish_dev(void* handle, void* d_wires, void* d_beta);
/* kernels launched so far by a session */
int tp_early_launches(void* handle);

/* packed-buffer variants of fold / compute_beta / mle_eval_base (asynchronous) */
int tp_fold_dev(const void* d_in, size_t n_out, uint64_t r_real, uint64_t r_imag, void* d_out,
                void* stream);
int tp_compute_beta_dev(const void* d_z, int n_z, uint64_t init_real, uint64_t init_imag,
                        void* d_out, void* stream);
int tp_mle_eval_base_dev(const void* d_inputs, const void* d_z, int n_z, void* d_out,
                         void* stream);

/* Input layer from a uint8 frame: n_copies rows of copy_size bytes (copy-major)
 * -> d_table, the packed wire-major table [n_wires][n_copies_padded] used by the
 * early session, and/or d_inputs, the copy-major base-field vector
 * x[c * n_wires + w] used by mle_eval_base (either may be NULL). Wire const_idx
 * holds const_val (const_idx < 0: none); other wires and padded copies are zero.
 * Layout of TruePix-main/Orion/Orion_nonzk/include/truepix/truepix_gkr.h:11-18
 * (copy-major-384-const128-pad512-v1). Asynchronous. */
int tp_table_from_pixels(const void* d_pixels, int n_copies, int n_copies_padded, int copy_size,
                         int n_wires, int const_idx, uint64_t const_val, void* d_table,
                         void* d_inputs, void* stream);

/* Early session whose input table is the implicit table of a uint8 frame in
 * device memory (the layout of tp_table_from_pixels), read directly from the
 * bytes: the first claim and the first fold never materialise the
 * n_wires x n_copies_padded Fp2 table, and only rows [0, copy_size) and the
 * constant row are stored afterwards (the other wires are zero). d_beta: packed
 * Fp2 [n_copies_padded] (copied). Claims, folds, finish and destroy as for any
 * session; the pixels must stay unchanged until the first fold has run. */
void* tp_early_create_pixels(int n_gates, const int* gate_type, const int* in0, const int* in1,
                             const uint64_t* z1_real, const uint64_t* z1_imag,
                             const void* d_pixels, int n_copies, int n_copies_padded,
                             int copy_size, int n_wires, int const_idx, uint64_t const_val,
                             const void* d_beta, void* stream);
/* mle_eval_base of the copy-major input vector of that frame (x[c * n_wires + w])
 * at the packed Fp2 point d_z (log2(n_wires) + log2(n_copies_padded) coordinates,
 * LSB first), computed from the bytes. n_wires <= 512, powers of two. Async. */
int tp_mle_eval_pixels(const void* d_pixels, int n_copies, int n_copies_padded, int copy_size,
                       int n_wires, int const_idx, uint64_t const_val, const void* d_z,
                       void* d_out, void* stream);

/* n_rounds x (claim into d_claims[8k..8k+7] on the device, fold by challenges[2k],
 * challenges[2k+1]) without returning to the caller in between: for callers that
 * already hold the challenges (replay, benchmarking). Asynchronous. */
int tp_early_rounds_dev(void* handle, int n_rounds, const uint64_t* challenges, void* d_claims);

/* ---- batches: one kernel launch per round for many frames ----
 * A batch holds n_frames independent early sessions (own table, beta, gate
 * weights z1, challenges; sizes may differ). tp_batch_claim evaluates the claim
 * of every frame that still has at least 2 copies, with one launch per source
 * kind present; frames whose early rounds are over are skipped and their claim
 * slots left untouched. Asynchronous on the batch's stream. */
void* tp_batch_create(int n_frames, void* stream);
/* frame i from a uint8 frame in device memory (layout of tp_table_from_pixels) */
int tp_batch_set_pixels(void* batch, int i, int n_gates, const int* gate_type, const int* in0,
                        const int* in1, const uint64_t* z1_real, const uint64_t* z1_imag,
                        const void* d_pixels, int n_copies, int n_copies_padded, int copy_size,
                        int n_wires, int const_idx, uint64_t const_val, const void* d_beta);
/* frame i from a packed device table (borrow as in tp_early_create_dev) */
int tp_batch_set_table(void* batch, int i, int n_gates, const int* gate_type, const int* in0,
                       const int* in1, const uint64_t* z1_real, const uint64_t* z1_imag,
                       int n_copies, int n_wires, const void* d_values, const void* d_beta,
                       int borrow);
/* claims into d_claims[8 * i .. 8 * i + 7] (device, u64) */
int tp_batch_claim(void* batch, void* d_claims);
/* fold every frame that has >= 2 copies by (challenges[2i], challenges[2i+1]) (host array) */
int tp_batch_fold(void* batch, const uint64_t* challenges);
/* tp_batch_fold with the challenges in device memory (n_frames packed {re, im}
 * Fp2, canonical, e.g. drawn by tp_fs_rand_ext_dev): they are read in stream
 * order when the next tp_batch_claim / tp_batch_finish is queued on the batch's
 * stream, so they must be written before that point in stream order and stay
 * unchanged until it. Every frame needs a claim or a finish before its next
 * fold. No host round trip between rounds. */
int tp_batch_fold_dev(void* batch, const void* d_challenges);
int tp_batch_n_copies(void* batch, int i);
/* d_wires: frame i at d_wires + 16 * (sum of n_wires of frames < i) bytes -- with equal
 * n_wires simply [n_frames][n_wires] packed Fp2; d_beta: [n_frames] packed Fp2 */
int tp_batch_finish(void* batch, void* d_wires, void* d_beta);
/* Every early round of the batch on device transcripts, as one CUDA graph (no
 * counterpart in the reference, whose session returns to the host every round,
 * native_fp2.cu:676-812): per
 * round k the claims of all frames (d_claims + 64 B k bytes, 8 u64 per frame),
 * tp_vole_round_dev's VOLE-committed round on the frames' transcripts and VOLE
 * states (label "sc-<layer>-<k>", challenges d_challenges + 16 B k bytes, proof
 * elements d_proof + 80 B k bytes or NULL), the fold by the drawn challenge;
 * then tp_batch_finish into d_wires / d_beta. Frames of different sizes leave
 * the loop after their own last round (their claims, challenges and proof
 * elements of later rounds are not written); the batch's stream must be a
 * stream of the caller's (capture). The
 * rounds' jobs are planned on the host and uploaded in one copy; the graph is
 * captured on the first call and replayed while the shape and the buffers stay
 * the same (tp_batch_graph_replays counts the launches of a graph). */
int tp_batch_vole_rounds_graph(void* batch, void* d_claims, void* d_fs_states, void* d_vole_states, const void* d_u,
                               const void* d_v, long long count, int layer, void* d_challenges, void* d_proof,
                               void* d_wires, void* d_beta);
int tp_batch_graph_replays(void* batch);
/* Autotuner of the round launches (no counterpart in the reference): with it on,
 * the first immediate claim launch of each (round kind, work bucket) is timed
 * under several splits of its CTAs over the frames' pair tiles and row groups
 * (2 to 16 CTAs per SM) and the fastest is kept for this device; launches of a
 * bucket not yet measured use 4 per SM. tp_batch_tune_table lists the measured
 * entries (returns their count), tp_batch_tune_set installs one (e.g. from a
 * saved table). Kinds: 0 table claim, 1 table fold + claim, 2 byte claim, 3 byte
 * fold + claim; bucket = floor(log2 of the launch's pairs x rows). */
int tp_batch_autotune(int on);
int tp_batch_tune_table(int* kind, int* bucket, int* ctas_per_sm, int max);
int tp_batch_tune_set(int kind, int bucket, int ctas_per_sm);
/* Serving: frames join and leave a running batch between rounds. Finish frame i
 * alone (its n_wires wires into d_wires, its beta into d_beta; NULL = the frame's
 * staging buffer), then free its slot for tp_batch_set_* of a new frame while the
 * others continue. tp_batch_release frees slot i without finishing; with
 * free_buffers its tables go back to the pool (admission by HBM footprint). */
int tp_batch_finish_frame(void* batch, int i, void* d_wires, void* d_beta);
void tp_batch_release(void* batch, int i, int free_buffers);
int tp_batch_launches(void* batch);
/* forget every frame's configuration (tp_batch_set_* may be called again) while
 * keeping the device buffers for the next batch of the same or smaller sizes */
void tp_batch_reset(void* batch);
void tp_batch_destroy(void* batch);

/* beta tables of n_frames frames in one pass: d_z packed Fp2 [n_frames][n_z],
 * d_out packed Fp2 [n_frames][2^n_z] (compute_beta with init 1). Async. */
int tp_compute_beta_batch_dev(const void* d_z, int n_z, int n_frames, void* d_out, void* stream);
/* tp_mle_eval_pixels for n_frames frames of one padded size in one pass:
 * d_pixels / n_copies host arrays [n_frames]; d_points packed Fp2
 * [n_frames][log2 n_wires + log2 n_copies_padded]; d_out packed Fp2 [n_frames]. */
int tp_mle_eval_pixels_batch(int n_frames, const void* const* d_pixels, const int* n_copies,
                             int n_copies_padded, int copy_size, int n_wires, int const_idx,
                             uint64_t const_val, const void* d_points, void* d_out, void* stream);

/* Claim-kernel timer: when enabled, every session claim records a CUDA event pair
 * with tag 1000*(reads pixels) + 100*(fold fused) + log2(copies claimed).
 * tp_timer_read (after a synchronise) returns the number of pairs and their ms. */
int tp_timer_enable(int max_pairs);
void tp_timer_disable(void);
void tp_timer_reset(void);
int tp_timer_read(float* ms, int* tags, int max_pairs);

/* ---- late rounds and line projection of the input layer ----
 * Replaces the reference's Python late rounds, LayerProver.compute_outputs /
 * next_round for rounds nCopyBits..nCopyBits + 2n - 1 (libTruePix/layerprover.py
 * :231-290, gateprover.py:105-185, layercompute.py:16-150) and the final
 * LayerComputeH output (layercompute.py:152-247), for n_frames frames in one
 * launch (one CTA each). Per frame, from the early phase's results: d_wires
 * [n_frames][2^n_in_bits] packed Fp2 (tp_batch_finish's wires), d_beta
 * [n_frames] (its beta); d_gate_weights: the gates' z1 eq values, [n_frames]
 * [n_gates] packed Fp2 with weights_per_frame = 1, or one [n_gates] vector for
 * all frames with 0. Gate tables in host memory (n_gates <= 768, n_in_bits <= 9).
 * Challenges, one of:
 *   d_challenges [n_frames][2 n_in_bits] given (the other transcript arguments NULL);
 *   d_challenges NULL: each round is the reference's VOLE-committed round
 *     (circuitnizkvec_vole.py:396-418) on the round's three coefficients, with
 *     the frame's transcript d_fs_states[i] (tp_fs_state_bytes() each), VOLE
 *     state d_vole_states[i] (tp_vole_state_bytes() each, continuing from the
 *     early rounds) and correlations d_u / d_v [n_frames][count] packed Fp2, the
 *     challenge rand_ext("sc-<layer>-<round0 + round>"); the states are updated
 *     in place. A frame whose correlations run out stops (VOLE state bad = 1).
 * Outputs: d_coefs [n_frames][2 n_in_bits][3] (util.interpolate_quadratic of
 * the values at 0, 1, -1), d_line [n_frames][n_in_bits + 1] (coefficients,
 * constant first, of the input values on the line w1 + t (w2 - w1): the
 * project_line output the layer's final proof commits), d_challenges_out
 * [n_frames][2 n_in_bits], d_proof (VOLE mode, optional) [n_frames][2 n_in_bits]
 * [4] (three commitments d, the equality value).
 * The layer's closing proofs (VOLE mode, d_closing not NULL), circuitnizkvec_vole.py
 * :433-500 for a one-layer circuit: create_final_prod_pok on the line's
 * coefficients, the wiring predicates' multilinear extensions times the committed
 * gate values (CircuitVerifier.eval_mlext with GateFunctionsPC) and beta's factor
 * from d_z2 [n_frames][round0] (the copy part of the layer's point) and the early
 * challenges d_w3 (frame i, round k at d_w3[i * w3_frame_stride + k *
 * w3_round_stride], packed Fp2 elements), the equality proof, tau =
 * rand_ext("tau-<layer>"), create_pok_final, put(["gkr_input_point", point]),
 * create_input_value_proof. Outputs: d_closing [n_frames][n_in_bits + 10] (the
 * Fp2 values in the order they are put: d of the first coefficient and of the
 * product, d of the other coefficients, the two proof-of-knowledge values, the
 * two product-proof values, the equality value, the two final proof-of-knowledge
 * values, the input value proof), d_point [n_frames][n_in_bits + round0] (the
 * input point: the line at tau, then the early challenges), d_tag [n_frames] (its
 * tag). zk != 0: the zero-knowledge prover's closing (circuitnizkvec_vole_ZK.py
 * :188-247, TruePix's default), whose product proof adds three mask commitments
 * of 1 after the proof-of-knowledge values and the masks' product proof after its
 * own: d_closing then holds n_in_bits + 15 values per frame. round0 is the number
 * of early rounds (<= 64). Asynchronous on `stream`. */
int tp_late_rounds_dev(int n_frames, int n_in_bits, int n_gates, const int* gate_type, const int* in0,
                       const int* in1, const void* d_wires, const void* d_beta, const void* d_gate_weights,
                       int weights_per_frame, const void* d_challenges, void* d_fs_states, void* d_vole_states,
                       const void* d_u, const void* d_v, long long count, int layer, int round0, void* d_coefs,
                       void* d_line, void* d_challenges_out, void* d_proof, const void* d_z2, const void* d_w3,
                       long long w3_frame_stride, long long w3_round_stride, void* d_closing, void* d_point,
                       void* d_tag, int zk, void* stream);

/* ---- the Orion opening's transcript ----
 * The queried columns of the Orion NIZK opening (Orion_nonzk / Orion_zk
 * src/VPD/linearPC.cpp tensor_product_protocol with the transcript of
 * src/truepix/orion_fs.cpp): a fresh transcript absorbs "tensor-open", the
 * commitment's root (32 bytes), N and use_group1 (u64), then r0 and r1 field by
 * field (each element's real, then its imaginary part, 8 bytes each); then count
 * indices are drawn: uniform in [0, cw_len) (group -1, the plain opening), or
 * the even (group 0, the masked polynomial) or odd (group 1, the mask) columns of
 * the zero-knowledge opening. r0, r1: (real, imag) u64 pairs. Host only. */
int tp_orion_open_queries(const unsigned char* root32, uint64_t N, int use_group1, const uint64_t* r0, int n_r0,
                          const uint64_t* r1, long long n_r1, long long cw_len, int group, int count,
                          long long* col_q);
/* The same draws followed by the opening's second batch: ec_q receives the next
 * count indices, uniform in [0, cw_len) in both modes (the positions at which
 * the EC(y1) step checks the code of the combined message, linearPC.cpp:573-575
 * in Orion_nonzk, :879-880 in Orion_zk). ec_q may be NULL. Host only. */
int tp_orion_open_queries2(const unsigned char* root32, uint64_t N, int use_group1, const uint64_t* r0, int n_r0,
                           const uint64_t* r1, long long n_r1, long long cw_len, int group, int count,
                           long long* col_q, long long* ec_q);
/* No counterpart in the reference (its prover opens one polynomial per
 * process). n (<= 64) independent opening transcripts, each as
 * tp_orion_open_queries2 with its own root, use_group1, r0, r1, group and
 * outputs (arrays of n pointers; the sizes are shared), hashed in lockstep: 16
 * (then 8) at a time in the lanes of an AVX-512 multi-buffer SHA-256 where the
 * host has AVX-512, the rest in pairs on the x86 SHA extensions. The draws of
 * each equal tp_orion_open_queries2's for the same arguments. Host only. */
int tp_orion_open_queries_multi(int n, const unsigned char* const* roots, uint64_t N, const int* use_group1,
                                const uint64_t* const* r0, int n_r0, const uint64_t* const* r1, long long n_r1,
                                long long cw_len, const int* groups, int count, long long* const* col_q,
                                long long* const* ec_q);

/* ---- circuit evaluation: the prover's output vector ----
 * Replaces ArithCircuitIncrementalBuilder.run (libTruePix/arithcircuitbuilder.py:71-108,
 * arithcircuit.py:121-131, 172-181) as called by CircuitProver.set_inputs
 * (circuitprover.py:82-98) for the one-layer TruePix circuits, and the output
 * vector circuitnizkvec_vole.py:351-355 puts into the transcript: for each real
 * copy c the values of gates 0..n_gates-1 on the copy's inputs, at
 * d_out[c << out_bits + g] with out_bits = tp_circuit_out_bits(n_gates) =
 * ceil(log2 n_gates); every other element (a copy's padding outputs, the copies
 * n_copies..n_copies_padded-1) is zero. u64, canonical mod 2^61 - 1; the bytes
 * of the array are the LE64 encoding the transcript absorbs (tp_fs_put_u64s).
 * Inputs in the layout of tp_table_from_pixels (d_pixels: n_copies * copy_size
 * bytes, constant wire const_idx, -1 for none). Gate values as in
 * native_fp2_core.hpp:32-51 (types 0..12). n_gates <= 960, n_wires <= 16384;
 * gate tables in host memory (copied into the launch). d_out: n_copies_padded
 * << out_bits u64. Asynchronous on `stream`. */
int tp_circuit_out_bits(int n_gates);
int tp_circuit_outputs_pixels_dev(const void* d_pixels, int n_copies, int n_copies_padded, int copy_size,
                                  int n_wires, int const_idx, uint64_t const_val, int n_gates,
                                  const int* gate_type, const int* in0, const int* in1, void* d_out,
                                  void* stream);

/* No counterpart in the reference. tp_mle_eval_base_dev for callers that cannot
 * allocate device memory (their GPU memory belongs to another allocator, or a
 * time-critical loop cannot afford cudaMalloc/cudaFree): it calls no allocator
 * and uses a fixed 339 KB scratch array compiled into the library, which every
 * GPU that loads the library keeps until exit. Inputs up to 2^26 base-field
 * values (n_z <= 26); larger n_z is rejected with an error (-1). All calls share
 * the scratch: calls that overlap on the GPU race, order them. The first call
 * on a device looks up the scratch's device address; make it before any stream
 * capture. d_inputs: 2^n_z u64; d_z: n_z packed Fp2; d_out: 1 packed Fp2. Async. */
int tp_mle_eval_base_noalloc(const void* d_inputs, const void* d_z, int n_z, void* d_out,
                             void* stream);

/* ---- Fiat-Shamir transcript (TruePix-main/libTruePix/fiatshamir.py) ----------
 * The reference prover's transcript in its binary format: one running SHA-256
 * over everything put, challenges drawn from digests of the running state. A
 * state is tp_fs_state_bytes() (= 120) bytes of caller memory, host or device; it
 * moves between the two by a plain copy (cudaMemcpy), so a transcript begun on
 * the host (the circuit's IO, the commitment roots) continues on the device.
 * Host calls take one state in host memory; *_dev calls take n states in device
 * memory, one per frame, and are asynchronous on `stream`. */
int tp_fs_state_bytes(void);
/* FiatShamir(q, protocol).__init__ (fiatshamir.py:27-74) for q = 2^61 - 1 */
int tp_fs_init(void* state, const char* protocol);
/* absorb raw bytes already in the transcript's encoding (fiatshamir.py:101-138:
 * e.g. 0x02 || LE64 for an int inside a mixed list, 0x05 for None) */
int tp_fs_absorb(void* state, const void* bytes, size_t n);
/* put(list of ints < 2^64): the array('Q') path (fiatshamir.py:112-120) */
int tp_fs_put_u64s(void* state, const uint64_t* values, size_t n);
/* For each of n_frames transcripts (host memory): put(the frame's circuit output
 * vector) as a list of ints, the bytes tp_fs_put_u64s absorbs for the vector
 * tp_circuit_outputs_pixels_dev writes (circuitnizkvec_vole.py:351-355), computed
 * on the host copy by copy from the frame's bytes (pixels[f]: n_copies *
 * copy_size bytes in host memory, of which the first n_bytes are read: past them
 * the inputs are zero, as in a frame whose last copy is not full) and hashed as
 * it is made; frames whose
 * transcripts stand at the same offset are hashed together, up to 16 at a time
 * (the lanes of an AVX-512 multi-buffer SHA-256 where the host has AVX-512, else
 * lockstep pairs on the SHA extensions): pass 16 frames per call for the best
 * host throughput, 2 for the lowest latency. The vector itself (2^23 values at
 * 1080p) is never stored. Arguments as for
 * tp_circuit_outputs_pixels_dev; n_gates <= 4096. */
int tp_fs_put_circuit_outputs_pixels(void* const* states, const void* const* pixels, long long n_bytes, int n_frames,
                                     int n_copies, int n_copies_padded, int copy_size, int n_wires, int const_idx,
                                     uint64_t const_val, int n_gates, const int* gate_type, const int* in0,
                                     const int* in1);
/* No counterpart in the reference: 1 when this host hashes groups of frames
 * with the AVX-512 multi-buffer SHA-256 (CPU and OS support AVX-512 F/BW/VL),
 * else 0. Host only. */
int tp_host_sha_mb_available(void);
/* put(Fp2) for each (re[i], im[i]) in turn (fiatshamir.py:129-131) */
int tp_fs_put_fp2s(void* state, const uint64_t* re, const uint64_t* im, size_t n);
/* put(str) (fiatshamir.py:132-136) */
int tp_fs_put_str(void* state, const char* str);
/* rand_scalar() (fiatshamir.py:141-148) */
int tp_fs_rand_scalar(void* state, uint64_t* out);
/* rand_ext(label) (fiatshamir.py:150-162); labels up to 64 bytes */
int tp_fs_rand_ext(void* state, const char* label, uint64_t* re, uint64_t* im);
/* hash.digest() of the running state (32 bytes; the state is unchanged) */
int tp_fs_digest(const void* state, unsigned char* out32);
/* state i puts the k Fp2 d_values[i * k .. i * k + k) (packed {re, im} u64 pairs,
 * e.g. a frame's four round claims) */
int tp_fs_put_fp2s_dev(void* d_states, int n, const void* d_values, int k, void* stream);
/* state i draws rand_ext(label) into d_out[i] (packed {re, im}) */
int tp_fs_rand_ext_dev(void* d_states, int n, const char* label, void* d_out, void* stream);

/* One VOLE-committed sumcheck round per frame, as the reference prover's round
 * loop does it (circuitnizkvec_vole.py:396-418 with create_pok_temp :113-128 and
 * create_eq_proof :220-234): the round polynomial's coefficients from the four
 * claims at (0, 1, -1, 2) (util.interpolate_cubic), each committed with the next
 * VOLE correlation (ExtVOLECommit.commit: d = c - u put into the transcript, tag
 * v kept), the equality proof of the tags at 0 + 1 against the previous round's
 * value (rand_ext("eq"), est_eq / est_val put), the fold challenge
 * rand_ext(label) into d_chal[i], and the next previous value (the tags'
 * polynomial at the challenge). Frame i's correlations: d_u / d_v[i * count ..
 * (i + 1) * count) (packed {re, im}, the prover's u and v, one repetition). A
 * VOLE state (tp_vole_state_bytes() = 160 bytes, device) per frame holds the
 * next correlation index, the previous value and the running sums of tags and
 * coefficients; a frame whose correlations run out is marked (its `bad` word)
 * and left unchanged. d_proof (optional): per frame the four d and the equality
 * value (5 packed Fp2), the round's proof elements. */
int tp_vole_state_bytes(void);
/* host: a fresh VOLE state (prev NULL: no previous value, the first round of a proof) */
int tp_vole_state_init(void* state, uint64_t first_correlation, const uint64_t* prev);
int tp_vole_round_dev(void* d_fs_states, void* d_vole_states, int n, const void* d_claims, const void* d_u,
                      const void* d_v, long long count, const char* label, void* d_chal, void* d_proof,
                      void* stream);
/* The same round for frames each at its own round (a serving loop's slots; no
 * counterpart in the reference, which proves one frame per process): d_meta[i]
 * = {round, rounds} as two ints (round < 0: slot idle); slot i's claims at
 * d_claims + 64 i bytes, correlations u / v at + 16 count i, label
 * "sc-<layer>-<round>"; its challenge to d_chal_cur[i] and d_chal_hist[i *
 * max_rounds + round], proof elements (optional) at d_proof + 80 (i * max_rounds
 * + round) bytes; then round + 1, or -1 after the last round. Async. */
int tp_vole_round_slots_dev(void* d_fs_states, void* d_vole_states, int n_slots, void* d_meta, const void* d_claims,
                            const void* d_u, const void* d_v, long long count, int layer, void* d_chal_cur,
                            void* d_chal_hist, void* d_proof, int max_rounds, void* stream);

#ifdef __cplusplus
}
#endif
#endif
