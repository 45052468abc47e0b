// GKR input-layer sumcheck ("early rounds") and the batch Fp2 operations on
// one B200. Host-side interface used by the C ABI (native_fp2_abi.cu).
#pragma once
#include <cuda_runtime.h>

#include <vector>

#include "fp2.cuh"
#include "gkr_internal.cuh"

namespace tp {

// Every reference gate function (TruePix-main/native_fp2/native_fp2_core.hpp:32-51)
// is k0 + k1*x + k2*y + k3*x*y with small integer k. The per-layer sum
// sum_g z1[g]*gate_g(V[in0[g]], V[in1[g]]) is therefore
//   K0 + sum_w L[w]*V[w] + sum_terms c*V[a]*V[b]
// with L and the product terms fixed for the whole early phase.
struct GateForm {
    fp2 K0;
    std::vector<fp2> L;        // [n_wires]
    std::vector<int> ta, tb;   // product terms V[a]*V[b], grouped by b
    std::vector<fp2> tc;       // their coefficients
};
// Returns false (error set) when a used wire index is outside [0, n_wires).
bool build_gate_form(int n_gates, const int* type, const int* in0, const int* in1,
                     const u64* z_re, const u64* z_im, int n_wires, GateForm& out);

// Device copy of a GateForm.
struct DevGateForm {
    fp2 K0;
    fp2* L = nullptr;
    int2* ab = nullptr;
    fp2* c = nullptr;
    int n_terms = 0;
    int n_wires = 0;
};
bool upload_gate_form(const GateForm& g, DevGateForm& d, cudaStream_t s);
void free_gate_form(DevGateForm& d, cudaStream_t s);

// Reduction workspace for one claim launch: per-block partials + ticket + out8.
struct ClaimWorkspace {
    fp2* partials = nullptr;
    size_t cap_blocks = 0;
    unsigned* ticket = nullptr;   // zero between launches
    u64* out8 = nullptr;          // 8 x u64 on device
};
bool workspace_init(ClaimWorkspace& w, size_t blocks, cudaStream_t s);
void workspace_free(ClaimWorkspace& w, cudaStream_t s);

// One frame (early-round session) of a batch: its table source, ping-pong
// buffers, beta, gate form and round state.
struct Frame {
    int n_wires = 0, W_rows = 0;
    int n_copies0 = 0;     // copies of the input table (a power of two >= 2)
    int n_copies = 0;      // logical copies (after a recorded fold)
    int n_phys = 0;        // copies held by the current source
    int cur = 0;           // table buffer holding the current source
    bool pix_cur = false;  // the current source is the frame's bytes
    PixSrc px;
    bool pending = false;  // fold recorded, applied by the next claim / fold / finish
    fp2 r;
    const fp2* r_dev = nullptr;  // the pending fold's challenge in device memory (batch_fold_dev)
    DevGateForm form;
    std::vector<fp2> L_host;
    fp2 Lc;                // L[const_idx] * const_val (byte source)
    fp2* buf[2] = {nullptr, nullptr};
    bool borrowed0 = false;
    fp2* beta[2] = {nullptr, nullptr};
    fp2* fin = nullptr;    // [n_wires + 1]: wires, then beta
    u64* out8 = nullptr;   // default claim slot
    bool configured = false;
    size_t cap0 = 0, cap1 = 0, capb = 0, capfin = 0;  // element capacities kept across resets
};

// A batch of frames advanced together: one launch per round for all frames
// whose early rounds are not finished.
struct Batch {
    std::vector<Frame*> frames;
    cudaStream_t stream = nullptr;
    Job* d_jobs = nullptr;
    size_t cap_jobs = 0;
    fp2* partials = nullptr;
    size_t cap_partials = 0;  // in CTAs (4 fp2 each)
    unsigned* tickets = nullptr;
    size_t cap_tickets = 0;
    void* d_patch = nullptr;   // (job, device challenge) pairs patched into the job array
    size_t cap_patch = 0;
    int launches = 0;
    // the graph path (batch_vole_rounds_graph): every round's jobs in one device
    // table, uploaded from a pinned stage, and the captured graph of the rounds
    Job* d_table = nullptr;
    size_t cap_table = 0;
    void* d_ptable = nullptr;
    size_t cap_ptable = 0;
    void* h_stage = nullptr;
    size_t cap_stage = 0;
    cudaEvent_t staged = nullptr;     // the last upload from h_stage has completed
    cudaGraphExec_t graph = nullptr;
    std::vector<long long> graph_key;
    int graph_kernels = 0;
    int graph_replays = 0;
};

Batch* batch_create(int n_frames, cudaStream_t s);
// configure frame i (gate form from z1; tables from host SoA, device packed, or bytes)
bool batch_set_gates(Batch* B, int i, int n_gates, const int* type, const int* in0,
                     const int* in1, const u64* z_re, const u64* z_im, int n_copies, int n_wires);
bool batch_load_host(Batch* B, int i, const u64* v_re, const u64* v_im, const u64* b_re,
                     const u64* b_im);
bool batch_load_device(Batch* B, int i, const fp2* d_values, const fp2* d_beta, bool borrow);
bool batch_load_pixels(Batch* B, int i, const PixSrc& px, const fp2* d_beta);
// claims of all unfinished frames; d_claims[i] (8 u64, device) or the frame's slot
bool batch_claim(Batch* B, u64* const* d_claims);
bool batch_fold(Batch* B, int i, fp2 r);
// the same with the challenge in device memory (read in stream order when the
// next claim or finish is queued); needs a claim or finish before the next fold
bool batch_fold_dev(Batch* B, int i, const fp2* d_r);
// wires / beta of every frame into d_wires[i] (n_wires packed) / d_beta[i] (1 packed);
// nullptr destinations use the frame's own staging buffer
bool batch_finish(Batch* B, fp2* const* d_wires, fp2* const* d_beta);
// Every early round of a batch on device transcripts, as one CUDA graph: per
// round the claims (d_claims + 8 B k u64), the VOLE-committed round
// (tp_vole_round_dev: challenge d_chal + B k, proof d_proof + 5 B k, labels
// "sc-<layer>-<k>"), the fold by the drawn challenge; then the finish. All
// frames must have the same number of rounds. The jobs of all rounds are planned
// on the host and uploaded in one copy; the graph is captured on the first call
// of a shape and replayed while the shape and the buffers stay the same.
bool batch_vole_rounds_graph(Batch* B, u64* d_claims, void* d_states, void* d_vole_states, const fp2* d_u,
                             const fp2* d_v, long long count, int layer, fp2* d_chal, fp2* d_proof,
                             fp2* const* d_wires, fp2* const* d_beta);
// measure the claim / fold launch split per (round kind, work bucket) on the next
// immediate rounds (autotuner on / off), and the table of measured splits
void batch_tune_enable(bool on);
int batch_tune_table(int* kind, int* bucket, int* ctas_per_sm, int max);
bool batch_tune_set(int kind, int bucket, int ctas_per_sm);
// one frame: its wires / beta (nullptr: the frame's staging buffer), then its slot
// is free for a new frame (serving: frames join and leave between rounds)
bool batch_finish_frame(Batch* B, int i, fp2* d_wires, fp2* d_beta);
// free slot i without finishing; free_buffers also returns its tables to the pool
void batch_release(Batch* B, int i, bool free_buffers);
void batch_destroy(Batch* B);
// forget every frame's configuration but keep its device buffers for reuse
void batch_reset(Batch* B);

// single-frame views used by the reference ABI
Batch* session_create(int n_gates, const int* type, const int* in0, const int* in1,
                      const u64* z_re, const u64* z_im, int n_copies, int n_wires,
                      cudaStream_t s);
bool session_claim(Batch* B, u64 out8[8]);
bool session_finish(Batch* B, u64* w_re, u64* w_im, u64* b_re, u64* b_im);

// ---- batch operations on device buffers (all asynchronous on stream s) ----
bool launch_fold_soa(const u64* in_re, const u64* in_im, size_t n_out, fp2 r, u64* out_re,
                     u64* out_im, cudaStream_t s);
bool launch_fold_aos(const fp2* in, size_t n_out, fp2 r, fp2* out, cudaStream_t s);
bool launch_expand_soa(const u64* in_re, const u64* in_im, size_t n_src, size_t ncopies,
                       u64* out_re, u64* out_im, cudaStream_t s);
// Claim with caller-supplied -1/2 tables (SoA, reference batch semantics).
bool launch_claim_explicit(const DevGateForm& g, int n_copies, const u64* const* t12,
                           ClaimWorkspace& ws, cudaStream_t s);
// eq table: out[i] = init * prod_j (bit_j(i) ? z_j : 1 - z_j), SoA or packed
bool launch_beta(const fp2* d_z, int n_z, fp2 init, u64* out_re, u64* out_im, fp2* out_aos,
                 cudaStream_t s);
// The same MLE with caller-provided scratch: tabs (2^min(n_z,12) + 2^(n_z-12) Fp2),
// partials (max_blocks Fp2) and a zeroed ticket; launches at most max_blocks blocks.
bool launch_mle_base_into(const u64* d_in, const fp2* d_z, int n_z, fp2* d_out, fp2* tabs,
                          fp2* partials, unsigned* ticket, unsigned max_blocks, cudaStream_t s);
// MLE of base-field inputs (2^n_z u64) at the Fp2 point z -> d_out (1 fp2)
bool launch_mle_base(const u64* d_in, const fp2* d_z, int n_z, fp2* d_out, cudaStream_t s);
// uint8 frame (n_real copies x copy_size bytes, copy-major) -> packed wire-major
// table [W][n_pad] and/or copy-major base inputs [n_pad * W]; wire const_idx holds
// const_val, other wires and copies >= n_real are zero
// (TruePix-main/Orion/Orion_nonzk/include/truepix/truepix_gkr.h:11-18,157-196).
bool launch_table_from_pixels(const unsigned char* d_pix, int n_real, int n_pad, int copy_size,
                              int W, int const_idx, u64 const_val, fp2* d_table, u64* d_inputs,
                              cudaStream_t s);
// number of kernels launched by the last batch call (for launch accounting)
int last_launch_count();

}  // namespace tp
