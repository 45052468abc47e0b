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

// Early-round session over a wire-major table V[w][c] of packed Fp2 (16 B).
struct EarlySession {
    int n_gates = 0, n_wires = 0;
    int n_copies = 0;      // logical copies (after a recorded fold)
    int n_phys = 0;        // copies held by buf[cur]
    int n_copies0 = 0;
    bool pending = false;  // fold recorded, applied by the next claim/fold/finish
    fp2 pending_r;
    fp2* buf[2] = {nullptr, nullptr};
    bool borrowed0 = false;
    fp2* beta[2] = {nullptr, nullptr};
    int cur = 0;
    DevGateForm form;
    ClaimWorkspace ws;
    fp2* fin = nullptr;    // finish staging [n_wires + 1]
    std::vector<fp2> L_host;  // the linear coefficients, kept for the constant wire
    cudaStream_t stream = nullptr;
    int launches = 0;      // kernels launched by this session
    int W_rows = 0;        // rows stored; rows >= W_rows are identically zero
    bool pix_mode = false; // the current table is the implicit table of a uint8 frame
    PixSrc px;
    fp2 Lc;                // L[const_idx] * const_val (pixel mode)
};

EarlySession* session_create(int n_gates, const int* type, const int* in0, const int* in1,
                             const u64* z_re, const u64* z_im, int n_copies, int n_wires,
                             cudaStream_t s);
// fill from host SoA tables (reference ABI)
bool session_load_host(EarlySession* S, const u64* v_re, const u64* v_im, const u64* b_re,
                       const u64* b_im);
// the table of a uint8 frame, read from device bytes (d_beta: packed, copied)
bool session_load_pixels(EarlySession* S, const PixSrc& px, const fp2* d_beta);
// fill from device packed tables; borrow=true adopts d_values as the first buffer
bool session_load_device(EarlySession* S, const fp2* d_values, const fp2* d_beta, bool borrow);
// claim; d_out8 receives the 4 Fp2 (0, 1, -1, 2) on device
bool session_claim_async(EarlySession* S, u64* d_out8);
bool session_claim(EarlySession* S, u64 out8[8]);
bool session_fold(EarlySession* S, fp2 r);
bool session_finish_async(EarlySession* S, fp2* d_wires, fp2* d_beta);
bool session_finish(EarlySession* S, u64* w_re, u64* w_im, u64* b_re, u64* b_im);
void session_destroy(EarlySession* S);

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
