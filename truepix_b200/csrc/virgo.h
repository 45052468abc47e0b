// Virgo (linear GKR) sumcheck round on the device -- see virgo.cu.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "fp2.cuh"

namespace tp {
namespace virgo {

// One sumcheck_phase{1,2}_update over tables of n linear_poly entries (n even):
// folded tables (n / 2 entries) into *_out, round polynomial {a, b, c} into ret
// (three {img, real} elements). r canonical; inputs canonical.
bool update(const ulonglong2* vma, const ulonglong2* addv, const ulonglong2* ams, long long n, fp2 r, int bit,
            ulonglong2* vma_out, ulonglong2* addv_out, ulonglong2* ams_out, ulonglong2* ret, cudaStream_t s);

// A layer of the layered circuit for the inits (prover.cpp:246-570, 645-930):
// the gates' (u, v) and, grouped by the table entry they add to, the terms of
// phase 1 (all gate kinds), of phase 2 (plain gates, by v) and of phase 2's
// addV_array[0] sum (sum, exp-sum, custom-comb gates). A term is a gate, its
// type and k: the offset into a gate's range (types 5, 12) or the index of a
// custom-comb (src, weight) pair (type 14).
struct Term {
    int gate, type, k;
};

struct Layer {
    int length_g = 0, length_u = 0;
    long long n_gates = 0, total_uv = 0, n_p2s = 0;
    long long* d_u = nullptr;
    long long* d_v = nullptr;
    unsigned* d_p1_ptr = nullptr;   // [total_uv + 1]
    Term* d_p1 = nullptr;
    unsigned* d_p2_ptr = nullptr;   // [total_uv + 1]
    Term* d_p2 = nullptr;
    Term* d_p2s = nullptr;          // [n_p2s]
    ulonglong2* d_w = nullptr;      // custom-comb weights {img, real}
    int* d_src = nullptr;           // custom-comb sources
    fp2* d_part = nullptr;          // grid-sum partials (+ a ticket after max_blocks entries)
    unsigned max_blocks = 1;
};

// Validates the gates (indices inside their layer, as the reference's arrays
// require; unknown types contribute nothing, as in the reference) and builds the
// term lists on the device. nullptr and the error set on failure.
Layer* layer_create(int length_g, int length_u, const int* ty, const long long* u, const long long* v,
                    const int* comb_ptr, const int* comb_src, const uint64_t* comb_w);
void layer_destroy(Layer* L);

// sumcheck_phase1_init: V_mult_add = {0, values}, addV_array / add_mult_sum from
// the gates; r0, r1 (length_g), alpha, beta host elements {img, real}.
bool phase1_init(const Layer& L, const ulonglong2* values, const uint64_t* r0, const uint64_t* r1,
                 const uint64_t* alpha, const uint64_t* beta, ulonglong2* vma, ulonglong2* addv, ulonglong2* ams,
                 cudaStream_t s);
// sumcheck_phase2_init(prev_r, r_u, 1 - r_u) with v_u = vma0.a prev_r + vma0.b
// (vma0: the one-entry V_mult_add phase 1's rounds leave, device).
bool phase2_init(const Layer& L, const ulonglong2* values, const uint64_t* r0, const uint64_t* r1,
                 const uint64_t* alpha, const uint64_t* beta, const ulonglong2* vma0, const uint64_t* prev_r,
                 const uint64_t* r_u, ulonglong2* vma, ulonglong2* addv, ulonglong2* ams, cudaStream_t s);

}  // namespace virgo
}  // namespace tp
