// C entry points over the reference's own Orion sources (TEST INFRASTRUCTURE).
//
// Compiled by `make -C oracle ref` together with the unmodified reference files
// under TruePix-main/Orion/Orion_nonzk (their own sources, compiled in place)
// into oracle/_ref/liborion_ref.so. The golden generator and the CPU baseline
// call these; the shipped library never links them.
#include <chrono>
#include <cstdint>
#include <cstdlib>
#include <cstring>

#include "infrastructure/RS_polynomial.h"
#include "infrastructure/merkle_tree.h"
#include "infrastructure/my_hhash.h"
#include "linear_code/linear_code_encode.h"
#include "linear_gkr/prime_field.h"
#include "linear_gkr/prover.h"
#include "poly_commitment/poly_commit.h"
#include "VPD/fri.h"
#include "VPD/linearPC.h"
#include "truepix/truepix_gkr.h"

// the codeword commit() retains (defined in src/VPD/linearPC.cpp)
extern prime_field::field_element** encoded_codeword;

namespace {
double g_seconds = 0;   // duration of the reference work of the last timed call
double now() { return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count(); }
}  // namespace

extern "C" {

// seconds the reference's own work took in the last ref_combine (the passes
// after commit()), ref_virgo_update (the update call), ref_fri_step (the step)
// or ref_virgo_init (the init call of the requested phase)
double ref_last_seconds(void) { return g_seconds; }

// SHA-256 of one 64-byte block exactly as Orion hashes it (my_hhash)
void ref_hhash64(const unsigned char* in, unsigned char* out32)
{
    my_hhash(in, out32);
}

// element pairs are (img, real), the reference's memory order
static_assert(sizeof(prime_field::field_element) == 16, "field_element layout");

// result[i] = P(w^i), w = get_root_of_unity(log2 order), P given by coef_len coefficients
void ref_fft(const uint64_t* coef, int coef_len, int order, uint64_t* result)
{
    prime_field::init();
    init_scratch_pad(order);
    const int lg = __builtin_ctz((unsigned)order);
    fast_fourier_transform(reinterpret_cast<const prime_field::field_element*>(coef), coef_len,
                           order, prime_field::get_root_of_unity(lg),
                           reinterpret_cast<prime_field::field_element*>(result));
    delete_scratch_pad();
}

// coefficients (coef_len of them) of the polynomial whose evaluations on the
// order-th roots of unity are `evals` (sub-sampled when coef_len < order)
void ref_ifft(const uint64_t* evals, int coef_len, int order, uint64_t* result)
{
    prime_field::init();
    init_scratch_pad(order);
    const int lg = __builtin_ctz((unsigned)order);
    prime_field::field_element* e = new prime_field::field_element[order];
    memcpy(e, evals, 16 * (size_t)order);
    inverse_fast_fourier_transform(e, coef_len, order, prime_field::get_root_of_unity(lg),
                                   reinterpret_cast<prime_field::field_element*>(result));
    delete[] e;
    delete_scratch_pad();
}

// Orion commit of N field elements (N a multiple of 128) exactly as
// linearPC_multi_commit does it in a fresh process (glibc rand() from its
// default seed drives expander_init). Writes the 32-byte root and its hex form
// (truepix::root_hex). Call once per process: the reference keeps encoder state.
void ref_commit(const uint64_t* src, long long N, unsigned char* root32, char* hex65)
{
    prime_field::init();
    srand(1);
    expander_init(N / column_size);
    set_retain_encoded_codeword(true);
    __hhash_digest* h = commit(reinterpret_cast<const prime_field::field_element*>(src), N);
    memcpy(root32, &h[1], 32);
    const std::string hx = truepix::root_hex(h[1]);
    memcpy(hex65, hx.c_str(), 65);
}

// Reed-Solomon commit of 2^log_len elements exactly as
// poly_commit_prover::commit_private_array does it: 64 slices, each an IFFT of
// 2^(log_len-6) evaluations followed by an FFT onto 2^(log_len-1) points (rate
// 2^-5), then fri::request_init_commit's interleave, leaf chains and Merkle
// tree. Writes the root and, when l_eval != NULL, the 2^(log_len+5) codeword
// elements (slice-major). Call once per process.
void ref_rs_commit(const uint64_t* src, int log_len, unsigned char* root32, uint64_t* l_eval)
{
    prime_field::init();
    const size_t n = (size_t)1 << log_len;
    prime_field::field_element* a = new prime_field::field_element[n];
    memcpy(a, src, 16 * n);
    poly_commit::poly_commit_prover p;
    __hhash_digest h = p.commit_private_array(a, log_len);
    memcpy(root32, &h, 32);
    if (l_eval) memcpy(l_eval, poly_commit::l_eval, 16 * (n << rs_code_rate));
    delete[] a;
}

// The prover-side passes of tensor_product_protocol (src/VPD/linearPC.cpp:480-531,
// 569-571) over the codeword that commit() retains, with the reference's own
// primitives: combined[t] = sum_j r0[j] * encoded_codeword[j][t]; leaves
// merkle_tree::hash_single_field_element(combined[i] or 0), i < 2 N/128, tree by
// create_tree; answer = sum_i r1[i] * combined[i], i < N/128. Call once per process.
void ref_combine(const uint64_t* src, long long N, const uint64_t* r0, const uint64_t* r1,
                 uint64_t* combined_out, unsigned char* root32, uint64_t* answer)
{
    typedef prime_field::field_element F;
    prime_field::init();
    srand(1);
    expander_init(N / column_size);
    set_retain_encoded_codeword(true);
    commit(reinterpret_cast<const F*>(src), N);
    const long long msg_len = N / column_size, cw_len = encode_output_len(msg_len);
    const F* R0 = reinterpret_cast<const F*>(r0);
    const F* R1 = reinterpret_cast<const F*>(r1);
    const double t0 = now();
    F* comb = new F[cw_len];
    for (long long t = 0; t < cw_len; ++t) comb[t] = F(0ULL);
    for (int j = 0; j < column_size; ++j)
        for (long long t = 0; t < cw_len; ++t) comb[t] = comb[t] + R0[j] * encoded_codeword[j][t];
    F ans = F(0ULL);
    for (long long i = 0; i < msg_len; ++i) ans = ans + R1[i] * comb[i];
    memcpy(answer, &ans, 16);
    memcpy(combined_out, comb, 16 * (size_t)cw_len);
    __hhash_digest* leaves = new __hhash_digest[msg_len * 2];
    F zero;
    memset(&zero, 0, sizeof(zero));
    for (long long i = 0; i < msg_len * 2; ++i)
        leaves[i] = merkle_tree::hash_single_field_element(i < cw_len ? comb[i] : zero);
    __hhash_digest* mt = nullptr;
    merkle_tree::merkle_tree_prover::create_tree(leaves, msg_len * 2, mt, sizeof(__hhash_digest), true);
    g_seconds = now() - t0;
    memcpy(root32, &mt[1], 32);
    free(mt);
    delete[] leaves;
    delete[] comb;
}

// One Virgo sumcheck update (zk_prover::sumcheck_phase1_update when phase == 1,
// sumcheck_phase2_update when phase == 2; src/linear_gkr/prover.cpp:576-644,
// 935-1006) on tables given as linear_poly arrays of n entries {a, b}: the folded
// tables (n / 2 entries each) and the returned quadratic_poly {a, b, c}.
void ref_virgo_update(int phase, const uint64_t* vma, const uint64_t* addv, const uint64_t* ams, int n,
                      const uint64_t* r, int current_bit, uint64_t* vma_out, uint64_t* addv_out,
                      uint64_t* ams_out, uint64_t* ret)
{
    prime_field::init();
    int bits = 0;
    while ((1 << bits) < n) ++bits;
    zk_prover* p = new zk_prover();
    p->init_array(bits);
    memcpy(p->V_mult_add, vma, 32 * (size_t)n);
    memcpy(p->addV_array, addv, 32 * (size_t)n);
    memcpy(p->add_mult_sum, ams, 32 * (size_t)n);
    p->total_uv = n;
    prime_field::field_element pr;
    memcpy(&pr, r, 16);
    const double t0 = now();
    quadratic_poly q = phase == 1 ? p->sumcheck_phase1_update(pr, current_bit)
                                  : p->sumcheck_phase2_update(pr, current_bit);
    g_seconds = now() - t0;
    memcpy(vma_out, p->V_mult_add, 16 * (size_t)n);
    memcpy(addv_out, p->addV_array, 16 * (size_t)n);
    memcpy(ams_out, p->add_mult_sum, 16 * (size_t)n);
    memcpy(ret, &q, 48);
    layered_circuit none;     // delete_self frees circuit_value[0 .. C->total_depth)
    none.total_depth = 0;
    p->C = &none;
    p->delete_self();
    delete p;
}

// One FRI commit-phase step (fri::commit_phase_step, src/VPD/fri.cpp:316-420) on
// a previous witness given in the interleaved layout of request_init_commit /
// earlier steps: w[(k << 7) | (j << 1) | h] = slice j's value at k + h M / 2,
// k < M / 2 = 2^(log_m - 1). The reference's globals are set up as after an
// earlier step (current_step_no 1, L_group = powers of the M-th root of unity).
// Writes the next interleaved witness (M / 2 * 64 elements) and the root of its
// tree. Call once per process.
void ref_fri_step(const uint64_t* witness, int log_m, const uint64_t* r, uint64_t* next, unsigned char* root32)
{
    typedef prime_field::field_element F;
    prime_field::init();
    const int M = 1 << log_m;
    poly_commit::slice_count = slice_number;
    fri::log_current_witness_size_per_slice = log_m;
    fri::current_step_no = 1;
    F* prev = new F[(size_t)M * slice_number];
    memcpy(prev, witness, 16 * (size_t)M * slice_number);
    int* map = new int[(size_t)M * slice_number];
    for (int i = 0; i < M / 2; ++i)
        for (int j = 0; j < slice_number; ++j) {
            map[(i << log_slice_number) | j] = (i << (log_slice_number + 1)) | (j << 1);
            map[((i + M / 2) << log_slice_number) | j] = (i << (log_slice_number + 1)) | (j << 1);
        }
    fri::cpd.rs_codeword[0] = prev;
    fri::cpd.rs_codeword_mapping[0] = map;
    fri::L_group = new F[M];
    const F w = prime_field::get_root_of_unity(log_m);
    fri::L_group[0] = F(1ULL);
    for (int i = 1; i < M; ++i) fri::L_group[i] = fri::L_group[i - 1] * w;
    F fr;
    memcpy(&fr, r, 16);
    const double t0 = now();
    __hhash_digest h = fri::commit_phase_step(fr);
    g_seconds = now() - t0;
    memcpy(root32, &h, 32);
    memcpy(next, fri::cpd.rs_codeword[1], 16 * (size_t)(M / 2) * slice_number);
}

// zk_prover::sumcheck_phase1_init (phase 1) or sumcheck_phase2_init (phase 2;
// src/linear_gkr/prover.cpp:246-570, 645-930) of layer 1 of a two-layer circuit:
// layer 1 has 2^length_g gates (ty, u, v; type-14 gates take (src, weight)
// lists comb_src / comb_w[comb_ptr[g] .. comb_ptr[g + 1])), layer 0 holds the
// 2^length_u values. r0, r1: length_g elements; alpha, beta: one each. Phase 2
// runs phase 1's init first (its beta tables), sets V_mult_add[0] to the
// linear_poly vma0 = {a, b} (the table phase 1's rounds leave) and calls
// sumcheck_phase2_init(prev_r, r_u, 1 - r_u), r_u of length_u elements. Writes
// the three linear_poly tables (2^length_u entries {a, b}). Call once per process.
void ref_virgo_init(int phase, int length_g, int length_u, const int* ty, const long long* u, const long long* v,
                    const int* comb_ptr, const int* comb_src, const uint64_t* comb_w, const uint64_t* values,
                    const uint64_t* r0, const uint64_t* r1, const uint64_t* alpha, const uint64_t* beta,
                    const uint64_t* vma0, const uint64_t* prev_r, const uint64_t* r_u, uint64_t* vma_out,
                    uint64_t* addv_out, uint64_t* ams_out)
{
    typedef prime_field::field_element F;
    prime_field::init();
    const long long G = 1LL << length_g, U = 1LL << length_u;
    layered_circuit* C = new layered_circuit();
    C->total_depth = 2;
    C->circuit = new layer[2];
    C->circuit[0].bit_length = length_u;
    C->circuit[1].bit_length = length_g;
    C->circuit[1].gates = new gate[G];
    for (long long g = 0; g < G; ++g) {
        gate& q = C->circuit[1].gates[g];
        q.ty = ty[g];
        q.u = u[g];
        q.v = v[g];
        if (ty[g] == 14 && comb_ptr) {
            const int n = comb_ptr[g + 1] - comb_ptr[g];
            q.parameter_length = n;
            q.src = new int[n > 0 ? n : 1];
            q.weight = new F[n > 0 ? n : 1];
            for (int k = 0; k < n; ++k) {
                q.src[k] = comb_src[comb_ptr[g] + k];
                memcpy(&q.weight[k], comb_w + 2 * (comb_ptr[g] + k), 16);
            }
        }
    }
    zk_prover* p = new zk_prover();
    p->init_array(length_g > length_u ? length_g : length_u);
    p->C = C;
    p->circuit_value[0] = new F[U];
    memcpy(p->circuit_value[0], values, 16 * (size_t)U);
    F* R0 = new F[length_g + 1];
    F* R1 = new F[length_g + 1];
    F* O0 = new F[length_g + 1];
    F* O1 = new F[length_g + 1];
    const F one(1ULL);
    for (int k = 0; k < length_g; ++k) {
        memcpy(&R0[k], r0 + 2 * k, 16);
        memcpy(&R1[k], r1 + 2 * k, 16);
        O0[k] = one - R0[k];
        O1[k] = one - R1[k];
    }
    F al, be;
    memcpy(&al, alpha, 16);
    memcpy(&be, beta, 16);
    p->sumcheck_init(1, length_g, length_u, length_u, al, be, R0, R1, O0, O1);
    const double t0 = now();
    p->sumcheck_phase1_init();
    if (phase == 2) {
        F a, b, pr;
        memcpy(&a, vma0, 16);
        memcpy(&b, vma0 + 2, 16);
        memcpy(&pr, prev_r, 16);
        p->V_mult_add[0] = linear_poly(a, b);
        F* RU = new F[length_u + 1];
        F* OU = new F[length_u + 1];
        for (int k = 0; k < length_u; ++k) {
            memcpy(&RU[k], r_u + 2 * k, 16);
            OU[k] = one - RU[k];
        }
        const double t1 = now();
        p->sumcheck_phase2_init(pr, RU, OU);
        g_seconds = now() - t1;
    } else {
        g_seconds = now() - t0;
    }
    memcpy(vma_out, p->V_mult_add, 32 * (size_t)U);
    memcpy(addv_out, p->addV_array, 32 * (size_t)U);
    memcpy(ams_out, p->add_mult_sum, 32 * (size_t)U);
}

// encoded length of a column of n elements (graphs generated from the default seed)
long long ref_encode_len(long long n)
{
    srand(1);
    expander_init(n);
    return encode_output_len(n);
}

// the codeword of one column of n elements: dst must hold ref_encode_len(n) elements
void ref_encode(const uint64_t* src, long long n, uint64_t* dst)
{
    prime_field::init();
    srand(1);
    expander_init(n);
    encode(reinterpret_cast<const prime_field::field_element*>(src),
           reinterpret_cast<prime_field::field_element*>(dst), n);
}

}  // extern "C"
