// Fp2 number-theoretic transforms over the 2^k-th roots of unity of
// Fp2 = F_{2^61-1}[i]/(i^2 + 1), with the reference's roots and element layout.
//
// Reference: TruePix-main/Orion/Orion_nonzk/src/infrastructure/RS_polynomial.cpp:46-206
// (fast_fourier_transform / inverse_fast_fourier_transform) and
// src/linear_gkr/prime_field.cpp:60-73 (get_root_of_unity: the generator
// g = (real 2147483648, img 1033321771269002680) of order 2^62, squared 62 - k
// times for the 2^k-th root).
//
// forward(coef, m, n): out[i] = sum_{j<m} coef[j] w_n^(ij), i < n (m <= n).
// inverse(evals, m, n): the m coefficients of the polynomial whose values on the
//   m-th roots of unity are evals[i * (n / m)], i.e.
//   out[j] = m^-1 sum_i evals[i n/m] w_m^(-ij).
// Both are exact, so any evaluation order gives the reference's values.
//
// Device algorithm: an n-point DFT as P <= 3 passes of radix R = 2^b <= 2^10
// (n = R_1 R_2 ... R_P). Pass t computes, for every column of R_t elements at
// stride S_t = R_{t+1}...R_P, the R_t-point DFT in shared memory (radix-2 stages on
// a bit-reversed load), multiplies by the twiddle w_{R_t S_t}^(k s) and stores in
// place; the last pass reads rows (stride 1) and writes the natural output order
// (digit reversal folded into its addresses). Elements are 16 bytes {img, real}.
#pragma once
#include <cuda_runtime.h>

#include <vector>

#include "fp2.cuh"

namespace tp {
namespace ntt {

constexpr int kMaxLog = 28;   // transforms up to 2^28 points

// get_root_of_unity(lg) on the host (canonical)
fp2 root_of_unity(int lg);

// Batched transforms: `batch` independent transforms; transform b reads
// in + b * in_batch and writes out + b * out_batch (element strides).
// scratch: n * batch elements when the plan has more than one pass (nullptr
// makes the call allocate from the pool). in == out is allowed for batch 1.
bool forward(const ulonglong2* in, long long m, long long n, ulonglong2* out, int batch, long long in_batch,
             long long out_batch, ulonglong2* scratch, cudaStream_t s);
bool inverse(const ulonglong2* in, long long m, long long n, ulonglong2* out, int batch, long long in_batch,
             long long out_batch, ulonglong2* scratch, cudaStream_t s);

// The device tables of w^t for w = the 2^logn-th root of unity (or its inverse):
// w^e = lo[e mod 2^h] * hi[e >> h], e < 2^logn. Cached per device.
bool power_tables(int logn, bool inverse, const fp2** lo, const fp2** hi, int* h);

// number of passes of an n-point transform
int passes(long long n);

int last_launches();

// Autotuner: times every split of a 2^logn transform into the default number of
// passes (and one more, up to three) of 3..10 bits on this device, batch
// transforms at a time, and keeps the fastest for later transforms of that size
// on this device. Results are exact whatever the split.
bool autotune(int logn, int batch, std::vector<int>& best, float* best_ms);

}  // namespace ntt

namespace rs {

// Reed-Solomon commit of 2^log_len elements at rate 2^-5 with 64 slices
// (include/poly_commitment/poly_commit.h:42-96 commit_private_array, then
// src/VPD/fri.cpp:36-123 request_init_commit):
//   l_eval[i][.] = FFT onto 2^(log_len-1) points of IFFT(slice i of 2^(log_len-6)
//   inputs), i < 64 (slice-major, 2^(log_len+5) elements);
//   leaf j < 2^(log_len-2) = chain over i of h <- SHA256(l_eval[i][j] ||
//   l_eval[i][j + 2^(log_len-2)] || h) from h = 0; tree over the leaves, root at 1.
// tree holds 2^(log_len-1) digests. Temporary buffers come from the pool.
constexpr int kMinLog = 6, kMaxLog = 25;
bool commit(const ulonglong2* src, int log_len, ulonglong2* l_eval, unsigned char* tree, cudaStream_t s);

// One FRI commit-phase step (src/VPD/fri.cpp:316-420) on a witness in the
// interleaved layout w[(k << 7) | (j << 1) | h] = slice j's value at k + h M/2
// (M = 2^log_m points per slice): next (M/2 x 64 elements, same layout) gets
// 2^-1 ((x + y) + w_M^-i r (x - y)) re-interleaved, tree (M/2 digests) the Merkle
// tree of its leaf chains SHA256(x || y || h) over the 64 slices, root at 1.
bool fri_step(const ulonglong2* w, int log_m, fp2 r, ulonglong2* next, unsigned char* tree, cudaStream_t s);

}  // namespace rs
}  // namespace tp
