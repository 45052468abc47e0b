// Virgo (linear GKR) sumcheck round on the device -- see virgo.cu.
#pragma once
#include <cuda_runtime.h>

#include "fp2.cuh"

namespace tp {
namespace virgo {

// One sumcheck_phase{1,2}_update over tables of n linear_poly entries (n even):
// folded tables (n / 2 entries) into *_out, round polynomial {a, b, c} into ret
// (three {img, real} elements). r canonical; inputs canonical.
bool update(const ulonglong2* vma, const ulonglong2* addv, const ulonglong2* ams, long long n, fp2 r, int bit,
            ulonglong2* vma_out, ulonglong2* addv_out, ulonglong2* ams_out, ulonglong2* ret, cudaStream_t s);

}  // namespace virgo
}  // namespace tp
