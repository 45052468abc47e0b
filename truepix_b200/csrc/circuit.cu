// Evaluation of a one-layer TruePix circuit over a frame's bytes: the output
// vector the prover puts into its transcript before drawing the first GKR
// point (circuitnizkvec_vole.py:351-355), computed on the device.
//
// The reference runs ArithCircuitIncrementalBuilder over Python lists, copy by
// copy (arithcircuitbuilder.py:36-46, arithcircuit.py:121-131): every gate of a
// copy evaluated on the copy's inputs, the copy's outputs padded with zeros to
// 2^ceil(log2 gates), the copies concatenated and the whole vector padded with
// zeros to 2^(out bits + copy bits). Gate values follow the native gate table
// (native_fp2_core.hpp:32-51) on base-field values, which is arithcircuit.py's
// C gates for every type but the multiplexer (3 = left input, 4 = right input
// here, as in that table). The inputs are the frame layout's: copy c's wire
// w < copy_size is byte c * copy_size + w, the constant wire holds const_val,
// every other wire is zero.
//
// One thread per output element, grid-stride over a persistent grid; the gate
// table sits in shared memory, the byte rows are read through the cache, and
// the outputs are written in order (8 bytes per element: the kernel is bound by
// its writes to HBM).
#include <stdint.h>

#include "fp2.cuh"
#include "runtime.h"
#include "../../include/native_fp2.h"

namespace {

using tp::u64;

constexpr int kT = 256;
// The packed gate table travels as a kernel parameter and stays under the
// classic 4 KB parameter limit.
constexpr int kMaxGates = 960;
constexpr int kMaxWires = 1 << 14;

struct Gates {
    uint32_t g[kMaxGates];   // type << 28 | in0 << 14 | in1
};

// native_fp2_core.hpp:32-51 on canonical base-field values
TP_HD u64 gate_value(unsigned type, u64 x, u64 y)
{
    using namespace tp;
    switch (type) {
    case 0: return fmul(x, y);
    case 1: return fadd(x, y);
    case 2: return fsub(x, y);
    case 3: return x;
    case 4: return y;
    case 5: return fsub(fadd(x, y), fmul(x, y));
    case 6: return fsub(fadd(x, y), fadd(fmul(x, y), fmul(x, y)));
    case 7: return fsub(1, x);
    case 8: return fsub(1, fmul(x, y));
    case 9: return fsub(fadd(1, fmul(x, y)), fadd(x, y));
    case 10: return fsub(fadd(1, fadd(fmul(x, y), fmul(x, y))), fadd(x, y));
    case 11: return fmul(fsub(1, x), y);
    default: return x;   // 12: pass
    }
}

__global__ void __launch_bounds__(kT) outputs_kernel(const uint8_t* __restrict__ pix, int n_copies, int cs,
                                                     int const_idx, u64 const_val, int n_gates, int out_bits,
                                                     long long total, u64* __restrict__ out,
                                                     const __grid_constant__ Gates G)
{
    __shared__ uint32_t sg[kMaxGates];
    for (int i = threadIdx.x; i < n_gates; i += blockDim.x) sg[i] = G.g[i];
    __syncthreads();
    const long long mask = (1ll << out_bits) - 1;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += stride) {
        const long long c = e >> out_bits;
        const int g = (int)(e & mask);
        u64 v = 0;
        if (c < n_copies && g < n_gates) {
            const uint32_t t = sg[g];
            const int i0 = (int)((t >> 14) & 0x3FFFu), i1 = (int)(t & 0x3FFFu);
            const uint8_t* row = pix + c * cs;
            const u64 x = i0 < cs ? (u64)__ldg(row + i0) : (i0 == const_idx ? const_val : 0);
            const u64 y = i1 < cs ? (u64)__ldg(row + i1) : (i1 == const_idx ? const_val : 0);
            v = gate_value(t >> 28, x, y);
        }
        out[e] = v;
    }
}

int ceil_log2(int n)
{
    int b = 0;
    while ((1 << b) < n) ++b;
    return b;
}

}  // namespace

extern "C" {

int tp_circuit_out_bits(int n_gates) { return n_gates >= 1 ? ceil_log2(n_gates) : -1; }

int tp_circuit_outputs_pixels_dev(const void* d_pixels, int n_copies, int n_copies_padded, int copy_size,
                                  int n_wires, int const_idx, uint64_t const_val, int n_gates,
                                  const int* gate_type, const int* in0, const int* in1, void* d_out, void* stream)
{
    tp::clear_error();
    tp::Ctx* cx = tp::ctx();
    if (!cx) return -1;
    if (!d_pixels || !d_out || !gate_type || !in0 || !in1 || n_copies < 1 || n_copies_padded < n_copies ||
        (n_copies_padded & (n_copies_padded - 1)) != 0 || copy_size < 1 || n_wires < copy_size ||
        n_wires > kMaxWires || const_idx >= n_wires || (const_idx >= 0 && const_idx < copy_size) ||
        const_val >= tp::P61 || n_gates < 1 || n_gates > kMaxGates) {
        tp::set_error(tp::TP_ERR_ARG, "tp_circuit_outputs_pixels_dev: bad arguments");
        return -1;
    }
    Gates G;
    for (int g = 0; g < n_gates; ++g) {
        if (gate_type[g] < 0 || gate_type[g] > 12 || in0[g] < 0 || in0[g] >= n_wires || in1[g] < 0 ||
            in1[g] >= n_wires) {
            tp::set_error(tp::TP_ERR_ARG, "tp_circuit_outputs_pixels_dev: gate %d out of range", g);
            return -1;
        }
        G.g[g] = ((uint32_t)gate_type[g] << 28) | ((uint32_t)in0[g] << 14) | (uint32_t)in1[g];
    }
    const int out_bits = ceil_log2(n_gates);
    const long long total = (long long)n_copies_padded << out_bits;
    const long long want = (total + kT - 1) / kT;
    const long long cap = (long long)cx->n_sm * 8;
    const int blocks = (int)(want < cap ? want : cap);
    outputs_kernel<<<blocks, kT, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
        static_cast<const uint8_t*>(d_pixels), n_copies, copy_size, const_idx, (u64)const_val, n_gates, out_bits,
        total, static_cast<u64*>(d_out), G);
    return tp::cuda_failed(cudaGetLastError(), "circuit outputs") ? -1 : 0;
}

}  // extern "C"
