// C ABI of the late rounds (late.cuh): one CTA per frame runs all 2n late rounds
// of its input layer and the line projection in one launch, with challenges
// given by the caller or drawn round by round from the frame's transcript by
// the VOLE-committed round (vole.cuh) -- the reference prover's loop
// circuitnizkvec_vole.py:396-418 for rounds nCopyBits..nCopyBits + 2n - 1.
#include <stdint.h>

#include "late.cuh"
#include "runtime.h"
#include "../../include/native_fp2.h"

namespace {

using namespace tp;
using late::kThreads;

struct Args {
    const fp2* wires;
    const fp2* beta;
    const fp2* zg;
    long long zg_stride;   // 0: one weight vector for every frame
    const fp2* chal;
    fs::State* st;
    vole::State* vs;
    const fp2* u;
    const fp2* v;
    fp2* coefs;
    fp2* h;
    fp2* chal_out;
    fp2* proof;
    const fp2* z2;
    const fp2* w3;
    long long w3_frame_stride, w3_round_stride;
    fp2* closing;
    fp2* point;
    fp2* tag;
    late::Shape sh;
};

// par.all / par.one of late::run_frame on the device
struct DevPar {
    template <class F>
    __device__ void all(F&& fn) const
    {
        fn((int)threadIdx.x);
        __syncthreads();
    }
    template <class F>
    __device__ void one(F&& fn) const
    {
        if (threadIdx.x == 0) fn();
        __syncthreads();
    }
};

__global__ void __launch_bounds__(kThreads) late_kernel(const Args a, const __grid_constant__ late::Gates G)
{
    __shared__ late::Work w;
    const long long i = blockIdx.x;
    const int n = a.sh.n, W = 1 << n;
    late::Frame f;
    f.wires = a.wires + i * W;
    f.beta = a.beta + i;
    f.zg = a.zg + i * a.zg_stride;
    f.chal = a.chal ? a.chal + i * 2 * n : nullptr;
    f.st = a.st ? a.st + i : nullptr;
    f.vs = a.vs ? a.vs + i : nullptr;
    f.u = a.u ? a.u + i * a.sh.count : nullptr;
    f.v = a.v ? a.v + i * a.sh.count : nullptr;
    f.coefs = a.coefs + i * 6 * n;
    f.h = a.h + i * (n + 1);
    f.chal_out = a.chal_out + i * 2 * n;
    f.proof = a.proof ? a.proof + i * 8 * n : nullptr;
    const int nb = a.sh.round0;
    f.z2 = a.closing ? a.z2 + i * nb : nullptr;
    f.w3 = a.closing ? a.w3 + i * a.w3_frame_stride : nullptr;
    f.w3_stride = a.w3_round_stride;
    f.closing = a.closing ? a.closing + i * (n + 10 + 5 * (a.sh.zk != 0)) : nullptr;
    f.point = a.closing ? a.point + i * (n + nb) : nullptr;
    f.tag = a.closing ? a.tag + i : nullptr;
    late::run_frame(w, f, a.sh, G.g, DevPar{});
}

}  // namespace

extern "C" {

int tp_late_rounds_dev(int n_frames, int n_in_bits, int n_gates, const int* gate_type, const int* in0,
                       const int* in1, const void* d_wires, const void* d_beta, const void* d_gate_weights,
                       int weights_per_frame, const void* d_challenges, void* d_fs_states, void* d_vole_states,
                       const void* d_u, const void* d_v, long long count, int layer, int round0, void* d_coefs,
                       void* d_line, void* d_challenges_out, void* d_proof, const void* d_z2, const void* d_w3,
                       long long w3_frame_stride, long long w3_round_stride, void* d_closing, void* d_point,
                       void* d_tag, int zk, void* stream)
{
    tp::clear_error();
    if (!tp::ctx()) return -1;
    const bool given = d_challenges != nullptr;
    const bool vole_mode = d_fs_states && d_vole_states && d_u && d_v && count >= 3;
    const bool closing = d_closing != nullptr;
    if (n_frames < 1 || n_in_bits < 1 || n_in_bits > late::kMaxInBits || n_gates < 1 || n_gates > late::kMaxGates ||
        !gate_type || !in0 || !in1 || !d_wires || !d_beta || !d_gate_weights || !d_coefs || !d_line ||
        !d_challenges_out || given == vole_mode || (d_proof && !vole_mode) || round0 < 0 || round0 > 64 ||
        (closing && (!vole_mode || !d_point || !d_tag || (round0 > 0 && (!d_z2 || !d_w3))))) {
        tp::set_error(tp::TP_ERR_ARG, "tp_late_rounds_dev: bad arguments");
        return -1;
    }
    late::Gates G;
    const int W = 1 << n_in_bits;
    for (int g = 0; g < n_gates; ++g) {
        if (gate_type[g] < 0 || gate_type[g] > 12 || in0[g] < 0 || in0[g] >= W || in1[g] < 0 || in1[g] >= W) {
            tp::set_error(tp::TP_ERR_ARG, "tp_late_rounds_dev: gate %d out of range", g);
            return -1;
        }
        G.g[g] = ((uint32_t)gate_type[g] << 28) | ((uint32_t)in0[g] << 14) | (uint32_t)in1[g];
    }
    Args a;
    a.wires = static_cast<const fp2*>(d_wires);
    a.beta = static_cast<const fp2*>(d_beta);
    a.zg = static_cast<const fp2*>(d_gate_weights);
    a.zg_stride = weights_per_frame ? n_gates : 0;
    a.chal = static_cast<const fp2*>(d_challenges);
    a.st = given ? nullptr : static_cast<fs::State*>(d_fs_states);
    a.vs = given ? nullptr : static_cast<vole::State*>(d_vole_states);
    a.u = given ? nullptr : static_cast<const fp2*>(d_u);
    a.v = given ? nullptr : static_cast<const fp2*>(d_v);
    a.coefs = static_cast<fp2*>(d_coefs);
    a.h = static_cast<fp2*>(d_line);
    a.chal_out = static_cast<fp2*>(d_challenges_out);
    a.proof = static_cast<fp2*>(d_proof);
    a.z2 = static_cast<const fp2*>(d_z2);
    a.w3 = static_cast<const fp2*>(d_w3);
    a.w3_frame_stride = w3_frame_stride;
    a.w3_round_stride = w3_round_stride;
    a.closing = static_cast<fp2*>(d_closing);
    a.point = static_cast<fp2*>(d_point);
    a.tag = static_cast<fp2*>(d_tag);
    a.sh.n = n_in_bits;
    a.sh.n_gates = n_gates;
    a.sh.count = given ? 0 : count;
    a.sh.layer = layer;
    a.sh.round0 = round0;
    a.sh.zk = zk ? 1 : 0;
    late_kernel<<<n_frames, kThreads, 0, reinterpret_cast<cudaStream_t>(stream)>>>(a, G);
    return tp::cuda_failed(cudaGetLastError(), "late rounds") ? -1 : 0;
}

}  // extern "C"
