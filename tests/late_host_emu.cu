// Test harness: the late-round CTA of the device library (late::run_frame in
// truepix_b200/csrc/late.cuh) run on the host, one frame, with a loop over the
// CTA's thread indices in place of the threads and a barrier between steps.
// The device kernel (truepix_b200/csrc/late.cu) runs the same steps with
// __syncthreads() between them, so this checks the CTA's algorithm and its
// step decomposition on the CPU against the reference's fixtures.
#include <stdint.h>

#include "../truepix_b200/csrc/late.cuh"

using namespace tp;

namespace {

struct HostPar {
    template <class F>
    void all(F&& fn) const
    {
        for (int t = 0; t < late::kThreads; ++t) fn(t);
    }
    template <class F>
    void one(F&& fn) const
    {
        fn();
    }
};

}  // namespace

// One frame's late rounds. chal != null: the 2n challenges are given (st, vs,
// u, v unused); otherwise they are drawn by the VOLE-committed rounds from the
// transcript st and VOLE state vs (updated in place). closing != null: the
// layer's closing proofs too (point, tag, z2, w3 then needed).
extern "C" int emu_late_frame(int n, int n_gates, const int* type, const int* in0, const int* in1, const void* wires,
                              const void* beta, const void* zg, const void* chal, void* st, void* vs, const void* u,
                              const void* v, long long count, int layer, int round0, void* coefs, void* line,
                              void* chal_out, void* proof, const void* z2, const void* w3, void* closing, void* point,
                              void* tag, int zk)
{
    if (n < 1 || n > late::kMaxInBits || n_gates < 1 || n_gates > late::kMaxGates) return -1;
    static late::Work w;   // 46 KB: the CTA's shared memory
    static late::Gates G;
    for (int g = 0; g < n_gates; ++g) {
        if (type[g] < 0 || type[g] > 12 || in0[g] < 0 || in0[g] >= (1 << n) || in1[g] < 0 || in1[g] >= (1 << n))
            return -1;
        G.g[g] = ((uint32_t)type[g] << 28) | ((uint32_t)in0[g] << 14) | (uint32_t)in1[g];
    }
    late::Frame f;
    f.wires = static_cast<const fp2*>(wires);
    f.beta = static_cast<const fp2*>(beta);
    f.zg = static_cast<const fp2*>(zg);
    f.chal = static_cast<const fp2*>(chal);
    f.st = static_cast<fs::State*>(st);
    f.vs = static_cast<vole::State*>(vs);
    f.u = static_cast<const fp2*>(u);
    f.v = static_cast<const fp2*>(v);
    f.coefs = static_cast<fp2*>(coefs);
    f.h = static_cast<fp2*>(line);
    f.chal_out = static_cast<fp2*>(chal_out);
    f.proof = static_cast<fp2*>(proof);
    f.z2 = static_cast<const fp2*>(z2);
    f.w3 = static_cast<const fp2*>(w3);
    f.w3_stride = 1;
    f.closing = static_cast<fp2*>(closing);
    f.point = static_cast<fp2*>(point);
    f.tag = static_cast<fp2*>(tag);
    late::Shape sh;
    sh.n = n;
    sh.n_gates = n_gates;
    sh.count = chal ? 0 : count;
    sh.layer = layer;
    sh.round0 = round0;
    sh.zk = zk ? 1 : 0;
    late::run_frame(w, f, sh, G.g, HostPar{});
    return w.bad ? 1 : 0;
}
