// tp_mle_eval_base_noalloc: the MLE of base-field inputs at an Fp2 point
// (the computation of tp_mle_eval_base_dev) for callers that cannot allocate
// device memory. Some callers cannot call cudaMalloc: a host application whose
// device memory is owned by another allocator that has already reserved the
// GPU, or a time-critical loop that must not pay the implicit synchronisation
// of cudaMalloc/cudaFree. This entry point uses a fixed scratch area compiled
// into the library instead of any allocation.
//
// The scratch is a file-scope device array sized for at most 2^26 inputs
// (n_z <= 26): the eq tables (2^12 + 2^14 Fp2), one partial sum per block
// (1184 blocks) and the reduction ticket, 339 KB. Every GPU that loads the
// library holds it until the process exits. All calls share it and it keeps
// the last call's contents, so the ticket is cleared at the start of each call,
// and two calls whose kernels overlap on the GPU (different streams, or
// different host threads on one device) race on it: the caller must order them.
//
// The host cannot use the array's name as a device address (on the host it is
// only a stand-in). The first call on a device, with that device current, asks
// the runtime for the array's device address (cudaGetSymbolAddress) and keeps
// it; make that first call before any stream capture.
#include <mutex>
#include <vector>

#include "gkr.h"
#include "runtime.h"

namespace {

constexpr int kMaxNz = 26;
constexpr int kLoBits = 12;
constexpr size_t kTabEntries = ((size_t)1 << kLoBits) + ((size_t)1 << (kMaxNz - kLoBits));
constexpr unsigned kMaxBlocks = 1184;  // 148 SMs x 8 blocks of 256 threads
constexpr size_t kScratchBytes = 16 * (kTabEntries + kMaxBlocks) + 256;

static __device__ __align__(256) unsigned char g_mle_scratch[kScratchBytes];

std::mutex g_mu;
std::vector<void*> g_addr;  // device address of g_mle_scratch, per device ordinal

// Device address of the scratch on the current device (looked up once per device).
void* scratch_on_current_device()
{
    int dev = 0;
    if (tp::cuda_failed(cudaGetDevice(&dev), "tp_mle_eval_base_noalloc: cudaGetDevice")) return nullptr;
    std::lock_guard<std::mutex> lock(g_mu);
    if ((int)g_addr.size() <= dev) g_addr.resize((size_t)dev + 1, nullptr);
    if (!g_addr[(size_t)dev]) {
        void* p = nullptr;
        if (tp::cuda_failed(cudaGetSymbolAddress(&p, g_mle_scratch),
                            "tp_mle_eval_base_noalloc: cudaGetSymbolAddress"))
            return nullptr;
        g_addr[(size_t)dev] = p;
    }
    return g_addr[(size_t)dev];
}

}  // namespace

extern "C" int tp_mle_eval_base_noalloc(const void* d_inputs, const void* d_z, int n_z,
                                        void* d_out, void* stream)
{
    tp::clear_error();
    if (n_z < 1 || n_z > kMaxNz) {
        tp::set_error(tp::TP_ERR_ARG,
                      "tp_mle_eval_base_noalloc: n_z = %d outside [1, %d]; its fixed scratch holds "
                      "at most 2^%d inputs (use tp_mle_eval_base_dev for larger inputs)",
                      n_z, kMaxNz, kMaxNz);
        return -1;
    }
    if (!d_inputs || !d_z || !d_out) {
        tp::set_error(tp::TP_ERR_ARG, "tp_mle_eval_base_noalloc: null pointer");
        return -1;
    }
    unsigned char* base = static_cast<unsigned char*>(scratch_on_current_device());
    if (!base) return -1;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    tp::fp2* tabs = reinterpret_cast<tp::fp2*>(base);
    tp::fp2* partials = tabs + kTabEntries;
    unsigned* ticket = reinterpret_cast<unsigned*>(partials + kMaxBlocks);
    // the previous call's ticket may not be zero if that call failed part way
    if (tp::cuda_failed(cudaMemsetAsync(ticket, 0, sizeof(unsigned), s),
                        "tp_mle_eval_base_noalloc: clear ticket"))
        return -1;
    return tp::launch_mle_base_into(static_cast<const tp::u64*>(d_inputs),
                                    static_cast<const tp::fp2*>(d_z), n_z,
                                    static_cast<tp::fp2*>(d_out), tabs, partials, ticket,
                                    kMaxBlocks, s)
               ? 0
               : -1;
}
