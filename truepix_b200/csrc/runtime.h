// Process-wide device context for the prover core: one CUDA device per process
// (the device current at first use), one library stream, a stream-ordered
// caching memory pool, and a thread-local error state that the C ABI reports
// through tp_last_error()/tp_last_error_code().
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>

namespace tp {

struct Ctx {
    int device = -1;
    int n_sm = 0;
    cudaStream_t stream = nullptr;   // library stream (non-blocking)
    cudaMemPool_t pool = nullptr;    // stream-ordered pool, memory kept cached
};

// Initialise once; returns nullptr (and sets the error) when no device is usable.
Ctx* ctx();
bool device_present();

// error state -----------------------------------------------------------
enum ErrCode { TP_OK = 0, TP_ERR_ARG = 1, TP_ERR_CUDA = 2, TP_ERR_NODEV = 3, TP_ERR_OOM = 4 };
void set_error(int code, const char* fmt, ...);
void clear_error();
int error_code();
const char* error_text();
// record a CUDA failure; returns true when `e` is an error
bool cuda_failed(cudaError_t e, const char* what);

// stream-ordered allocation from the library pool ------------------------
void* dev_alloc(size_t bytes, cudaStream_t s);
void dev_free(void* p, cudaStream_t s);

// Asynchronous host->device upload of a small host buffer through a pinned
// staging ring (64 slots of 256 KB, each reused only after its previous copy has
// completed). The host buffer may be reused as soon as the call returns. Larger
// uploads are copied synchronously.
bool upload_async(void* d_dst, const void* h_src, size_t bytes, cudaStream_t s);

// Large copies between caller-owned host buffers and the device. A pinned host
// buffer is copied directly; a pageable one of 4 MB or more goes through two
// 16 MB pinned staging buffers filled (or drained) by several host threads while
// the other buffer's DMA runs. host_to_device returns once the host buffer has
// been read (the device copy completes in stream order on s); device_to_host
// returns once the host buffer holds the data (it synchronises s).
bool host_to_device(void* d_dst, const void* h_src, size_t bytes, cudaStream_t s);
bool device_to_host(void* h_dst, const void* d_src, size_t bytes, cudaStream_t s);

// Kernel timer: when enabled, kernels that support it record a CUDA event pair
// around their launch with an integer tag; read back after synchronising.
bool timer_enable(int max_pairs);
void timer_disable();
void timer_reset();
bool timer_on();
void timer_begin(cudaStream_t s, int tag);
void timer_end(cudaStream_t s);
int timer_read(float* ms, int* tags, int max_pairs);

// grid sizing helpers ----------------------------------------------------
inline unsigned blocks_for(size_t n, unsigned threads)
{
    return (unsigned)((n + threads - 1) / threads);
}

}  // namespace tp

#define TP_CUDA_OK(expr, what)                   \
    do {                                         \
        if (::tp::cuda_failed((expr), (what)))   \
            return false;                        \
    } while (0)
