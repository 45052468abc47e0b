#include "runtime.h"

#include <stdarg.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <mutex>
#include <vector>

namespace tp {

namespace {
thread_local int t_code = 0;
thread_local char t_text[512] = {0};
std::once_flag g_once;
Ctx g_ctx;
bool g_ok = false;

void init_once()
{
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n <= 0) {
        cudaGetLastError();
        return;
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return;
    g_ctx.device = dev;
    cudaDeviceGetAttribute(&g_ctx.n_sm, cudaDevAttrMultiProcessorCount, dev);
    if (cudaStreamCreateWithFlags(&g_ctx.stream, cudaStreamNonBlocking) != cudaSuccess) return;
    cudaMemPoolProps props;
    memset(&props, 0, sizeof(props));
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    if (cudaMemPoolCreate(&g_ctx.pool, &props) != cudaSuccess) return;
    // keep freed blocks cached for reuse instead of returning them to the driver
    uint64_t keep = UINT64_MAX;
    cudaMemPoolSetAttribute(g_ctx.pool, cudaMemPoolAttrReleaseThreshold, &keep);
    g_ok = true;
}
}  // namespace

Ctx* ctx()
{
    std::call_once(g_once, init_once);
    if (!g_ok) {
        set_error(TP_ERR_NODEV, "no usable CUDA device");
        return nullptr;
    }
    return &g_ctx;
}

bool device_present()
{
    std::call_once(g_once, init_once);
    return g_ok;
}

void set_error(int code, const char* fmt, ...)
{
    t_code = code;
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(t_text, sizeof(t_text), fmt, ap);
    va_end(ap);
}

void clear_error()
{
    t_code = 0;
    t_text[0] = 0;
}

int error_code() { return t_code; }
const char* error_text() { return t_text; }

bool cuda_failed(cudaError_t e, const char* what)
{
    if (e == cudaSuccess) return false;
    set_error(e == cudaErrorMemoryAllocation ? TP_ERR_OOM : TP_ERR_CUDA, "%s: %s", what,
              cudaGetErrorString(e));
    return true;
}

void* dev_alloc(size_t bytes, cudaStream_t s)
{
    Ctx* c = ctx();
    if (!c) return nullptr;
    if (bytes == 0) bytes = 256;
    void* p = nullptr;
    cudaError_t e = cudaMallocFromPoolAsync(&p, bytes, c->pool, s);
    if (e != cudaSuccess) {
        cuda_failed(e, "device allocation");
        return nullptr;
    }
    return p;
}

void dev_free(void* p, cudaStream_t s)
{
    if (p) cudaFreeAsync(p, s);
}

namespace {
constexpr int kRingSlots = 64;
constexpr size_t kRingSlot = 256 * 1024;
std::mutex g_ring_mu;
unsigned char* g_ring = nullptr;
cudaEvent_t g_ring_ev[kRingSlots];
bool g_ring_used[kRingSlots] = {false};
int g_ring_next = 0;
}  // namespace

bool upload_async(void* d_dst, const void* h_src, size_t bytes, cudaStream_t s)
{
    if (bytes == 0) return true;
    if (!ctx()) return false;
    if (bytes > kRingSlot) {
        if (cuda_failed(cudaMemcpyAsync(d_dst, h_src, bytes, cudaMemcpyHostToDevice, s), "upload"))
            return false;
        return !cuda_failed(cudaStreamSynchronize(s), "upload");
    }
    std::lock_guard<std::mutex> lock(g_ring_mu);
    if (!g_ring) {
        if (cuda_failed(cudaHostAlloc((void**)&g_ring, kRingSlots * kRingSlot, cudaHostAllocDefault),
                        "pinned staging"))
            return false;
        for (int i = 0; i < kRingSlots; ++i)
            if (cuda_failed(cudaEventCreateWithFlags(&g_ring_ev[i], cudaEventDisableTiming),
                            "staging event"))
                return false;
    }
    const int slot = g_ring_next;
    g_ring_next = (g_ring_next + 1) % kRingSlots;
    if (g_ring_used[slot] && cuda_failed(cudaEventSynchronize(g_ring_ev[slot]), "staging wait"))
        return false;
    unsigned char* h = g_ring + (size_t)slot * kRingSlot;
    memcpy(h, h_src, bytes);
    if (cuda_failed(cudaMemcpyAsync(d_dst, h, bytes, cudaMemcpyHostToDevice, s), "upload"))
        return false;
    g_ring_used[slot] = true;
    return !cuda_failed(cudaEventRecord(g_ring_ev[slot], s), "staging record");
}

namespace {
std::vector<cudaEvent_t> g_tev;
std::vector<int> g_ttag;
int g_tn = 0;      // events recorded
bool g_ton = false;
}  // namespace

bool timer_enable(int max_pairs)
{
    if (!ctx()) return false;
    while ((int)g_tev.size() < 2 * max_pairs) {
        cudaEvent_t e;
        if (cuda_failed(cudaEventCreate(&e), "timer event")) return false;
        g_tev.push_back(e);
    }
    g_ttag.assign((size_t)max_pairs, 0);
    g_tn = 0;
    g_ton = true;
    return true;
}
void timer_disable() { g_ton = false; }
void timer_reset() { g_tn = 0; }
bool timer_on() { return g_ton; }
void timer_begin(cudaStream_t s, int tag)
{
    if (!g_ton || g_tn + 2 > (int)g_tev.size()) return;
    g_ttag[(size_t)(g_tn / 2)] = tag;
    cudaEventRecord(g_tev[(size_t)g_tn++], s);
}
void timer_end(cudaStream_t s)
{
    if (!g_ton || (g_tn & 1) == 0) return;
    cudaEventRecord(g_tev[(size_t)g_tn++], s);
}
int timer_read(float* ms, int* tags, int max_pairs)
{
    const int n = std::min(g_tn / 2, max_pairs);
    for (int i = 0; i < n; ++i) {
        float t = 0.f;
        if (cuda_failed(cudaEventElapsedTime(&t, g_tev[(size_t)2 * i], g_tev[(size_t)2 * i + 1]),
                        "timer read"))
            return -1;
        ms[i] = t;
        tags[i] = g_ttag[(size_t)i];
    }
    return n;
}

}  // namespace tp
