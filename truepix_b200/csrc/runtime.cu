#include "runtime.h"

#include <stdarg.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <condition_variable>
#include <mutex>
#include <thread>
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
// Pinned staging rings for small uploads: a slot is reused once the copy that
// last read it has run (its event). Uploads of a batch's per-frame tables (a few
// KB each, three per frame) take the small ring, whose 1024 slots outlast several
// batches: a ring that wrapped inside one batch would make the launching thread
// wait for copies queued behind the device's earlier work.
struct Ring {
    int slots;
    size_t slot_bytes;
    unsigned char* mem = nullptr;
    std::vector<cudaEvent_t> ev;
    std::vector<bool> used;
    int next = 0;
};
Ring g_small{1024, 16 * 1024};
Ring g_large{64, 256 * 1024};
std::mutex g_ring_mu;

bool ring_upload(Ring& r, void* d_dst, const void* h_src, size_t bytes, cudaStream_t s)
{
    if (!r.mem) {
        if (cuda_failed(cudaHostAlloc((void**)&r.mem, (size_t)r.slots * r.slot_bytes, cudaHostAllocDefault),
                        "pinned staging"))
            return false;
        r.ev.assign((size_t)r.slots, nullptr);
        r.used.assign((size_t)r.slots, false);
        for (int i = 0; i < r.slots; ++i)
            if (cuda_failed(cudaEventCreateWithFlags(&r.ev[(size_t)i], cudaEventDisableTiming), "staging event"))
                return false;
    }
    const int slot = r.next;
    r.next = (r.next + 1) % r.slots;
    if (r.used[(size_t)slot] && cuda_failed(cudaEventSynchronize(r.ev[(size_t)slot]), "staging wait"))
        return false;
    unsigned char* h = r.mem + (size_t)slot * r.slot_bytes;
    memcpy(h, h_src, bytes);
    if (cuda_failed(cudaMemcpyAsync(d_dst, h, bytes, cudaMemcpyHostToDevice, s), "upload")) return false;
    r.used[(size_t)slot] = true;
    return !cuda_failed(cudaEventRecord(r.ev[(size_t)slot], s), "staging record");
}
}  // namespace

bool upload_async(void* d_dst, const void* h_src, size_t bytes, cudaStream_t s)
{
    if (bytes == 0) return true;
    if (!ctx()) return false;
    if (bytes > g_large.slot_bytes) {
        if (cuda_failed(cudaMemcpyAsync(d_dst, h_src, bytes, cudaMemcpyHostToDevice, s), "upload"))
            return false;
        return !cuda_failed(cudaStreamSynchronize(s), "upload");
    }
    std::lock_guard<std::mutex> lock(g_ring_mu);
    return ring_upload(bytes <= g_small.slot_bytes ? g_small : g_large, d_dst, h_src, bytes, s);
}

namespace {

// Host threads that copy one buffer in parts (the caller takes parts too).
// Jobs are serialised by the caller (g_big_mu); the pool lives until exit.
class CopyPool {
public:
    explicit CopyPool(int workers) : n_(workers + 1)
    {
        for (int i = 0; i < workers; ++i) th_.emplace_back([this] { loop(); });
    }
    void copy(void* dst, const void* src, size_t len)
    {
        {
            std::lock_guard<std::mutex> lk(m_);
            dst_ = static_cast<unsigned char*>(dst);
            src_ = static_cast<const unsigned char*>(src);
            len_ = len;
            parts_ = n_;
            taken_ = done_ = 0;
        }
        work_.notify_all();
        for (;;) {
            int part;
            {
                std::lock_guard<std::mutex> lk(m_);
                if (taken_ >= parts_) break;
                part = taken_++;
            }
            run(part);
        }
        std::unique_lock<std::mutex> lk(m_);
        idle_.wait(lk, [this] { return done_ == parts_; });
        parts_ = taken_ = done_ = 0;
    }

private:
    void run(int part)
    {
        const size_t step = (len_ + parts_ - 1) / parts_;
        const size_t lo = std::min(len_, step * part), hi = std::min(len_, lo + step);
        if (hi > lo) memcpy(dst_ + lo, src_ + lo, hi - lo);
        std::lock_guard<std::mutex> lk(m_);
        if (++done_ == parts_) idle_.notify_all();
    }
    void loop()
    {
        for (;;) {
            int part;
            {
                std::unique_lock<std::mutex> lk(m_);
                work_.wait(lk, [this] { return taken_ < parts_; });
                part = taken_++;
            }
            run(part);
        }
    }
    std::vector<std::thread> th_;
    std::mutex m_;
    std::condition_variable work_, idle_;
    unsigned char* dst_ = nullptr;
    const unsigned char* src_ = nullptr;
    size_t len_ = 0;
    const int n_;
    int parts_ = 0, taken_ = 0, done_ = 0;
};

constexpr size_t kBigChunk = 16u << 20;   // bytes per staging buffer
constexpr size_t kBigMin = 4u << 20;      // smaller copies go straight to cudaMemcpyAsync
std::mutex g_big_mu;
CopyPool* g_copy_pool = nullptr;
unsigned char* g_big_stage[2] = {nullptr, nullptr};
cudaEvent_t g_big_ev[2];
bool g_big_used[2] = {false, false};

bool host_pinned(const void* h)
{
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, h) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

// under g_big_mu
bool big_init()
{
    if (g_copy_pool) return true;
    for (int b = 0; b < 2; ++b) {
        if (cuda_failed(cudaHostAlloc((void**)&g_big_stage[b], kBigChunk, cudaHostAllocDefault), "pinned staging"))
            return false;
        if (cuda_failed(cudaEventCreateWithFlags(&g_big_ev[b], cudaEventDisableTiming), "staging event"))
            return false;
    }
    const unsigned hc = std::thread::hardware_concurrency();
    g_copy_pool = new CopyPool((int)std::min(7u, std::max(1u, hc / 2)));
    return true;
}

bool big_wait(int b)
{
    if (!g_big_used[b]) return true;
    g_big_used[b] = false;
    return !cuda_failed(cudaEventSynchronize(g_big_ev[b]), "staging wait");
}

}  // namespace

bool host_to_device(void* d_dst, const void* h_src, size_t bytes, cudaStream_t s)
{
    if (bytes == 0) return true;
    if (bytes < kBigMin || host_pinned(h_src))
        return !cuda_failed(cudaMemcpyAsync(d_dst, h_src, bytes, cudaMemcpyHostToDevice, s), "H2D");
    std::lock_guard<std::mutex> lock(g_big_mu);
    if (!big_init()) return false;
    const unsigned char* h = static_cast<const unsigned char*>(h_src);
    unsigned char* d = static_cast<unsigned char*>(d_dst);
    for (size_t off = 0, k = 0; off < bytes; off += kBigChunk, ++k) {
        const int b = (int)(k & 1);
        const size_t len = std::min(kBigChunk, bytes - off);
        if (!big_wait(b)) return false;
        g_copy_pool->copy(g_big_stage[b], h + off, len);
        if (cuda_failed(cudaMemcpyAsync(d + off, g_big_stage[b], len, cudaMemcpyHostToDevice, s), "H2D") ||
            cuda_failed(cudaEventRecord(g_big_ev[b], s), "staging record"))
            return false;
        g_big_used[b] = true;
    }
    return true;
}

bool device_to_host(void* h_dst, const void* d_src, size_t bytes, cudaStream_t s)
{
    if (bytes == 0) return true;
    if (bytes < kBigMin || host_pinned(h_dst)) {
        return !cuda_failed(cudaMemcpyAsync(h_dst, d_src, bytes, cudaMemcpyDeviceToHost, s), "D2H") &&
               !cuda_failed(cudaStreamSynchronize(s), "synchronize");
    }
    std::lock_guard<std::mutex> lock(g_big_mu);
    if (!big_init()) return false;
    unsigned char* h = static_cast<unsigned char*>(h_dst);
    const unsigned char* d = static_cast<const unsigned char*>(d_src);
    const size_t n_chunks = (bytes + kBigChunk - 1) / kBigChunk;
    // chunk k goes to staging k & 1; chunk k + 1 is in flight while chunk k is copied out
    auto issue = [&](size_t k) {
        const int b = (int)(k & 1);
        const size_t off = k * kBigChunk, len = std::min(kBigChunk, bytes - off);
        if (!big_wait(b)) return false;
        if (cuda_failed(cudaMemcpyAsync(g_big_stage[b], d + off, len, cudaMemcpyDeviceToHost, s), "D2H") ||
            cuda_failed(cudaEventRecord(g_big_ev[b], s), "staging record"))
            return false;
        g_big_used[b] = true;
        return true;
    };
    if (!issue(0)) return false;
    for (size_t k = 0; k < n_chunks; ++k) {
        if (k + 1 < n_chunks && !issue(k + 1)) return false;
        const int b = (int)(k & 1);
        if (!big_wait(b)) return false;
        const size_t off = k * kBigChunk, len = std::min(kBigChunk, bytes - off);
        g_copy_pool->copy(h + off, g_big_stage[b], len);
    }
    return true;
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
