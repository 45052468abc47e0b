// C ABI of the Fiat-Shamir transcript (include/native_fp2.h, "transcript"):
// host calls on one state in host memory, and batched device calls on arrays of
// states in device memory (one thread per state), so that the per-frame
// transcripts of a batch can absorb their claims and draw their next challenges
// without a round trip to the host.
#include <stdint.h>
#include <string.h>

#include "runtime.h"
#include "transcript.cuh"
#include "../../include/native_fp2.h"

namespace {

using tp::fs::State;

constexpr int kMaxLabel = 64;

struct Label {
    uint8_t b[kMaxLabel];
    uint32_t len;
};

bool make_label(const char* label, Label* L, const char* who)
{
    if (!label) {
        tp::set_error(tp::TP_ERR_ARG, "%s: null label", who);
        return false;
    }
    const size_t n = strlen(label);
    if (n > (size_t)kMaxLabel) {
        tp::set_error(tp::TP_ERR_ARG, "%s: label longer than %d bytes", who, kMaxLabel);
        return false;
    }
    memcpy(L->b, label, n);
    L->len = (uint32_t)n;
    return true;
}

__global__ void put_fp2s_kernel(State* __restrict__ st, int n, const ulonglong2* __restrict__ vals, int k)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    State s = st[i];
    for (int j = 0; j < k; ++j) {
        const ulonglong2 v = vals[(long long)i * k + j];   // packed {re, im}
        tp::fs::put_fp2(s, v.x, v.y);
    }
    st[i] = s;
}

__global__ void rand_ext_kernel(State* __restrict__ st, int n, Label L, ulonglong2* __restrict__ out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    State s = st[i];
    unsigned long long re, im;
    tp::fs::rand_ext(s, L.b, L.len, (uint64_t*)&re, (uint64_t*)&im);
    st[i] = s;
    out[i] = make_ulonglong2(re, im);
}

bool state_ok(const void* state, const char* who)
{
    if (!state) {
        tp::set_error(tp::TP_ERR_ARG, "%s: null state", who);
        return false;
    }
    return true;
}

}  // namespace

extern "C" {

int tp_fs_state_bytes(void) { return (int)sizeof(State); }

int tp_fs_init(void* state, const char* protocol)
{
    tp::clear_error();
    if (!state_ok(state, "tp_fs_init") || !protocol) {
        if (!protocol) tp::set_error(tp::TP_ERR_ARG, "tp_fs_init: null protocol");
        return -1;
    }
    State& s = *static_cast<State*>(state);
    tp::fs::init(s);
    const char* head = "TruePix,";
    tp::fs::absorb(s, reinterpret_cast<const uint8_t*>(head), strlen(head));
    tp::fs::absorb(s, reinterpret_cast<const uint8_t*>(protocol), strlen(protocol));
    tp::fs::absorb(s, reinterpret_cast<const uint8_t*>(","), 1);
    const char* tag = "binhash1,";
    tp::fs::absorb(s, reinterpret_cast<const uint8_t*>(tag), strlen(tag));
    return 0;
}

int tp_fs_put_u64s(void* state, const uint64_t* v, size_t n)
{
    tp::clear_error();
    if (!state_ok(state, "tp_fs_put_u64s")) return -1;
    if (n == 0 || n > 0xFFFFFFFFu || !v) {
        tp::set_error(tp::TP_ERR_ARG, "tp_fs_put_u64s: need 1 <= n < 2^32 values");
        return -1;
    }
    tp::fs::put_u64s(*static_cast<State*>(state), v, n);
    return 0;
}

int tp_fs_put_fp2s(void* state, const uint64_t* re, const uint64_t* im, size_t n)
{
    tp::clear_error();
    if (!state_ok(state, "tp_fs_put_fp2s")) return -1;
    if (n && (!re || !im)) {
        tp::set_error(tp::TP_ERR_ARG, "tp_fs_put_fp2s: null values");
        return -1;
    }
    State& s = *static_cast<State*>(state);
    for (size_t i = 0; i < n; ++i) tp::fs::put_fp2(s, re[i], im[i]);
    return 0;
}

int tp_fs_put_str(void* state, const char* str)
{
    tp::clear_error();
    if (!state_ok(state, "tp_fs_put_str")) return -1;
    if (!str) {
        tp::set_error(tp::TP_ERR_ARG, "tp_fs_put_str: null string");
        return -1;
    }
    tp::fs::put_str(*static_cast<State*>(state), reinterpret_cast<const uint8_t*>(str), (uint32_t)strlen(str));
    return 0;
}

int tp_fs_rand_scalar(void* state, uint64_t* out)
{
    tp::clear_error();
    if (!state_ok(state, "tp_fs_rand_scalar") || !out) return -1;
    *out = tp::fs::rand_scalar(*static_cast<State*>(state));
    return 0;
}

int tp_fs_rand_ext(void* state, const char* label, uint64_t* re, uint64_t* im)
{
    tp::clear_error();
    Label L;
    if (!state_ok(state, "tp_fs_rand_ext") || !make_label(label, &L, "tp_fs_rand_ext")) return -1;
    if (!re || !im) {
        tp::set_error(tp::TP_ERR_ARG, "tp_fs_rand_ext: null output");
        return -1;
    }
    tp::fs::rand_ext(*static_cast<State*>(state), L.b, L.len, re, im);
    return 0;
}

int tp_fs_digest(const void* state, unsigned char* out32)
{
    tp::clear_error();
    if (!state_ok(state, "tp_fs_digest") || !out32) return -1;
    tp::fs::digest(*static_cast<const State*>(state), out32);
    return 0;
}

int tp_fs_put_fp2s_dev(void* d_states, int n, const void* d_vals, int k, void* stream)
{
    tp::clear_error();
    if (!tp::ctx()) return -1;
    if (!d_states || n < 1 || k < 0 || (k > 0 && !d_vals)) {
        tp::set_error(tp::TP_ERR_ARG, "tp_fs_put_fp2s_dev: bad arguments");
        return -1;
    }
    if (k == 0) return 0;
    put_fp2s_kernel<<<(n + 127) / 128, 128, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
        static_cast<State*>(d_states), n, static_cast<const ulonglong2*>(d_vals), k);
    return tp::cuda_failed(cudaGetLastError(), "transcript put") ? -1 : 0;
}

int tp_fs_rand_ext_dev(void* d_states, int n, const char* label, void* d_out, void* stream)
{
    tp::clear_error();
    if (!tp::ctx()) return -1;
    Label L;
    if (!make_label(label, &L, "tp_fs_rand_ext_dev")) return -1;
    if (!d_states || n < 1 || !d_out) {
        tp::set_error(tp::TP_ERR_ARG, "tp_fs_rand_ext_dev: bad arguments");
        return -1;
    }
    rand_ext_kernel<<<(n + 127) / 128, 128, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
        static_cast<State*>(d_states), n, L, static_cast<ulonglong2*>(d_out));
    return tp::cuda_failed(cudaGetLastError(), "transcript rand_ext") ? -1 : 0;
}

}  // extern "C"
