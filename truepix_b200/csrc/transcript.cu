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

// ---- VOLE-committed sumcheck round (circuitnizkvec_vole.py:396-418) ----------
// Per frame: the round polynomial's coefficients from the claims at (0, 1, -1, 2)
// (util.interpolate_cubic), each committed with the next correlation (d = c - u
// put, tag v kept), the equality proof of the tags' value at 0 + 1 against the
// previous round's (challenge rand_ext("eq"), (prev - now) * challenge put; the
// value alone, now * challenge, when there is none), the fold challenge
// rand_ext(label) and the next previous value, the tags' polynomial at it.
struct VoleState {
    unsigned long long idx;   // next correlation
    unsigned has_prev, bad;   // bad: the correlations ran out (nothing done)
    tp::fp2 prev;
    tp::fp2 v_elem[4], out_elem[4];   // running sums of tags / coefficients (the final proof of knowledge)
};
static_assert(sizeof(VoleState) == 160, "vole state layout");

__global__ void vole_round_kernel(State* __restrict__ st, VoleState* __restrict__ vs, int n,
                                  const tp::fp2* __restrict__ claims, const tp::fp2* __restrict__ u,
                                  const tp::fp2* __restrict__ v, long long count, Label L,
                                  tp::fp2* __restrict__ chal, tp::fp2* __restrict__ proof)
{
    using namespace tp;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    VoleState w = vs[i];
    if (w.bad || w.idx + 4 > (unsigned long long)count) {
        w.bad = 1;
        vs[i] = w;
        chal[i] = f2zero();
        return;
    }
    State s = st[i];
    const fp2 f0 = claims[4 * i], f1 = claims[4 * i + 1], fm1 = claims[4 * i + 2], f2 = claims[4 * i + 3];
    const u64 half = 1ull << 60, third = 1537228672809129301ull;
    const fp2 a = f2sub(f2zero(), fm1);
    const fp2 b = f2scale(f2add(f1, fm1), half);
    const fp2 c = f2scale(f2add(f1, a), half);
    const fp2 d = f2scale(f2add(f2, a), third);
    const fp2 c2 = f2sub(b, f0);
    const fp2 c3 = f2scale(f2sub(f2sub(d, c), c2), half);
    const fp2 coef[4] = {f0, f2sub(c, c3), c2, c3};
    const long long base = (long long)i * count;
    fp2 tag[4];
    for (int k = 0; k < 4; ++k) {
        tag[k] = v[base + w.idx];
        const fp2 dm = f2sub(coef[k], u[base + w.idx]);
        ++w.idx;
        fs::put_fp2(s, dm.re, dm.im);
        if (proof) proof[5 * i + k] = dm;
        w.v_elem[k] = f2add(w.v_elem[k], tag[k]);
        w.out_elem[k] = f2add(w.out_elem[k], coef[k]);
    }
    const fp2 now = f2add(f2add(f2add(f2add(tag[0], tag[1]), tag[2]), tag[3]), tag[0]);
    const uint8_t eq[2] = {'e', 'q'};
    fp2 e;
    fs::rand_ext(s, eq, 2, reinterpret_cast<uint64_t*>(&e.re), reinterpret_cast<uint64_t*>(&e.im));
    const fp2 vz = w.has_prev ? f2mul(f2sub(w.prev, now), e) : f2mul(now, e);
    fs::put_fp2(s, vz.re, vz.im);
    if (proof) proof[5 * i + 4] = vz;
    fp2 r;
    fs::rand_ext(s, L.b, L.len, reinterpret_cast<uint64_t*>(&r.re), reinterpret_cast<uint64_t*>(&r.im));
    w.prev = f2add(f2mul(f2add(f2mul(f2add(f2mul(tag[3], r), tag[2]), r), tag[1]), r), tag[0]);
    w.has_prev = 1;
    st[i] = s;
    vs[i] = w;
    chal[i] = r;
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

int tp_fs_absorb(void* state, const void* bytes, size_t n)
{
    tp::clear_error();
    if (!state_ok(state, "tp_fs_absorb")) return -1;
    if (n && !bytes) {
        tp::set_error(tp::TP_ERR_ARG, "tp_fs_absorb: null bytes");
        return -1;
    }
    tp::fs::absorb(*static_cast<State*>(state), static_cast<const uint8_t*>(bytes), n);
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

int tp_vole_state_bytes(void) { return (int)sizeof(VoleState); }

int tp_vole_state_init(void* state, uint64_t first_correlation, const uint64_t* prev)
{
    tp::clear_error();
    if (!state_ok(state, "tp_vole_state_init")) return -1;
    if (prev && (prev[0] >= tp::P61 || prev[1] >= tp::P61)) {
        tp::set_error(tp::TP_ERR_ARG, "tp_vole_state_init: previous value is not canonical");
        return -1;
    }
    VoleState w;
    memset(&w, 0, sizeof(w));
    w.idx = first_correlation;
    if (prev) {
        w.has_prev = 1;
        w.prev = tp::mk(prev[0], prev[1]);
    }
    memcpy(state, &w, sizeof(w));
    return 0;
}

int tp_vole_round_dev(void* d_fs_states, void* d_vole_states, int n, const void* d_claims, const void* d_u,
                      const void* d_v, long long count, const char* label, void* d_chal, void* d_proof,
                      void* stream)
{
    tp::clear_error();
    if (!tp::ctx()) return -1;
    Label L;
    if (!make_label(label, &L, "tp_vole_round_dev")) return -1;
    if (!d_fs_states || !d_vole_states || n < 1 || !d_claims || !d_u || !d_v || count < 4 || !d_chal) {
        tp::set_error(tp::TP_ERR_ARG, "tp_vole_round_dev: bad arguments");
        return -1;
    }
    vole_round_kernel<<<(n + 127) / 128, 128, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
        static_cast<State*>(d_fs_states), static_cast<VoleState*>(d_vole_states), n,
        static_cast<const tp::fp2*>(d_claims), static_cast<const tp::fp2*>(d_u), static_cast<const tp::fp2*>(d_v),
        count, L, static_cast<tp::fp2*>(d_chal), static_cast<tp::fp2*>(d_proof));
    return tp::cuda_failed(cudaGetLastError(), "vole round") ? -1 : 0;
}

}  // extern "C"
