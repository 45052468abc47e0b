// C ABI of the Fiat-Shamir transcript (include/native_fp2.h, "transcript"):
// host calls on one state in host memory, and batched device calls on arrays of
// states in device memory (one thread per state), so that the per-frame
// transcripts of a batch can absorb their claims and draw their next challenges
// without a round trip to the host.
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <array>
#include <vector>

#include "gkr_internal.cuh"
#include "native_fp2.h"
#include "runtime.h"
#include "transcript.cuh"
#include "vole.cuh"
#include "../../include/native_fp2.h"

extern "C" int tp_host_sha_ext_available(void);
extern "C" void tp_host_sha_ext_blocks(uint32_t h[8], const uint8_t* p, size_t nblocks, const uint32_t K[64]);
extern "C" void tp_host_sha_ext_hash64(const uint8_t* const* in, uint8_t* const* out, int n, const uint32_t K[64]);
extern "C" int tp_host_sha_mb_available(void);
extern "C" int tp_host_sha_mb_blocks(uint32_t* const* h, const uint8_t* const* p, int n, size_t nblocks,
                                     const uint32_t K[64]);
extern "C" int tp_host_sha_mb_hash64(const uint8_t* const* in, uint8_t* const* out, int n, const uint32_t K[64]);
extern "C" void tp_host_sha_ext_multi(uint32_t* const* h, const uint8_t* const* p, int n, size_t nblocks,
                                      const uint32_t K[64]);

namespace {

using tp::fs::State;
static_assert(__BYTE_ORDER__ == __ORDER_LITTLE_ENDIAN__, "the LE64 encoding is the host's own u64 bytes");

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

// a label for device code, held by value (at most 32 bytes)
bool make_device_label(const char* label, tp::fs::Label* L, const char* who)
{
    if (!label) {
        tp::set_error(tp::TP_ERR_ARG, "%s: null label", who);
        return false;
    }
    const size_t n = strlen(label);
    if (n > 32) {
        tp::set_error(tp::TP_ERR_ARG, "%s: a device label holds at most 32 bytes", who);
        return false;
    }
    *L = tp::fs::label_empty();
    for (size_t i = 0; i < n; ++i) tp::fs::label_push(*L, (uint8_t)label[i]);
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

__global__ void rand_ext_kernel(State* __restrict__ st, int n, tp::fs::Label L, ulonglong2* __restrict__ out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    State s = st[i];
    const tp::fp2 r = tp::fs::rand_fp2(s, L);
    st[i] = s;
    out[i] = make_ulonglong2(r.re, r.im);
}

// ---- VOLE-committed early round (vole.cuh), one thread per frame ----------------
using VoleState = tp::vole::State;

// rounds (optional): frame i takes part only while this round k < rounds[i]
__global__ void vole_round_kernel(State* __restrict__ st, VoleState* __restrict__ vs, int n,
                                  const tp::fp2* __restrict__ claims, const tp::fp2* __restrict__ u,
                                  const tp::fp2* __restrict__ v, long long count, tp::fs::Label L,
                                  tp::fp2* __restrict__ chal, tp::fp2* __restrict__ proof,
                                  const int* __restrict__ rounds, int k)
{
    using namespace tp;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || (rounds && k >= rounds[i])) return;
    VoleState w = vs[i];
    State s = st[i];
    fp2 coef[4];
    vole::interpolate_cubic(claims[4 * i], claims[4 * i + 1], claims[4 * i + 2], claims[4 * i + 3], coef);
    const long long base = (long long)i * count;
    fp2 r;
    vole::round(s, w, coef, 4, u + base, v + base, count, L, proof ? proof + 5 * i : nullptr, &r);
    st[i] = s;
    vs[i] = w;
    chal[i] = r;
}

// ---- VOLE-committed rounds of frames each at its own round (the serving loop) ----
// meta[slot] = {round, rounds}: round < 0 means the slot is idle; after its round
// the slot moves to round + 1, or to -1 after its last round.
__global__ void vole_round_slots_kernel(State* __restrict__ st, VoleState* __restrict__ vs, int n,
                                        int2* __restrict__ meta, const tp::fp2* __restrict__ claims,
                                        const tp::fp2* __restrict__ u, const tp::fp2* __restrict__ v,
                                        long long count, int layer, tp::fp2* __restrict__ chal_cur,
                                        tp::fp2* __restrict__ chal_hist, tp::fp2* __restrict__ proof, int max_rounds)
{
    using namespace tp;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int2 m = meta[i];
    if (m.x < 0 || m.x >= m.y || m.x >= max_rounds) return;
    VoleState w = vs[i];
    State s = st[i];
    fp2 coef[4];
    vole::interpolate_cubic(claims[4 * i], claims[4 * i + 1], claims[4 * i + 2], claims[4 * i + 3], coef);
    const long long base = (long long)i * count;
    fp2 r;
    const long long at = (long long)i * max_rounds + m.x;
    vole::round(s, w, coef, 4, u + base, v + base, count, vole::sc_label(layer, m.x), proof ? proof + 5 * at : nullptr,
                &r);
    st[i] = s;
    vs[i] = w;
    chal_cur[i] = r;
    chal_hist[at] = r;
    meta[i] = make_int2(m.x + 1 < m.y ? m.x + 1 : -1, m.y);
}

// ---- host absorbs: whole blocks compressed straight from the caller's bytes,
// with the x86 SHA extensions where the CPU has them (sha256_host.cpp) ----------
constexpr tp::sha::Tables kHostTables = tp::sha::make_tables();

// TRUEPIX_HOST_SHA_PORTABLE=1 selects the portable compression on any CPU
bool host_sha_ext()
{
    static const bool ok = tp_host_sha_ext_available() != 0 && !getenv("TRUEPIX_HOST_SHA_PORTABLE");
    return ok;
}

// TRUEPIX_HOST_SHA_NO_MULTIBUFFER=1 keeps groups of chains off the AVX-512
// multi-buffer compression (the portable setting does too)
bool host_sha_mb()
{
    static const bool ok = tp_host_sha_mb_available() != 0 && !getenv("TRUEPIX_HOST_SHA_PORTABLE") &&
                           !getenv("TRUEPIX_HOST_SHA_NO_MULTIBUFFER");
    return ok;
}

void host_blocks(uint32_t h[8], const uint8_t* p, size_t nblocks)
{
    if (host_sha_ext()) {
        tp_host_sha_ext_blocks(h, p, nblocks, kHostTables.k);
        return;
    }
    for (size_t b = 0; b < nblocks; ++b, p += 64) {
        uint32_t w[16];
        for (int i = 0; i < 16; ++i)
            w[i] = ((uint32_t)p[4 * i] << 24) | ((uint32_t)p[4 * i + 1] << 16) | ((uint32_t)p[4 * i + 2] << 8) |
                   (uint32_t)p[4 * i + 3];
        tp::sha::compress(h, w, tp::sha::AddAlu{});
    }
}

// the same bytes and state as tp::fs::absorb
void host_absorb(State& s, const uint8_t* p, uint64_t n)
{
    s.total += n;
    if (s.nbuf) {
        const uint64_t take = n < 64u - s.nbuf ? n : 64u - s.nbuf;
        memcpy(s.buf + s.nbuf, p, take);
        s.nbuf += (uint32_t)take;
        p += take;
        n -= take;
        if (s.nbuf < 64) return;
        host_blocks(s.h, s.buf, 1);
        s.nbuf = 0;
    }
    const uint64_t nb = n / 64;
    if (nb) {
        host_blocks(s.h, p, nb);
        p += 64 * nb;
        n -= 64 * nb;
    }
    memcpy(s.buf, p, n);
    s.nbuf = (uint32_t)n;
}

void host_absorb_header(State& s, uint8_t tag, uint32_t n)
{
    const uint8_t b[5] = {tag, (uint8_t)n, (uint8_t)(n >> 8), (uint8_t)(n >> 16), (uint8_t)(n >> 24)};
    host_absorb(s, b, 5);
}

// n chains of nblocks whole blocks each: groups of 16 (then 8) in the lanes of
// the AVX-512 multi-buffer compression, the rest with the SHA extensions in
// lockstep pairs
void host_blocks_multi(uint32_t* const* h, const uint8_t* const* p, int n, size_t nblocks)
{
    const int done = host_sha_mb() ? tp_host_sha_mb_blocks(h, p, n, nblocks, kHostTables.k) : 0;
    h += done;
    p += done;
    n -= done;
    if (n == 0) return;
    if (host_sha_ext()) {
        tp_host_sha_ext_multi(h, p, n, nblocks, kHostTables.k);
        return;
    }
    for (int c = 0; c < n; ++c) host_blocks(h[c], p[c], nblocks);
}

// ---- a frame's circuit outputs put into its transcript, computed on the host --
// The output vector (tp_circuit_outputs_pixels_dev's, 64 MiB at 1080p) is
// generated copy by copy from the frame's bytes into a small staging buffer per
// frame and hashed from there: nothing of the size of the vector is written or
// copied. Frames whose transcripts stand at the same offset in their pending
// block hash together, up to kGroup at a time (host_blocks_multi: the lanes of
// the multi-buffer compression, else lockstep pairs).
constexpr int kGroup = 16;

// native_fp2_core.hpp:32-51 on canonical base-field values (as the device kernel)
uint64_t host_gate_value(unsigned type, uint64_t x, uint64_t y)
{
    using tp::fadd;
    using tp::fsub;
    auto mul = [](uint64_t a, uint64_t b) { return tp::fmul(a, b); };
    switch (type) {
    case 0: return mul(x, y);
    case 1: return fadd(x, y);
    case 2: return fsub(x, y);
    case 3: return x;
    case 4: return y;
    case 5: return fsub(fadd(x, y), mul(x, y));
    case 6: return fsub(fadd(x, y), fadd(mul(x, y), mul(x, y)));
    case 7: return fsub(1, x);
    case 8: return fsub(1, mul(x, y));
    case 9: return fsub(fadd(1, mul(x, y)), fadd(x, y));
    case 10: return fsub(fadd(1, fadd(mul(x, y), mul(x, y))), fadd(x, y));
    case 11: return mul(fsub(1, x), y);
    default: return x;
    }
}

struct OutputCircuit {
    int n_copies, n_copies_padded, cs, n_wires, const_idx, n_gates, out_bits;
    uint64_t const_val;
    long long n_bytes;                        // the frame's bytes; past them a copy's inputs are zero
    std::vector<uint32_t> type, src0, src1;   // src: the byte's index, or cs for "zero", cs + 1 for the constant
    std::vector<uint8_t> direct;              // the gate's value is one of its inputs (pass, multiplexer)
};

// copy c's outputs (2^out_bits LE64 values) at out; ext: cs + 2 words of scratch
// (the copy's inputs widened, then zero and the constant, indexed by src)
void copy_outputs(const OutputCircuit& C, const uint8_t* pix, long long c, uint64_t* ext, uint64_t* out)
{
    const int G = 1 << C.out_bits;
    if (c >= C.n_copies) {
        memset(out, 0, 8 * (size_t)G);
        return;
    }
    const uint8_t* row = pix + c * C.cs;
    const long long left = C.n_bytes - c * (long long)C.cs;
    const int cs = C.cs, avail = left >= cs ? cs : left > 0 ? (int)left : 0;
    for (int a = 0; a < avail; ++a) ext[a] = row[a];
    for (int a = avail; a < cs; ++a) ext[a] = 0;
    ext[cs] = 0;
    ext[cs + 1] = C.const_val;
    for (int g = 0; g < C.n_gates; ++g) {
        const uint64_t va = ext[C.src0[g]];
        out[g] = C.direct[g] ? va : host_gate_value(C.type[g], va, ext[C.src1[g]]);
    }
    if (G > C.n_gates) memset(out + C.n_gates, 0, 8 * (size_t)(G - C.n_gates));
}

// the values of copies [c0, c0 + nc) of every frame of a group, hashed in lockstep
void put_outputs_group(State* const* st, const uint8_t* const* pix, int k, const OutputCircuit& C)
{
    constexpr long long kCopiesPerChunk = 16;
    const size_t copy_bytes = (size_t)8 << C.out_bits;
    const size_t cap = 64 + kCopiesPerChunk * copy_bytes;
    std::vector<uint8_t> stage((size_t)k * cap);
    std::vector<uint64_t> ext((size_t)C.cs + 2);
    uint32_t* h[kGroup];
    const uint8_t* p[kGroup];
    size_t fill = st[0]->nbuf;   // equal for every frame of the group
    for (int c = 0; c < k; ++c) memcpy(&stage[(size_t)c * cap], st[c]->buf, fill);
    const uint64_t n_values = (uint64_t)C.n_copies_padded << C.out_bits;
    for (long long c0 = 0; c0 < C.n_copies_padded; c0 += kCopiesPerChunk) {
        const long long nc = C.n_copies_padded - c0 < kCopiesPerChunk ? C.n_copies_padded - c0 : kCopiesPerChunk;
        for (int c = 0; c < k; ++c) {
            uint8_t* base = &stage[(size_t)c * cap] + fill;
            for (long long q = 0; q < nc; ++q)
                copy_outputs(C, pix[c], c0 + q, ext.data(), reinterpret_cast<uint64_t*>(base + q * copy_bytes));
        }
        const size_t total = fill + (size_t)nc * copy_bytes;
        const size_t nblk = total / 64;
        for (int c = 0; c < k; ++c) {
            h[c] = st[c]->h;
            p[c] = &stage[(size_t)c * cap];
        }
        host_blocks_multi(h, p, k, nblk);
        fill = total - 64 * nblk;
        for (int c = 0; c < k; ++c) memmove(&stage[(size_t)c * cap], &stage[(size_t)c * cap] + 64 * nblk, fill);
    }
    for (int c = 0; c < k; ++c) {
        memcpy(st[c]->buf, &stage[(size_t)c * cap], fill);
        st[c]->nbuf = (uint32_t)fill;
        st[c]->total += 8 * n_values;
    }
}

// ---- the Orion opening's transcript (truepix_orion::FsTranscript, orion_fs.cpp) --
// state' = SHA-256(state || chunk || zero pad) for each chunk of <= 32 bytes
struct OrionFs {
    uint8_t state[32];
    uint8_t pool[32];
    int used;
};

void sha256_64(const uint8_t in[64], uint8_t out[32])
{
    if (host_sha_ext()) {       // both blocks in registers, the padding block's schedule precomputed
        const uint8_t* ip = in;
        uint8_t* op = out;
        tp_host_sha_ext_hash64(&ip, &op, 1, kHostTables.k);
        return;
    }
    static const uint8_t kPad[64] = {0x80, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0,
                                     0,    0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0,
                                     0,    0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0x02, 0};
    uint32_t h[8];
    tp::sha::init(h);
    host_blocks(h, in, 1);
    host_blocks(h, kPad, 1);
    for (int i = 0; i < 8; ++i) {
        out[4 * i] = (uint8_t)(h[i] >> 24);
        out[4 * i + 1] = (uint8_t)(h[i] >> 16);
        out[4 * i + 2] = (uint8_t)(h[i] >> 8);
        out[4 * i + 3] = (uint8_t)h[i];
    }
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

namespace tp {

bool launch_vole_round_batch(void* d_states, void* d_vole_states, int n, const void* d_claims, const void* d_u,
                             const void* d_v, long long count, const char* label, void* d_chal, void* d_proof,
                             cudaStream_t s, const int* d_rounds, int k)
{
    fs::Label L;
    if (!make_device_label(label, &L, "vole round")) return false;
    vole_round_kernel<<<(n + 127) / 128, 128, 0, s>>>(
        static_cast<State*>(d_states), static_cast<VoleState*>(d_vole_states), n, static_cast<const fp2*>(d_claims),
        static_cast<const fp2*>(d_u), static_cast<const fp2*>(d_v), count, L, static_cast<fp2*>(d_chal),
        static_cast<fp2*>(d_proof), d_rounds, k);
    return !cuda_failed(cudaGetLastError(), "vole round");
}

}  // namespace tp

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
    host_absorb(*static_cast<State*>(state), static_cast<const uint8_t*>(bytes), n);
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
    State& s = *static_cast<State*>(state);
    host_absorb_header(s, 0x01, (uint32_t)n);
    host_absorb(s, reinterpret_cast<const uint8_t*>(v), 8 * (uint64_t)n);
    return 0;
}

int tp_fs_put_circuit_outputs_pixels(void* const* states, const void* const* pixels, long long n_bytes, int n_frames,
                                     int n_copies, int n_copies_padded, int copy_size, int n_wires, int const_idx,
                                     uint64_t const_val, int n_gates, const int* gate_type, const int* in0,
                                     const int* in1)
{
    tp::clear_error();
    const long long values = n_copies_padded >= 1 && n_gates >= 1
                                 ? ((long long)n_copies_padded << tp_circuit_out_bits(n_gates)) : 0;
    if (!states || !pixels || n_frames < 1 || n_copies < 1 || n_copies_padded < n_copies ||
        (n_copies_padded & (n_copies_padded - 1)) != 0 || copy_size < 1 || n_wires < copy_size ||
        n_wires > (1 << 14) || const_idx >= n_wires || (const_idx >= 0 && const_idx < copy_size) ||
        const_val >= tp::P61 || n_gates < 1 || n_gates > 4096 || !gate_type || !in0 || !in1 ||
        values >= (1ll << 32) || n_bytes < 0) {
        tp::set_error(tp::TP_ERR_ARG, "tp_fs_put_circuit_outputs_pixels: bad arguments");
        return -1;
    }
    OutputCircuit C;
    C.n_copies = n_copies;
    C.n_copies_padded = n_copies_padded;
    C.cs = copy_size;
    C.n_wires = n_wires;
    C.const_idx = const_idx;
    C.const_val = const_val;
    C.n_gates = n_gates;
    C.out_bits = tp_circuit_out_bits(n_gates);
    C.n_bytes = std::min<long long>(n_bytes, (long long)n_copies * copy_size);
    // sources: a byte of the copy (wire < copy_size), the constant (copy_size + 1), else zero (copy_size)
    auto src = [&](int w) -> uint32_t {
        return w < copy_size ? (uint32_t)w : w == const_idx ? (uint32_t)copy_size + 1 : (uint32_t)copy_size;
    };
    for (int g = 0; g < n_gates; ++g) {
        if (gate_type[g] < 0 || gate_type[g] > 12 || in0[g] < 0 || in0[g] >= n_wires || in1[g] < 0 ||
            in1[g] >= n_wires) {
            tp::set_error(tp::TP_ERR_ARG, "tp_fs_put_circuit_outputs_pixels: gate %d out of range", g);
            return -1;
        }
        const int t = gate_type[g];
        const bool right = t == 4;
        C.type.push_back((uint32_t)t);
        C.src0.push_back(src(right ? in1[g] : in0[g]));
        C.src1.push_back(src(in1[g]));
        C.direct.push_back(t == 3 || t == 4 || t == 12);
    }
    for (int f = 0; f < n_frames; ++f) {
        if (!states[f] || !pixels[f]) {
            tp::set_error(tp::TP_ERR_ARG, "tp_fs_put_circuit_outputs_pixels: null state or frame %d", f);
            return -1;
        }
        State& s = *static_cast<State*>(states[f]);
        host_absorb_header(s, 0x01, (uint32_t)values);
    }
    // frames at the same offset hash together, up to kGroup at a time
    std::vector<int> done(n_frames, 0);
    for (int f = 0; f < n_frames; ++f) {
        if (done[f]) continue;
        done[f] = 1;
        State* st[kGroup] = {static_cast<State*>(states[f])};
        const uint8_t* px[kGroup] = {static_cast<const uint8_t*>(pixels[f])};
        int k = 1;
        for (int g = f + 1; g < n_frames && k < kGroup; ++g)
            if (!done[g] && static_cast<State*>(states[g])->nbuf == st[0]->nbuf) {
                done[g] = 1;
                st[k] = static_cast<State*>(states[g]);
                px[k] = static_cast<const uint8_t*>(pixels[g]);
                ++k;
            }
        put_outputs_group(st, px, k, C);
    }
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
    uint8_t buf[17 * 240];
    size_t nb = 0;
    for (size_t i = 0; i < n; ++i) {
        buf[nb] = 0x03;
        memcpy(buf + nb + 1, re + i, 8);
        memcpy(buf + nb + 9, im + i, 8);
        nb += 17;
        if (nb == sizeof(buf) || i + 1 == n) {
            host_absorb(s, buf, nb);
            nb = 0;
        }
    }
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
    State& s = *static_cast<State*>(state);
    const size_t len = strlen(str);
    host_absorb_header(s, 0x04, (uint32_t)len);
    host_absorb(s, reinterpret_cast<const uint8_t*>(str), len);
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
    tp::fs::Label L;
    if (!make_device_label(label, &L, "tp_fs_rand_ext_dev")) return -1;
    if (!d_states || n < 1 || !d_out) {
        tp::set_error(tp::TP_ERR_ARG, "tp_fs_rand_ext_dev: bad arguments");
        return -1;
    }
    rand_ext_kernel<<<(n + 127) / 128, 128, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
        static_cast<State*>(d_states), n, L, static_cast<ulonglong2*>(d_out));
    return tp::cuda_failed(cudaGetLastError(), "transcript rand_ext") ? -1 : 0;
}

int tp_orion_open_queries(const unsigned char* root32, uint64_t N, int use_group1, const uint64_t* r0, int n_r0,
                          const uint64_t* r1, long long n_r1, long long cw_len, int group, int count,
                          long long* col_q)
{
    return tp_orion_open_queries2(root32, N, use_group1, r0, n_r0, r1, n_r1, cw_len, group, count, col_q, nullptr);
}

int tp_orion_open_queries2(const unsigned char* root32, uint64_t N, int use_group1, const uint64_t* r0, int n_r0,
                           const uint64_t* r1, long long n_r1, long long cw_len, int group, int count,
                           long long* col_q, long long* ec_q)
{
    return tp_orion_open_queries_multi(1, &root32, N, &use_group1, &r0, n_r0, &r1, n_r1, cw_len, &group, count, &col_q,
                                       ec_q ? &ec_q : nullptr);
}

int tp_orion_open_queries_multi(int n, const unsigned char* const* roots, uint64_t N, const int* use_group1,
                                const uint64_t* const* r0, int n_r0, const uint64_t* const* r1, long long n_r1,
                                long long cw_len, const int* groups, int count, long long* const* col_q,
                                long long* const* ec_q)
{
    tp::clear_error();
    bool ok = n >= 1 && n <= 64 && roots && use_group1 && r0 && r1 && groups && col_q && n_r0 >= 1 && n_r1 >= 1 &&
              cw_len >= 2 && count >= 0;
    for (int c = 0; ok && c < n; ++c)
        ok = roots[c] && r0[c] && r1[c] && col_q[c] && groups[c] >= -1 && groups[c] <= 1 && (!ec_q || ec_q[c]);
    if (!ok) {
        tp::set_error(tp::TP_ERR_ARG, "tp_orion_open_queries: bad arguments");
        return -1;
    }
    // the n transcripts take the same steps on their own bytes, their hashes in
    // lockstep (multi-buffer lanes, else pairs of interleaved SHA-extension chains)
    std::vector<OrionFs> t((size_t)n);
    std::vector<std::array<uint8_t, 64>> blocks((size_t)n);
    std::vector<const uint8_t*> in((size_t)n);
    std::vector<uint8_t*> out((size_t)n);
    for (OrionFs& x : t) memset(&x, 0, sizeof(x));
    auto hash_all = [&]() {
        // groups of 16 (then 8) in the lanes of the multi-buffer compression, the
        // rest in lockstep pairs on the SHA extensions
        const int done = host_sha_mb() ? tp_host_sha_mb_hash64(in.data(), out.data(), n, kHostTables.k) : 0;
        if (done == n) return;
        if (host_sha_ext()) {
            tp_host_sha_ext_hash64(in.data() + done, out.data() + done, n - done, kHostTables.k);
        } else {
            for (int c = done; c < n; ++c) sha256_64(in[(size_t)c], out[(size_t)c]);
        }
    };
    // absorb of `len` <= 32 bytes, chain c's bytes at src(c)
    auto absorb = [&](auto src, size_t len) {
        for (int c = 0; c < n; ++c) {
            uint8_t* b = blocks[(size_t)c].data();
            memcpy(b, t[(size_t)c].state, 32);
            memcpy(b + 32, src(c), len);
            memset(b + 32 + len, 0, 32 - len);
            in[(size_t)c] = b;
            out[(size_t)c] = t[(size_t)c].state;
        }
        hash_all();
        for (OrionFs& x : t) x.used = 32;
    };
    static const char kDom[] = "truepix/orion-fs/v1";
    static const char kLabel[] = "tensor-open";
    absorb([&](int) { return (const void*)kDom; }, sizeof(kDom) - 1);
    absorb([&](int) { return (const void*)kLabel; }, sizeof(kLabel) - 1);
    absorb([&](int c) { return (const void*)roots[c]; }, 32);
    absorb([&](int) { return (const void*)&N; }, 8);
    std::vector<uint64_t> g1((size_t)n);
    for (int c = 0; c < n; ++c) g1[(size_t)c] = use_group1[c] ? 1 : 0;
    absorb([&](int c) { return (const void*)&g1[(size_t)c]; }, 8);
    for (int i = 0; i < n_r0; ++i) {
        absorb([&](int c) { return (const void*)(r0[c] + 2 * i); }, 8);
        absorb([&](int c) { return (const void*)(r0[c] + 2 * i + 1); }, 8);
    }
    for (long long i = 0; i < n_r1; ++i) {
        absorb([&](int c) { return (const void*)(r1[c] + 2 * i); }, 8);
        absorb([&](int c) { return (const void*)(r1[c] + 2 * i + 1); }, 8);
    }
    // draws: every 4th refills each chain's pool (SHA256(state || 0x01 || 0)) and
    // moves its state on (SHA256(state || 0x02 || 0)), as orion_squeeze
    auto squeeze = [&](std::vector<uint64_t>& v) {
        if (t[0].used + 8 > 32) {
            for (int tag = 1; tag <= 2; ++tag) {
                for (int c = 0; c < n; ++c) {
                    uint8_t* b = blocks[(size_t)c].data();
                    memset(b, 0, 64);
                    memcpy(b, t[(size_t)c].state, 32);
                    b[32] = (uint8_t)tag;
                    in[(size_t)c] = b;
                    out[(size_t)c] = tag == 1 ? t[(size_t)c].pool : t[(size_t)c].state;
                }
                hash_all();
            }
            for (OrionFs& x : t) x.used = 0;
        }
        for (int c = 0; c < n; ++c) {
            memcpy(&v[(size_t)c], t[(size_t)c].pool + t[(size_t)c].used, 8);
            t[(size_t)c].used += 8;
        }
    };
    std::vector<uint64_t> v((size_t)n);
    for (int i = 0; i < count; ++i) {
        squeeze(v);
        for (int c = 0; c < n; ++c) {
            const int group = groups[c];
            const uint64_t size =
                group < 0 ? (uint64_t)cw_len : group == 0 ? (uint64_t)(cw_len + 1) / 2 : (uint64_t)cw_len / 2;
            const uint64_t k = v[(size_t)c] % size;
            col_q[c][i] = group < 0 ? (long long)k : 2 * (long long)k + group;
        }
    }
    // the EC(y1) positions: the next draws, over the whole codeword
    // (linearPC.cpp:573-575; Orion_zk linearPC.cpp:879-880)
    if (ec_q)
        for (int i = 0; i < count; ++i) {
            squeeze(v);
            for (int c = 0; c < n; ++c) ec_q[c][i] = (long long)(v[(size_t)c] % (uint64_t)cw_len);
        }
    return 0;
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

int tp_vole_round_slots_dev(void* d_fs_states, void* d_vole_states, int n_slots, void* d_meta, const void* d_claims,
                            const void* d_u, const void* d_v, long long count, int layer, void* d_chal_cur,
                            void* d_chal_hist, void* d_proof, int max_rounds, void* stream)
{
    tp::clear_error();
    if (!tp::ctx()) return -1;
    if (!d_fs_states || !d_vole_states || n_slots < 1 || !d_meta || !d_claims || !d_u || !d_v || count < 4 ||
        !d_chal_cur || !d_chal_hist || max_rounds < 1 || max_rounds > 64 || layer < 0) {
        tp::set_error(tp::TP_ERR_ARG, "tp_vole_round_slots_dev: bad arguments");
        return -1;
    }
    vole_round_slots_kernel<<<(n_slots + 127) / 128, 128, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
        static_cast<State*>(d_fs_states), static_cast<VoleState*>(d_vole_states), n_slots, static_cast<int2*>(d_meta),
        static_cast<const tp::fp2*>(d_claims), static_cast<const tp::fp2*>(d_u), static_cast<const tp::fp2*>(d_v),
        count, layer, static_cast<tp::fp2*>(d_chal_cur), static_cast<tp::fp2*>(d_chal_hist),
        static_cast<tp::fp2*>(d_proof), max_rounds);
    return tp::cuda_failed(cudaGetLastError(), "vole round slots") ? -1 : 0;
}

int tp_vole_round_dev(void* d_fs_states, void* d_vole_states, int n, const void* d_claims, const void* d_u,
                      const void* d_v, long long count, const char* label, void* d_chal, void* d_proof,
                      void* stream)
{
    tp::clear_error();
    if (!tp::ctx()) return -1;
    tp::fs::Label L;
    if (!make_device_label(label, &L, "tp_vole_round_dev")) return -1;
    if (!d_fs_states || !d_vole_states || n < 1 || !d_claims || !d_u || !d_v || count < 4 || !d_chal) {
        tp::set_error(tp::TP_ERR_ARG, "tp_vole_round_dev: bad arguments");
        return -1;
    }
    vole_round_kernel<<<(n + 127) / 128, 128, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
        static_cast<State*>(d_fs_states), static_cast<VoleState*>(d_vole_states), n,
        static_cast<const tp::fp2*>(d_claims), static_cast<const tp::fp2*>(d_u), static_cast<const tp::fp2*>(d_v),
        count, L, static_cast<tp::fp2*>(d_chal), static_cast<tp::fp2*>(d_proof), nullptr, 0);
    return tp::cuda_failed(cudaGetLastError(), "vole round") ? -1 : 0;
}

}  // extern "C"
