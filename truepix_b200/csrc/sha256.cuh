// SHA-256 (FIPS 180-4) of one 64-byte message, the only hash the Orion commit
// path uses (TruePix-main/Orion/Orion_nonzk/include/infrastructure/my_hhash.h:46-54:
// a full SHA-256 of 64 bytes, i.e. the message block plus the fixed padding block).
//
// Digests are kept as eight 32-bit state words (big-endian words of the digest
// bytes). A message block is sixteen big-endian words; the padding block of a
// 64-byte message is a constant, so its expanded schedule is a constant too and
// is folded into the round constants at compile time (no schedule work for the
// second compression). Host and device share the code so that constant leaves
// (the all-zero row chain, SHA-256 of 64 zero bytes) are computed on the host.
#pragma once
#include <cstdint>

namespace tp {
namespace sha {

struct Tables {
    uint32_t k[64];
    uint32_t pad_kw[64];  // k[t] + w[t] of the padding block of a 64-byte message
};

__host__ __device__ constexpr uint32_t rotr_c(uint32_t x, int n) { return (x >> n) | (x << (32 - n)); }

__host__ __device__ constexpr Tables make_tables()
{
    Tables t{};
    const uint32_t k[64] = {
        0x428a2f98u, 0x71374491u, 0xb5c0fbcfu, 0xe9b5dba5u, 0x3956c25bu, 0x59f111f1u, 0x923f82a4u, 0xab1c5ed5u,
        0xd807aa98u, 0x12835b01u, 0x243185beu, 0x550c7dc3u, 0x72be5d74u, 0x80deb1feu, 0x9bdc06a7u, 0xc19bf174u,
        0xe49b69c1u, 0xefbe4786u, 0x0fc19dc6u, 0x240ca1ccu, 0x2de92c6fu, 0x4a7484aau, 0x5cb0a9dcu, 0x76f988dau,
        0x983e5152u, 0xa831c66du, 0xb00327c8u, 0xbf597fc7u, 0xc6e00bf3u, 0xd5a79147u, 0x06ca6351u, 0x14292967u,
        0x27b70a85u, 0x2e1b2138u, 0x4d2c6dfcu, 0x53380d13u, 0x650a7354u, 0x766a0abbu, 0x81c2c92eu, 0x92722c85u,
        0xa2bfe8a1u, 0xa81a664bu, 0xc24b8b70u, 0xc76c51a3u, 0xd192e819u, 0xd6990624u, 0xf40e3585u, 0x106aa070u,
        0x19a4c116u, 0x1e376c08u, 0x2748774cu, 0x34b0bcb5u, 0x391c0cb3u, 0x4ed8aa4au, 0x5b9cca4fu, 0x682e6ff3u,
        0x748f82eeu, 0x78a5636fu, 0x84c87814u, 0x8cc70208u, 0x90befffau, 0xa4506cebu, 0xbef9a3f7u, 0xc67178f2u};
    uint32_t w[64] = {};
    w[0] = 0x80000000u;  // 0x80 terminator right after the 64 message bytes
    w[15] = 512u;        // message length in bits
    for (int i = 16; i < 64; ++i) {
        const uint32_t s0 = rotr_c(w[i - 15], 7) ^ rotr_c(w[i - 15], 18) ^ (w[i - 15] >> 3);
        const uint32_t s1 = rotr_c(w[i - 2], 17) ^ rotr_c(w[i - 2], 19) ^ (w[i - 2] >> 10);
        w[i] = w[i - 16] + s0 + w[i - 7] + s1;
    }
    for (int i = 0; i < 64; ++i) {
        t.k[i] = k[i];
        t.pad_kw[i] = k[i] + w[i];
    }
    return t;
}

__host__ __device__ __forceinline__ uint32_t rotr(uint32_t x, int n)
{
#ifdef __CUDA_ARCH__
    return __funnelshift_r(x, x, n);
#else
    return (x >> n) | (x << (32 - n));
#endif
}

__host__ __device__ __forceinline__ uint32_t bswap32(uint32_t x)
{
#ifdef __CUDA_ARCH__
    return __byte_perm(x, 0, 0x0123);
#else
    return __builtin_bswap32(x);
#endif
}

__host__ __device__ __forceinline__ void init(uint32_t st[8])
{
    st[0] = 0x6a09e667u; st[1] = 0xbb67ae85u; st[2] = 0x3c6ef372u; st[3] = 0xa54ff53au;
    st[4] = 0x510e527fu; st[5] = 0x9b05688cu; st[6] = 0x1f83d9abu; st[7] = 0x5be0cd19u;
}

// Additions. On the device the SHA-256 rounds are bound by the integer ALU pipe
// (funnel shifts and LOP3 for the sigma/choice/majority functions); routing the
// additions through the multiply-add pipe as x * one + y, with `one` == 1 known
// only at run time, takes them off that pipe. The host adds directly.
struct AddAlu {
    __host__ __device__ __forceinline__ uint32_t operator()(uint32_t a, uint32_t b) const { return a + b; }
};
struct AddMad {
    uint32_t one;   // 1, passed in at run time
    __host__ __device__ __forceinline__ uint32_t operator()(uint32_t a, uint32_t b) const { return a * one + b; }
};

#define TP_SHA_ROUND(a, b, c, d, e, f, g, h, kw)                                          \
    do {                                                                                  \
        const uint32_t s1 = rotr(e, 6) ^ rotr(e, 11) ^ rotr(e, 25);                       \
        const uint32_t ch = (e & f) ^ (~e & g);                                           \
        const uint32_t t1 = add(add(add(h, s1), ch), (kw));                               \
        const uint32_t s0 = rotr(a, 2) ^ rotr(a, 13) ^ rotr(a, 22);                       \
        const uint32_t mj = (a & b) ^ (a & c) ^ (b & c);                                  \
        d = add(d, t1);                                                                   \
        h = add(t1, add(s0, mj));                                                         \
    } while (0)

// one compression of the message block w[16] into st[8] (w is consumed as the
// rolling schedule)
template <class Add>
__host__ __device__ __forceinline__ void compress(uint32_t st[8], uint32_t w[16], Add add)
{
    constexpr Tables T = make_tables();
    uint32_t a = st[0], b = st[1], c = st[2], d = st[3], e = st[4], f = st[5], g = st[6], h = st[7];
#pragma unroll
    for (int i = 0; i < 64; i += 8) {
        if (i >= 16) {
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const int t = i + j;
                const uint32_t x = w[(t - 15) & 15], y = w[(t - 2) & 15];
                w[t & 15] = add(add(w[t & 15], rotr(x, 7) ^ rotr(x, 18) ^ (x >> 3)),
                                add(w[(t - 7) & 15], rotr(y, 17) ^ rotr(y, 19) ^ (y >> 10)));
            }
        }
        TP_SHA_ROUND(a, b, c, d, e, f, g, h, add(w[(i + 0) & 15], T.k[i + 0]));
        TP_SHA_ROUND(h, a, b, c, d, e, f, g, add(w[(i + 1) & 15], T.k[i + 1]));
        TP_SHA_ROUND(g, h, a, b, c, d, e, f, add(w[(i + 2) & 15], T.k[i + 2]));
        TP_SHA_ROUND(f, g, h, a, b, c, d, e, add(w[(i + 3) & 15], T.k[i + 3]));
        TP_SHA_ROUND(e, f, g, h, a, b, c, d, add(w[(i + 4) & 15], T.k[i + 4]));
        TP_SHA_ROUND(d, e, f, g, h, a, b, c, add(w[(i + 5) & 15], T.k[i + 5]));
        TP_SHA_ROUND(c, d, e, f, g, h, a, b, add(w[(i + 6) & 15], T.k[i + 6]));
        TP_SHA_ROUND(b, c, d, e, f, g, h, a, add(w[(i + 7) & 15], T.k[i + 7]));
    }
    st[0] = add(st[0], a); st[1] = add(st[1], b); st[2] = add(st[2], c); st[3] = add(st[3], d);
    st[4] = add(st[4], e); st[5] = add(st[5], f); st[6] = add(st[6], g); st[7] = add(st[7], h);
}

// the second compression of a 64-byte message: constant block, constant schedule
template <class Add>
__host__ __device__ __forceinline__ void compress_pad64(uint32_t st[8], Add add)
{
    constexpr Tables T = make_tables();
    uint32_t a = st[0], b = st[1], c = st[2], d = st[3], e = st[4], f = st[5], g = st[6], h = st[7];
#pragma unroll
    for (int i = 0; i < 64; i += 8) {
        TP_SHA_ROUND(a, b, c, d, e, f, g, h, T.pad_kw[i + 0]);
        TP_SHA_ROUND(h, a, b, c, d, e, f, g, T.pad_kw[i + 1]);
        TP_SHA_ROUND(g, h, a, b, c, d, e, f, T.pad_kw[i + 2]);
        TP_SHA_ROUND(f, g, h, a, b, c, d, e, T.pad_kw[i + 3]);
        TP_SHA_ROUND(e, f, g, h, a, b, c, d, T.pad_kw[i + 4]);
        TP_SHA_ROUND(d, e, f, g, h, a, b, c, T.pad_kw[i + 5]);
        TP_SHA_ROUND(c, d, e, f, g, h, a, b, T.pad_kw[i + 6]);
        TP_SHA_ROUND(b, c, d, e, f, g, h, a, T.pad_kw[i + 7]);
    }
    st[0] = add(st[0], a); st[1] = add(st[1], b); st[2] = add(st[2], c); st[3] = add(st[3], d);
    st[4] = add(st[4], e); st[5] = add(st[5], f); st[6] = add(st[6], g); st[7] = add(st[7], h);
}

#ifdef __CUDACC__
// round constants (and the padding block's k + w) for the device's compact form
static __constant__ Tables kShaTables = make_tables();

// One compression in compact form: four passes over a 16-round body (the
// schedule's rolling index and the round variables' rotation repeat every 16
// rounds, so the body indexes registers statically) with the round constants
// read from constant memory. A quarter of the fully unrolled code: the leaf and
// tree kernels, which keep one hash in flight per thread, then run from the
// instruction cache instead of streaming ~40 KB of straight-line code per hash.
// kSched: message block w (consumed as the rolling schedule); otherwise the
// constant padding block, K holding its k + w.
template <bool kSched, class Add>
__device__ __forceinline__ void compress_compact(uint32_t st[8], uint32_t w[16], const uint32_t* K, Add add)
{
    uint32_t a = st[0], b = st[1], c = st[2], d = st[3], e = st[4], f = st[5], g = st[6], h = st[7];
#pragma unroll 1
    for (int i = 0; i < 64; i += 16) {
#pragma unroll
        for (int j = 0; j < 16; j += 8) {
            if (kSched && i > 0) {
#pragma unroll
                for (int q = 0; q < 8; ++q) {
                    const int t = j + q;    // w[t] holds word i + t - 16 here
                    const uint32_t x = w[(t + 1) & 15], y = w[(t + 14) & 15];
                    w[t] = add(add(w[t], rotr(x, 7) ^ rotr(x, 18) ^ (x >> 3)),
                               add(w[(t + 9) & 15], rotr(y, 17) ^ rotr(y, 19) ^ (y >> 10)));
                }
            }
#define TP_SHA_KW(q) (kSched ? add(w[j + q], K[i + j + q]) : K[i + j + q])
            TP_SHA_ROUND(a, b, c, d, e, f, g, h, TP_SHA_KW(0));
            TP_SHA_ROUND(h, a, b, c, d, e, f, g, TP_SHA_KW(1));
            TP_SHA_ROUND(g, h, a, b, c, d, e, f, TP_SHA_KW(2));
            TP_SHA_ROUND(f, g, h, a, b, c, d, e, TP_SHA_KW(3));
            TP_SHA_ROUND(e, f, g, h, a, b, c, d, TP_SHA_KW(4));
            TP_SHA_ROUND(d, e, f, g, h, a, b, c, TP_SHA_KW(5));
            TP_SHA_ROUND(c, d, e, f, g, h, a, b, TP_SHA_KW(6));
            TP_SHA_ROUND(b, c, d, e, f, g, h, a, TP_SHA_KW(7));
#undef TP_SHA_KW
        }
    }
    st[0] = add(st[0], a); st[1] = add(st[1], b); st[2] = add(st[2], c); st[3] = add(st[3], d);
    st[4] = add(st[4], e); st[5] = add(st[5], f); st[6] = add(st[6], g); st[7] = add(st[7], h);
}
#endif

// SHA-256 of the 64-byte message given as 16 big-endian words; out = state words
template <class Add = AddAlu>
__host__ __device__ __forceinline__ void hash64(uint32_t w[16], uint32_t out[8], Add add = Add())
{
    init(out);
#ifdef __CUDA_ARCH__
    compress_compact<true>(out, w, kShaTables.k, add);
    compress_compact<false>(out, w, kShaTables.pad_kw, add);
#else
    compress(out, w, add);
    compress_pad64(out, add);
#endif
}

// The message words of a field element (16 bytes: u64 img then u64 real, both
// little-endian, the reference's memory order) -- 4 big-endian words.
__host__ __device__ __forceinline__ void fe_words(uint64_t img, uint64_t real, uint32_t* w)
{
    w[0] = bswap32((uint32_t)img);
    w[1] = bswap32((uint32_t)(img >> 32));
    w[2] = bswap32((uint32_t)real);
    w[3] = bswap32((uint32_t)(real >> 32));
}

}  // namespace sha
}  // namespace tp
