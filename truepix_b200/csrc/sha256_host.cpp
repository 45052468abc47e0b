// SHA-256 compression of whole 64-byte blocks on the host with the x86 SHA
// extensions (SHA256RNDS2 / SHA256MSG1 / SHA256MSG2), for the transcript's long
// absorbs (a frame's circuit outputs are 64 MiB). The state is kept in the two
// registers the round instruction works on, {A, B, E, F} and {C, D, G, H}, and
// the message schedule in four registers of four words that roll every four
// rounds (Intel, "Intel SHA Extensions", 2013). Used only when CPUID reports the
// extensions; the portable compression in sha256.cuh serves every other host.
// Many chains at once (a group of frames' transcripts) go through the AVX-512
// multi-buffer compression below, where the CPU and OS support it.
#include <stddef.h>
#include <stdint.h>

#if defined(__x86_64__) || defined(__i386__)
#include <cpuid.h>
#include <immintrin.h>

extern "C" int tp_host_sha_ext_available(void)
{
    unsigned a, b, c, d;
    if (!__get_cpuid(1, &a, &b, &c, &d)) return 0;
    const bool ssse3 = (c >> 9) & 1, sse41 = (c >> 19) & 1;
    if (!__get_cpuid_count(7, 0, &a, &b, &c, &d)) return 0;
    const bool sha = (b >> 29) & 1;
    return ssse3 && sse41 && sha;
}

// h[8]: chaining words; p: nblocks x 64 message bytes; K: the 64 round constants
extern "C" __attribute__((target("sha,sse4.1,ssse3"))) void tp_host_sha_ext_blocks(uint32_t h[8], const uint8_t* p,
                                                                                   size_t nblocks, const uint32_t K[64])
{
    // big-endian message words
    const __m128i bswap = _mm_set_epi64x(0x0c0d0e0f08090a0bULL, 0x0405060700010203ULL);
    __m128i abcd = _mm_shuffle_epi32(_mm_loadu_si128(reinterpret_cast<const __m128i*>(h)), 0xB1);   // b a d c
    __m128i efgh = _mm_shuffle_epi32(_mm_loadu_si128(reinterpret_cast<const __m128i*>(h + 4)), 0x1B);  // h g f e
    __m128i abef = _mm_alignr_epi8(abcd, efgh, 8);     // lanes f e b a
    __m128i cdgh = _mm_blend_epi16(efgh, abcd, 0xF0);  // lanes h g d c
    for (size_t blk = 0; blk < nblocks; ++blk, p += 64) {
        const __m128i abef0 = abef, cdgh0 = cdgh;
        __m128i m[4];
        for (int i = 0; i < 4; ++i)
            m[i] = _mm_shuffle_epi8(_mm_loadu_si128(reinterpret_cast<const __m128i*>(p + 16 * i)), bswap);
#pragma GCC unroll 16
        for (int g = 0; g < 16; ++g) {
            if (g >= 4) {
                // words 4g..4g+3 from the four groups before: W[t-16] + s0(W[t-15]) + W[t-7] + s1(W[t-2])
                const __m128i w7 = _mm_alignr_epi8(m[(g + 3) & 3], m[(g + 2) & 3], 4);
                m[g & 3] = _mm_sha256msg2_epu32(_mm_add_epi32(_mm_sha256msg1_epu32(m[g & 3], m[(g + 1) & 3]), w7),
                                                m[(g + 3) & 3]);
            }
            __m128i wk = _mm_add_epi32(m[g & 3], _mm_loadu_si128(reinterpret_cast<const __m128i*>(K + 4 * g)));
            cdgh = _mm_sha256rnds2_epu32(cdgh, abef, wk);   // rounds 4g, 4g + 1 (result: the new A B E F)
            wk = _mm_shuffle_epi32(wk, 0x0E);
            abef = _mm_sha256rnds2_epu32(abef, cdgh, wk);   // rounds 4g + 2, 4g + 3
        }
        abef = _mm_add_epi32(abef, abef0);
        cdgh = _mm_add_epi32(cdgh, cdgh0);
    }
    const __m128i feba = _mm_shuffle_epi32(abef, 0x1B);   // lanes a b e f
    const __m128i dchg = _mm_shuffle_epi32(cdgh, 0xB1);   // lanes g h c d
    _mm_storeu_si128(reinterpret_cast<__m128i*>(h), _mm_blend_epi16(feba, dchg, 0xF0));      // a b c d
    _mm_storeu_si128(reinterpret_cast<__m128i*>(h + 4), _mm_alignr_epi8(dchg, feba, 8));  // e f g h
}

// N independent chains compressed in lockstep: chain c's state h[c], its blocks
// at p[c]. One chain is bound by the latency of SHA256RNDS2 (each round pair
// needs the previous one's result); interleaving the round pairs of N chains
// keeps the SHA unit busy. The 16 XMM registers the SHA instructions can name
// hold two chains' state and schedules without spilling.
template <int N>
__attribute__((target("sha,sse4.1,ssse3"), always_inline)) inline void sha_ext_lockstep(uint32_t* const* h,
                                                                                        const uint8_t* const* p,
                                                                                        size_t nblocks,
                                                                                        const uint32_t K[64])
{
    const __m128i bswap = _mm_set_epi64x(0x0c0d0e0f08090a0bULL, 0x0405060700010203ULL);
    __m128i abef[N], cdgh[N];
    for (int c = 0; c < N; ++c) {
        const __m128i abcd = _mm_shuffle_epi32(_mm_loadu_si128(reinterpret_cast<const __m128i*>(h[c])), 0xB1);
        const __m128i efgh = _mm_shuffle_epi32(_mm_loadu_si128(reinterpret_cast<const __m128i*>(h[c] + 4)), 0x1B);
        abef[c] = _mm_alignr_epi8(abcd, efgh, 8);
        cdgh[c] = _mm_blend_epi16(efgh, abcd, 0xF0);
    }
    for (size_t blk = 0; blk < nblocks; ++blk) {
        __m128i abef0[N], cdgh0[N], m[N][4];
        for (int c = 0; c < N; ++c) {
            abef0[c] = abef[c];
            cdgh0[c] = cdgh[c];
            const uint8_t* q = p[c] + 64 * blk;
            for (int i = 0; i < 4; ++i)
                m[c][i] = _mm_shuffle_epi8(_mm_loadu_si128(reinterpret_cast<const __m128i*>(q + 16 * i)), bswap);
        }
#pragma GCC unroll 16
        for (int g = 0; g < 16; ++g) {
            const __m128i k = _mm_loadu_si128(reinterpret_cast<const __m128i*>(K + 4 * g));
            for (int c = 0; c < N; ++c) {
                if (g >= 4) {
                    const __m128i w7 = _mm_alignr_epi8(m[c][(g + 3) & 3], m[c][(g + 2) & 3], 4);
                    m[c][g & 3] = _mm_sha256msg2_epu32(
                        _mm_add_epi32(_mm_sha256msg1_epu32(m[c][g & 3], m[c][(g + 1) & 3]), w7), m[c][(g + 3) & 3]);
                }
                const __m128i wk = _mm_add_epi32(m[c][g & 3], k);
                cdgh[c] = _mm_sha256rnds2_epu32(cdgh[c], abef[c], wk);
                abef[c] = _mm_sha256rnds2_epu32(abef[c], cdgh[c], _mm_shuffle_epi32(wk, 0x0E));
            }
        }
        for (int c = 0; c < N; ++c) {
            abef[c] = _mm_add_epi32(abef[c], abef0[c]);
            cdgh[c] = _mm_add_epi32(cdgh[c], cdgh0[c]);
        }
    }
    for (int c = 0; c < N; ++c) {
        const __m128i feba = _mm_shuffle_epi32(abef[c], 0x1B);
        const __m128i dchg = _mm_shuffle_epi32(cdgh[c], 0xB1);
        _mm_storeu_si128(reinterpret_cast<__m128i*>(h[c]), _mm_blend_epi16(feba, dchg, 0xF0));
        _mm_storeu_si128(reinterpret_cast<__m128i*>(h[c] + 4), _mm_alignr_epi8(dchg, feba, 8));
    }
}

// n chains (any n >= 1) of nblocks blocks each, in lockstep pairs
extern "C" __attribute__((target("sha,sse4.1,ssse3"))) void tp_host_sha_ext_multi(uint32_t* const* h,
                                                                                  const uint8_t* const* p, int n,
                                                                                  size_t nblocks,
                                                                                  const uint32_t K[64])
{
    int c = 0;
    for (; c + 2 <= n; c += 2) sha_ext_lockstep<2>(h + c, p + c, nblocks, K);
    if (c < n) sha_ext_lockstep<1>(h + c, p + c, nblocks, K);
}

// SHA-256 of N independent 64-byte messages (the Orion transcript's absorbs and
// draws: each hashes its 32-byte state with up to 32 bytes), digests written as
// bytes. The second block of a 64-byte message is the constant padding block
// (0x80, zeros, bit length 512), so its message schedule plus the round
// constants (pad_wk) is computed once and its rounds need no schedule work; the
// state stays in registers between the two blocks.
namespace {
inline uint32_t rotr32(uint32_t x, int n) { return (x >> n) | (x << (32 - n)); }

struct PadWk {
    uint32_t wk[64];
    explicit PadWk(const uint32_t K[64])
    {
        uint32_t w[64] = {0x80000000u};
        w[15] = 512;
        for (int t = 16; t < 64; ++t) {
            const uint32_t s0 = rotr32(w[t - 15], 7) ^ rotr32(w[t - 15], 18) ^ (w[t - 15] >> 3);
            const uint32_t s1 = rotr32(w[t - 2], 17) ^ rotr32(w[t - 2], 19) ^ (w[t - 2] >> 10);
            w[t] = w[t - 16] + s0 + w[t - 7] + s1;
        }
        for (int t = 0; t < 64; ++t) wk[t] = w[t] + K[t];
    }
};
}  // namespace

template <int N>
__attribute__((target("sha,sse4.1,ssse3"), always_inline)) inline void sha_ext_hash64(const uint8_t* const* in,
                                                                                      uint8_t* const* out,
                                                                                      const uint32_t K[64],
                                                                                      const uint32_t PWK[64])
{
    const __m128i bswap = _mm_set_epi64x(0x0c0d0e0f08090a0bULL, 0x0405060700010203ULL);
    // the initial hash value in the round instruction's lanes: {F E B A}, {H G D C}
    const __m128i abef_iv = _mm_set_epi32(0x6a09e667, 0xbb67ae85, 0x510e527f, 0x9b05688c);
    const __m128i cdgh_iv = _mm_set_epi32(0x3c6ef372, 0xa54ff53a, 0x1f83d9ab, 0x5be0cd19);
    __m128i abef[N], cdgh[N], m[N][4];
    for (int c = 0; c < N; ++c) {
        abef[c] = abef_iv;
        cdgh[c] = cdgh_iv;
        for (int i = 0; i < 4; ++i)
            m[c][i] = _mm_shuffle_epi8(_mm_loadu_si128(reinterpret_cast<const __m128i*>(in[c] + 16 * i)), bswap);
    }
#pragma GCC unroll 16
    for (int g = 0; g < 16; ++g) {
        const __m128i k = _mm_loadu_si128(reinterpret_cast<const __m128i*>(K + 4 * g));
        for (int c = 0; c < N; ++c) {
            if (g >= 4) {
                const __m128i w7 = _mm_alignr_epi8(m[c][(g + 3) & 3], m[c][(g + 2) & 3], 4);
                m[c][g & 3] = _mm_sha256msg2_epu32(_mm_add_epi32(_mm_sha256msg1_epu32(m[c][g & 3], m[c][(g + 1) & 3]), w7),
                                                   m[c][(g + 3) & 3]);
            }
            const __m128i wk = _mm_add_epi32(m[c][g & 3], k);
            cdgh[c] = _mm_sha256rnds2_epu32(cdgh[c], abef[c], wk);
            abef[c] = _mm_sha256rnds2_epu32(abef[c], cdgh[c], _mm_shuffle_epi32(wk, 0x0E));
        }
    }
    __m128i abef1[N], cdgh1[N];
    for (int c = 0; c < N; ++c) {
        abef[c] = abef1[c] = _mm_add_epi32(abef[c], abef_iv);
        cdgh[c] = cdgh1[c] = _mm_add_epi32(cdgh[c], cdgh_iv);
    }
#pragma GCC unroll 16
    for (int g = 0; g < 16; ++g) {
        const __m128i wk = _mm_loadu_si128(reinterpret_cast<const __m128i*>(PWK + 4 * g));
        for (int c = 0; c < N; ++c) {
            cdgh[c] = _mm_sha256rnds2_epu32(cdgh[c], abef[c], wk);
            abef[c] = _mm_sha256rnds2_epu32(abef[c], cdgh[c], _mm_shuffle_epi32(wk, 0x0E));
        }
    }
    for (int c = 0; c < N; ++c) {
        abef[c] = _mm_add_epi32(abef[c], abef1[c]);
        cdgh[c] = _mm_add_epi32(cdgh[c], cdgh1[c]);
        const __m128i feba = _mm_shuffle_epi32(abef[c], 0x1B);
        const __m128i dchg = _mm_shuffle_epi32(cdgh[c], 0xB1);
        const __m128i abcd = _mm_blend_epi16(feba, dchg, 0xF0), efgh = _mm_alignr_epi8(dchg, feba, 8);
        _mm_storeu_si128(reinterpret_cast<__m128i*>(out[c]), _mm_shuffle_epi8(abcd, bswap));
        _mm_storeu_si128(reinterpret_cast<__m128i*>(out[c] + 16), _mm_shuffle_epi8(efgh, bswap));
    }
}

// n messages of 64 bytes (any n >= 1), in lockstep pairs; out[c]: 32 digest bytes
extern "C" __attribute__((target("sha,sse4.1,ssse3"))) void tp_host_sha_ext_hash64(const uint8_t* const* in,
                                                                                   uint8_t* const* out, int n,
                                                                                   const uint32_t K[64])
{
    static const PadWk pad(K);
    int c = 0;
    for (; c + 2 <= n; c += 2) sha_ext_hash64<2>(in + c, out + c, K, pad.wk);
    if (c < n) sha_ext_hash64<1>(in + c, out + c, K, pad.wk);
}

// ---- multi-buffer SHA-256 with AVX-512 ----
// 16 independent chains in the 32-bit lanes of zmm registers (8 in ymm): each
// vector instruction does one step of the same round for every chain (Intel,
// "Fast Multi-buffer IPsec Implementations on Intel Architecture Processors",
// 2010). A round is 17 vector operations: the sigma functions as three rotates
// and one three-way XOR (VPTERNLOGD), choice and majority one VPTERNLOGD each.
// Each chain's next 64-byte block is loaded as one vector (two for 8 lanes) and
// the 16 x 16 word matrix transposed by four rounds of pairwise interleaves
// (register k with register k + L/2), so lane c of W[i] holds word i of chain c.
// One chain alone is slower than with SHA256RNDS2, 16 together are faster.
#define TP_MB_TARGET __attribute__((target("avx512f,avx512vl,avx512bw")))

extern "C" int tp_host_sha_mb_available(void)
{
    unsigned a, b, c, d;
    if (!__get_cpuid(1, &a, &b, &c, &d)) return 0;
    if (!((c >> 27) & 1)) return 0;   // OSXSAVE
    unsigned lo, hi;
    __asm__ volatile("xgetbv" : "=a"(lo), "=d"(hi) : "c"(0));
    if ((lo & 0xE6) != 0xE6) return 0;   // XMM, YMM, opmask and ZMM state enabled by the OS
    if (!__get_cpuid_count(7, 0, &a, &b, &c, &d)) return 0;
    const bool f = (b >> 16) & 1, bw = (b >> 30) & 1, vl = (b >> 31) & 1;
    return f && bw && vl;
}

namespace {

struct Lanes16 {
    using V = __m512i;
    static constexpr int L = 16;
    TP_MB_TARGET static V add(V a, V b) { return _mm512_add_epi32(a, b); }
    template <int n> TP_MB_TARGET static V ror(V a) { return _mm512_ror_epi32(a, n); }
    template <int n> TP_MB_TARGET static V shr(V a) { return _mm512_srli_epi32(a, n); }
    template <int imm> TP_MB_TARGET static V tern(V a, V b, V c) { return _mm512_ternarylogic_epi32(a, b, c, imm); }
    TP_MB_TARGET static V set1(uint32_t k) { return _mm512_set1_epi32((int)k); }
    TP_MB_TARGET static V load(const void* p) { return _mm512_loadu_si512(p); }
    TP_MB_TARGET static void store(void* p, V v) { _mm512_storeu_si512(p, v); }
    TP_MB_TARGET static V bswap(V v)
    {
        return _mm512_shuffle_epi8(v, _mm512_set4_epi32(0x0c0d0e0f, 0x08090a0b, 0x04050607, 0x00010203));
    }
    // lo = a0 b0 a1 b1 ... a7 b7, hi = a8 b8 ... a15 b15
    TP_MB_TARGET static void interleave(V a, V b, V& lo, V& hi)
    {
        lo = _mm512_permutex2var_epi32(a, _mm512_set_epi32(23, 7, 22, 6, 21, 5, 20, 4, 19, 3, 18, 2, 17, 1, 16, 0), b);
        hi = _mm512_permutex2var_epi32(a, _mm512_set_epi32(31, 15, 30, 14, 29, 13, 28, 12, 27, 11, 26, 10, 25, 9, 24, 8),
                                       b);
    }
};

struct Lanes8 {
    using V = __m256i;
    static constexpr int L = 8;
    TP_MB_TARGET static V add(V a, V b) { return _mm256_add_epi32(a, b); }
    template <int n> TP_MB_TARGET static V ror(V a) { return _mm256_ror_epi32(a, n); }
    template <int n> TP_MB_TARGET static V shr(V a) { return _mm256_srli_epi32(a, n); }
    template <int imm> TP_MB_TARGET static V tern(V a, V b, V c) { return _mm256_ternarylogic_epi32(a, b, c, imm); }
    TP_MB_TARGET static V set1(uint32_t k) { return _mm256_set1_epi32((int)k); }
    TP_MB_TARGET static V load(const void* p) { return _mm256_loadu_si256(reinterpret_cast<const __m256i*>(p)); }
    TP_MB_TARGET static void store(void* p, V v) { _mm256_storeu_si256(reinterpret_cast<__m256i*>(p), v); }
    TP_MB_TARGET static V bswap(V v)
    {
        const V m = _mm256_set_epi32(0x0c0d0e0f, 0x08090a0b, 0x04050607, 0x00010203, 0x0c0d0e0f, 0x08090a0b,
                                     0x04050607, 0x00010203);
        return _mm256_shuffle_epi8(v, m);
    }
    TP_MB_TARGET static void interleave(V a, V b, V& lo, V& hi)
    {
        lo = _mm256_permutex2var_epi32(a, _mm256_set_epi32(11, 3, 10, 2, 9, 1, 8, 0), b);
        hi = _mm256_permutex2var_epi32(a, _mm256_set_epi32(15, 7, 14, 6, 13, 5, 12, 4), b);
    }
};

// x[c] lane i -> x[i] lane c for an L x L matrix of words: log2(L) rounds of
// interleaving register k with register k + L/2 (a perfect shuffle of the rows)
template <class T>
TP_MB_TARGET inline void transpose(typename T::V* x)
{
    using V = typename T::V;
    constexpr int L = T::L;
    for (int r = 0; (1 << r) < L; ++r) {
        V y[L];
        for (int k = 0; k < L / 2; ++k) T::interleave(x[k], x[k + L / 2], y[2 * k], y[2 * k + 1]);
        for (int k = 0; k < L; ++k) x[k] = y[k];
    }
}

// one SHA-256 round for every lane: T1 = h + S1(e) + Ch(e, f, g) + wk (wk = K[t] +
// W[t]); d += T1; h = T1 + S0(a) + Maj(a, b, c) (the other words are renamed by the caller)
#define TP_MB_ROUND(a, b, c, d, e, f, g, h, wk)                                                                   \
    {                                                                                                          \
        const V t1 = T::add(T::add(h, T::template tern<0x96>(T::template ror<6>(e), T::template ror<11>(e),     \
                                                             T::template ror<25>(e))),                          \
                            T::add(T::template tern<0xCA>(e, f, g), wk));                                      \
        d = T::add(d, t1);                                                                                     \
        h = T::add(t1, T::add(T::template tern<0x96>(T::template ror<2>(a), T::template ror<13>(a),            \
                                                     T::template ror<22>(a)),                                  \
                              T::template tern<0xE8>(a, b, c)));                                               \
    }

// 16 rounds t0 .. t0 + 15, round t's K[t] + W[t] given by WK(t, i) (i = t mod 16)
#define TP_MB_16_ROUNDS(WK)                                                                                    \
    TP_MB_ROUND(a, b, c, d, e, f, g, hh, WK(t0 + 0, 0));                                                       \
    TP_MB_ROUND(hh, a, b, c, d, e, f, g, WK(t0 + 1, 1));                                                       \
    TP_MB_ROUND(g, hh, a, b, c, d, e, f, WK(t0 + 2, 2));                                                       \
    TP_MB_ROUND(f, g, hh, a, b, c, d, e, WK(t0 + 3, 3));                                                       \
    TP_MB_ROUND(e, f, g, hh, a, b, c, d, WK(t0 + 4, 4));                                                       \
    TP_MB_ROUND(d, e, f, g, hh, a, b, c, WK(t0 + 5, 5));                                                       \
    TP_MB_ROUND(c, d, e, f, g, hh, a, b, WK(t0 + 6, 6));                                                       \
    TP_MB_ROUND(b, c, d, e, f, g, hh, a, WK(t0 + 7, 7));                                                       \
    TP_MB_ROUND(a, b, c, d, e, f, g, hh, WK(t0 + 8, 8));                                                       \
    TP_MB_ROUND(hh, a, b, c, d, e, f, g, WK(t0 + 9, 9));                                                       \
    TP_MB_ROUND(g, hh, a, b, c, d, e, f, WK(t0 + 10, 10));                                                     \
    TP_MB_ROUND(f, g, hh, a, b, c, d, e, WK(t0 + 11, 11));                                                     \
    TP_MB_ROUND(e, f, g, hh, a, b, c, d, WK(t0 + 12, 12));                                                     \
    TP_MB_ROUND(d, e, f, g, hh, a, b, c, WK(t0 + 13, 13));                                                     \
    TP_MB_ROUND(c, d, e, f, g, hh, a, b, WK(t0 + 14, 14));                                                     \
    TP_MB_ROUND(b, c, d, e, f, g, hh, a, WK(t0 + 15, 15));

// chain c's next block (64 bytes at p[c]) into the lanes of W: lane c of W[i] is
// its big-endian word i
template <class T>
TP_MB_TARGET inline void load_block(typename T::V* W, const uint8_t* const* p, size_t off)
{
    if constexpr (T::L == 16) {
        for (int c = 0; c < 16; ++c) W[c] = T::bswap(T::load(p[c] + off));
        transpose<T>(W);
    } else {   // words 0-7 and 8-15 of the 8 chains, transposed separately
        for (int c = 0; c < 8; ++c) W[c] = T::bswap(T::load(p[c] + off));
        for (int c = 0; c < 8; ++c) W[8 + c] = T::bswap(T::load(p[c] + off + 32));
        transpose<T>(W);
        transpose<T>(W + 8);
    }
}

// one block for every lane: s += the compression of W (the schedule is built in W)
template <class T>
TP_MB_TARGET inline void compress(typename T::V* s, typename T::V* W, const uint32_t K[64])
{
    using V = typename T::V;
    V a = s[0], b = s[1], c = s[2], d = s[3], e = s[4], f = s[5], g = s[6], hh = s[7];
#define TP_MB_WK(t, i) T::add(T::set1(K[t]), W[i])
#pragma GCC unroll 4
    for (int t0 = 0; t0 < 64; t0 += 16) {
        if (t0) {   // W[t] = s1(W[t-2]) + W[t-7] + s0(W[t-15]) + W[t-16], 16 at a time in place
            for (int i = 0; i < 16; ++i) {
                const V w2 = W[(i + 14) & 15], w15 = W[(i + 1) & 15];
                const V s1 = T::template tern<0x96>(T::template ror<17>(w2), T::template ror<19>(w2),
                                                    T::template shr<10>(w2));
                const V s0 = T::template tern<0x96>(T::template ror<7>(w15), T::template ror<18>(w15),
                                                    T::template shr<3>(w15));
                W[i] = T::add(T::add(W[i], s0), T::add(W[(i + 9) & 15], s1));
            }
        }
        TP_MB_16_ROUNDS(TP_MB_WK)
    }
#undef TP_MB_WK
    s[0] = T::add(s[0], a);
    s[1] = T::add(s[1], b);
    s[2] = T::add(s[2], c);
    s[3] = T::add(s[3], d);
    s[4] = T::add(s[4], e);
    s[5] = T::add(s[5], f);
    s[6] = T::add(s[6], g);
    s[7] = T::add(s[7], hh);
}

// the padding block of a 64-byte message for every lane: its W[t] + K[t] are the
// constants PWK[t], so there is no schedule
template <class T>
TP_MB_TARGET inline void compress_pad(typename T::V* s, const uint32_t PWK[64])
{
    using V = typename T::V;
    V a = s[0], b = s[1], c = s[2], d = s[3], e = s[4], f = s[5], g = s[6], hh = s[7];
#define TP_MB_PWK(t, i) T::set1(PWK[t])
#pragma GCC unroll 4
    for (int t0 = 0; t0 < 64; t0 += 16) {
        TP_MB_16_ROUNDS(TP_MB_PWK)
    }
#undef TP_MB_PWK
    s[0] = T::add(s[0], a);
    s[1] = T::add(s[1], b);
    s[2] = T::add(s[2], c);
    s[3] = T::add(s[3], d);
    s[4] = T::add(s[4], e);
    s[5] = T::add(s[5], f);
    s[6] = T::add(s[6], g);
    s[7] = T::add(s[7], hh);
}
#undef TP_MB_16_ROUNDS
#undef TP_MB_ROUND

// T::L chains of nblocks blocks: chain c's state h[c], its blocks at p[c]
template <class T>
TP_MB_TARGET void mb_blocks(uint32_t* const* h, const uint8_t* const* p, size_t nblocks, const uint32_t K[64])
{
    using V = typename T::V;
    constexpr int L = T::L;
    alignas(64) uint32_t tmp[8][L];
    for (int w = 0; w < 8; ++w)
        for (int c = 0; c < L; ++c) tmp[w][c] = h[c][w];
    V s[8];
    for (int w = 0; w < 8; ++w) s[w] = T::load(tmp[w]);
    for (size_t blk = 0; blk < nblocks; ++blk) {
        V W[16];
        load_block<T>(W, p, 64 * blk);
        compress<T>(s, W, K);
    }
    for (int w = 0; w < 8; ++w) T::store(tmp[w], s[w]);
    for (int w = 0; w < 8; ++w)
        for (int c = 0; c < L; ++c) h[c][w] = tmp[w][c];
}

// SHA-256 of T::L messages of 64 bytes each (in[c]), digests as bytes (out[c])
template <class T>
TP_MB_TARGET void mb_hash64(const uint8_t* const* in, uint8_t* const* out, const uint32_t K[64],
                            const uint32_t PWK[64])
{
    using V = typename T::V;
    constexpr int L = T::L;
    static const uint32_t iv[8] = {0x6a09e667, 0xbb67ae85, 0x3c6ef372, 0xa54ff53a,
                                   0x510e527f, 0x9b05688c, 0x1f83d9ab, 0x5be0cd19};
    V s[8], W[16];
    for (int w = 0; w < 8; ++w) s[w] = T::set1(iv[w]);
    load_block<T>(W, in, 0);
    compress<T>(s, W, K);
    compress_pad<T>(s, PWK);
    alignas(64) uint32_t tmp[8][L];
    for (int w = 0; w < 8; ++w) T::store(tmp[w], s[w]);
    for (int c = 0; c < L; ++c)
        for (int w = 0; w < 8; ++w) {
            const uint32_t x = tmp[w][c];
            out[c][4 * w] = (uint8_t)(x >> 24);
            out[c][4 * w + 1] = (uint8_t)(x >> 16);
            out[c][4 * w + 2] = (uint8_t)(x >> 8);
            out[c][4 * w + 3] = (uint8_t)x;
        }
}

}  // namespace

// the first n chains, in groups of 16 lanes and then one of 8 where n allows;
// returns how many chains were hashed (the caller hashes the rest another way)
extern "C" TP_MB_TARGET int tp_host_sha_mb_blocks(uint32_t* const* h, const uint8_t* const* p, int n,
                                                  size_t nblocks, const uint32_t K[64])
{
    int c = 0;
    for (; c + 16 <= n; c += 16) mb_blocks<Lanes16>(h + c, p + c, nblocks, K);
    if (c + 8 <= n) {
        mb_blocks<Lanes8>(h + c, p + c, nblocks, K);
        c += 8;
    }
    return c;
}

// SHA-256 of the first n 64-byte messages in groups of 16 lanes and then one of 8
// where n allows; returns how many were hashed (the caller hashes the rest)
extern "C" TP_MB_TARGET int tp_host_sha_mb_hash64(const uint8_t* const* in, uint8_t* const* out, int n,
                                                  const uint32_t K[64])
{
    static const PadWk pad(K);
    int c = 0;
    for (; c + 16 <= n; c += 16) mb_hash64<Lanes16>(in + c, out + c, K, pad.wk);
    if (c + 8 <= n) {
        mb_hash64<Lanes8>(in + c, out + c, K, pad.wk);
        c += 8;
    }
    return c;
}
#undef TP_MB_TARGET

#else

extern "C" int tp_host_sha_ext_available(void) { return 0; }
extern "C" void tp_host_sha_ext_blocks(uint32_t*, const uint8_t*, size_t, const uint32_t*) {}
extern "C" void tp_host_sha_ext_multi(uint32_t* const*, const uint8_t* const*, int, size_t, const uint32_t*) {}
extern "C" void tp_host_sha_ext_hash64(const uint8_t* const*, uint8_t* const*, int, const uint32_t*) {}
extern "C" int tp_host_sha_mb_available(void) { return 0; }
extern "C" int tp_host_sha_mb_blocks(uint32_t* const*, const uint8_t* const*, int, size_t, const uint32_t*) { return 0; }
extern "C" int tp_host_sha_mb_hash64(const uint8_t* const*, uint8_t* const*, int, const uint32_t*) { return 0; }

#endif
