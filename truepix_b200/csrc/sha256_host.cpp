// SHA-256 compression of whole 64-byte blocks on the host with the x86 SHA
// extensions (SHA256RNDS2 / SHA256MSG1 / SHA256MSG2), for the transcript's long
// absorbs (a frame's circuit outputs are 64 MiB). The state is kept in the two
// registers the round instruction works on, {A, B, E, F} and {C, D, G, H}, and
// the message schedule in four registers of four words that roll every four
// rounds (Intel, "Intel SHA Extensions", 2013). Used only when CPUID reports the
// extensions; the portable compression in sha256.cuh serves every other host.
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

#else

extern "C" int tp_host_sha_ext_available(void) { return 0; }
extern "C" void tp_host_sha_ext_blocks(uint32_t*, const uint8_t*, size_t, const uint32_t*) {}
extern "C" void tp_host_sha_ext_multi(uint32_t* const*, const uint8_t* const*, int, size_t, const uint32_t*) {}
extern "C" void tp_host_sha_ext_hash64(const uint8_t* const*, uint8_t* const*, int, const uint32_t*) {}

#endif
