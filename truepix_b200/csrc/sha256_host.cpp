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

#else

extern "C" int tp_host_sha_ext_available(void) { return 0; }
extern "C" void tp_host_sha_ext_blocks(uint32_t*, const uint8_t*, size_t, const uint32_t*) {}
extern "C" void tp_host_sha_ext_multi(uint32_t* const*, const uint8_t* const*, int, size_t, const uint32_t*) {}

#endif
