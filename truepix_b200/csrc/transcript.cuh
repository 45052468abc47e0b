// Fiat-Shamir transcript in the binary format of the reference prover
// (TruePix-main/libTruePix/fiatshamir.py): one running SHA-256 over everything
// absorbed, challenges drawn from digests of the running state.
//
//   init:        "TruePix," || protocol || "," || "binhash1,"          (:70-74)
//   put(list of u64 ints):  0x01 || LE32(count) || LE64 each          (:112-120)
//   put(Fp2):               0x03 || LE64(real) || LE64(imag)          (:129-131)
//   put(str):               0x04 || LE32(byte length) || UTF-8 bytes  (:132-136)
//   put(int inside a mixed list): 0x02 || LE64;  put(None): 0x05    (:126-138)
//   rand_scalar: absorb [rnum] (a one-int list), rnum += 1, take the low 61
//                bits of the digest read as a big-endian integer, again while
//                the value is >= p (:141-148)
//   rand_ext(label): "ext", label, "real" -> rand_scalar; "ext", label,
//                "imag" -> rand_scalar (:150-162)
//
// The state is a plain struct (the SHA-256 chaining words, the pending partial
// block, the byte count and the challenge counter), so it can move between host
// and device memory by a copy; host and device run the same code.
#pragma once
#include <stdint.h>

#include "fp2.cuh"
#include "sha256.cuh"

namespace tp {
namespace fs {

struct State {
    uint32_t h[8];
    uint8_t buf[64];
    uint64_t total;   // bytes absorbed
    uint64_t rnum;    // rand_scalar's counter
    uint32_t nbuf;    // bytes pending in buf
    uint32_t pad;
};
static_assert(sizeof(State) == 120, "transcript state layout");

TP_HD void block(State& s)
{
    uint32_t w[16];
#pragma unroll
    for (int i = 0; i < 16; ++i)
        w[i] = ((uint32_t)s.buf[4 * i] << 24) | ((uint32_t)s.buf[4 * i + 1] << 16) | ((uint32_t)s.buf[4 * i + 2] << 8) |
               (uint32_t)s.buf[4 * i + 3];
#ifdef __CUDA_ARCH__
    sha::compress_compact<true>(s.h, w, sha::kShaTables.k, sha::AddAlu{});
#else
    sha::compress(s.h, w, sha::AddAlu{});
#endif
}

// one byte into the running hash
TP_HD void absorb_byte(State& s, uint8_t b)
{
    s.buf[s.nbuf++] = b;
    if (s.nbuf == 64) {
        block(s);
        s.nbuf = 0;
    }
    s.total += 1;
}

// bytes from memory (the host entry points' caller-owned data)
TP_HD void absorb(State& s, const uint8_t* p, uint64_t n)
{
    for (uint64_t i = 0; i < n; ++i) absorb_byte(s, p[i]);
}

// the low `bytes` bytes of v, least significant first
TP_HD void absorb_le(State& s, uint64_t v, int bytes)
{
    for (int i = 0; i < bytes; ++i) absorb_byte(s, (uint8_t)(v >> (8 * i)));
}

// A label of at most 32 bytes held by value in four 64-bit words (byte i in
// bits 8 (i mod 8) of word i / 8). Device code builds, passes and absorbs labels
// only in this form: no pointer to a local byte array is handed to the inlined
// hash code (on sm_100a such a pointer, passed down through the fully inlined
// draw, was observed to read the wrong bytes).
struct Label {
    uint64_t w0, w1, w2, w3;
    uint32_t len;
};

TP_HD Label label_empty()
{
    Label L;
    L.w0 = L.w1 = L.w2 = L.w3 = 0;
    L.len = 0;
    return L;
}

// append one byte (ignored past 32)
TP_HD void label_push(Label& L, uint8_t b)
{
    const uint64_t v = (uint64_t)b << (8 * (L.len & 7));
    const uint32_t q = L.len >> 3;
    L.w0 |= q == 0 ? v : 0;
    L.w1 |= q == 1 ? v : 0;
    L.w2 |= q == 2 ? v : 0;
    L.w3 |= q == 3 ? v : 0;
    L.len += q < 4 ? 1 : 0;
}

// a label from a string literal of at most 32 characters
template <int N>
TP_HD Label label_lit(const char (&str)[N])
{
    static_assert(N - 1 <= 32, "labels hold at most 32 bytes");
    Label L = label_empty();
#pragma unroll
    for (int i = 0; i < N - 1; ++i) label_push(L, (uint8_t)str[i]);
    return L;
}

// the decimal digits of v (|v| < 2^31) appended, as Python's str(int) writes them
TP_HD void label_decimal(Label& L, long long v)
{
    if (v < 0) {
        label_push(L, '-');
        v = -v;
    }
    long long p = 1;
    while (p <= v / 10) p *= 10;
    for (; p > 0; p /= 10) {
        label_push(L, (uint8_t)('0' + (v / p) % 10));
    }
}

TP_HD uint8_t label_byte(const Label& L, int i)
{
    const uint64_t w = i < 8 ? L.w0 : i < 16 ? L.w1 : i < 24 ? L.w2 : L.w3;
    return (uint8_t)(w >> (8 * (i & 7)));
}

TP_HD void init(State& s)
{
    sha::init(s.h);
    s.nbuf = 0;
    s.total = 0;
    s.rnum = 0;
    s.pad = 0;
}

// put(list of ints), every value below 2^64 (the reference's array('Q') path)
TP_HD void put_u64s(State& s, const uint64_t* v, uint64_t n)
{
    absorb_byte(s, 0x01);
    absorb_le(s, n, 4);
    for (uint64_t i = 0; i < n; ++i) absorb_le(s, v[i], 8);
}

TP_HD void put_fp2(State& s, uint64_t re, uint64_t im)
{
    absorb_byte(s, 0x03);
    absorb_le(s, re, 8);
    absorb_le(s, im, 8);
}

TP_HD void put_str(State& s, const uint8_t* p, uint32_t len)
{
    absorb_byte(s, 0x04);
    absorb_le(s, len, 4);
    absorb(s, p, len);
}

// put(str) of a label held by value
TP_HD void put_label(State& s, const Label& L)
{
    absorb_byte(s, 0x04);
    absorb_le(s, L.len, 4);
#pragma unroll
    for (int i = 0; i < 32; ++i)
        if (i < (int)L.len) absorb_byte(s, label_byte(L, i));
}

// the running state with the SHA-256 padding absorbed: its words are the digest
// of everything absorbed so far (the running state itself is unchanged)
TP_HD State padded(const State& s)
{
    State t = s;
    const uint64_t bits = t.total * 8;
    // pad without counting the padding in `total`
    t.buf[t.nbuf++] = 0x80;
    if (t.nbuf > 56) {
        while (t.nbuf < 64) t.buf[t.nbuf++] = 0;
        block(t);
        t.nbuf = 0;
    }
    while (t.nbuf < 56) t.buf[t.nbuf++] = 0;
    for (int i = 0; i < 8; ++i) t.buf[56 + i] = (uint8_t)(bits >> (56 - 8 * i));
    block(t);
    return t;
}

// the digest bytes (big-endian words)
TP_HD void digest(const State& s, uint8_t out[32])
{
    const State t = padded(s);
    for (int i = 0; i < 8; ++i) {
        out[4 * i] = (uint8_t)(t.h[i] >> 24);
        out[4 * i + 1] = (uint8_t)(t.h[i] >> 16);
        out[4 * i + 2] = (uint8_t)(t.h[i] >> 8);
        out[4 * i + 3] = (uint8_t)t.h[i];
    }
}

// A draw is redrawn only when its 61 bits are all ones (probability 2^-61); the
// loop is bounded all the same, and past the bound returns the value reduced.
// The low 64 bits of the big-endian digest are its last two words.
TP_HD uint64_t rand_scalar(State& s)
{
    uint64_t v = 0;
    for (int it = 0; it < 1000; ++it) {
        // put([rnum]): a one-int list
        absorb_byte(s, 0x01);
        absorb_le(s, 1, 4);
        absorb_le(s, s.rnum, 8);
        s.rnum += 1;
        const State t = padded(s);
        v = (((uint64_t)t.h[6] << 32) | t.h[7]) & P61;
        if (v < P61) return v;
    }
    return v % P61;
}

// rand_ext(label) as an Fp2: "ext", label, "real" -> the real limb; "ext",
// label, "imag" -> the imaginary limb
TP_HD fp2 rand_fp2(State& s, const Label& L)
{
    const Label ext = label_lit("ext"), real = label_lit("real"), imag = label_lit("imag");
    put_label(s, ext);
    put_label(s, L);
    put_label(s, real);
    const uint64_t re = rand_scalar(s);
    put_label(s, ext);
    put_label(s, L);
    put_label(s, imag);
    const uint64_t im = rand_scalar(s);
    return mk(re, im);
}

// the same draw with a label in memory (host entry points: labels of any length)
TP_HD void rand_ext(State& s, const uint8_t* label, uint32_t len, uint64_t* re, uint64_t* im)
{
    const Label ext = label_lit("ext"), real = label_lit("real"), imag = label_lit("imag");
    put_label(s, ext);
    put_str(s, label, len);
    put_label(s, real);
    *re = rand_scalar(s);
    put_label(s, ext);
    put_str(s, label, len);
    put_label(s, imag);
    *im = rand_scalar(s);
}

}  // namespace fs
}  // namespace tp
