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

TP_HD void absorb(State& s, const uint8_t* p, uint64_t n)
{
    for (uint64_t i = 0; i < n; ++i) {
        s.buf[s.nbuf++] = p[i];
        if (s.nbuf == 64) {
            block(s);
            s.nbuf = 0;
        }
    }
    s.total += n;
}

TP_HD void absorb_byte(State& s, uint8_t b) { absorb(s, &b, 1); }

TP_HD void absorb_le(State& s, uint64_t v, int bytes)
{
    uint8_t b[8];
    for (int i = 0; i < bytes; ++i) b[i] = (uint8_t)(v >> (8 * i));
    absorb(s, b, (uint64_t)bytes);
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

// the digest of everything absorbed so far (the running state is unchanged)
TP_HD void digest(const State& s, uint8_t out[32])
{
    State t = s;
    const uint64_t bits = t.total * 8;
    uint8_t pad = 0x80;
    // pad without counting the padding in `total`
    t.buf[t.nbuf++] = pad;
    if (t.nbuf > 56) {
        while (t.nbuf < 64) t.buf[t.nbuf++] = 0;
        block(t);
        t.nbuf = 0;
    }
    while (t.nbuf < 56) t.buf[t.nbuf++] = 0;
    for (int i = 0; i < 8; ++i) t.buf[56 + i] = (uint8_t)(bits >> (56 - 8 * i));
    block(t);
    for (int i = 0; i < 8; ++i) {
        out[4 * i] = (uint8_t)(t.h[i] >> 24);
        out[4 * i + 1] = (uint8_t)(t.h[i] >> 16);
        out[4 * i + 2] = (uint8_t)(t.h[i] >> 8);
        out[4 * i + 3] = (uint8_t)t.h[i];
    }
}

// A draw is redrawn only when its 61 bits are all ones (probability 2^-61); the
// loop is bounded all the same, and past the bound returns the value reduced.
TP_HD uint64_t rand_scalar(State& s)
{
    uint64_t v = 0;
    for (int it = 0; it < 1000; ++it) {
        const uint64_t r = s.rnum;
        put_u64s(s, &r, 1);
        s.rnum += 1;
        uint8_t d[32];
        digest(s, d);
        v = 0;
        for (int i = 24; i < 32; ++i) v = (v << 8) | d[i];
        v &= P61;
        if (v < P61) return v;
    }
    return v % P61;
}

TP_HD void rand_ext(State& s, const uint8_t* label, uint32_t len, uint64_t* re, uint64_t* im)
{
    const uint8_t ext[3] = {'e', 'x', 't'};
    const uint8_t real[4] = {'r', 'e', 'a', 'l'};
    const uint8_t imag[4] = {'i', 'm', 'a', 'g'};
    put_str(s, ext, 3);
    put_str(s, label, len);
    put_str(s, real, 4);
    *re = rand_scalar(s);
    put_str(s, ext, 3);
    put_str(s, label, len);
    put_str(s, imag, 4);
    *im = rand_scalar(s);
}

// rand_ext returned by value as an Fp2. The draw is written to uint64_t
// (unsigned long) locals and converted; writing it through a uint64_t pointer
// into an fp2's unsigned long long limbs would be a strict-aliasing violation,
// which the device compiler may exploit by reading the limbs as never written.
TP_HD fp2 rand_fp2(State& s, const uint8_t* label, uint32_t len)
{
    uint64_t re, im;
    rand_ext(s, label, len, &re, &im);
    return mk(re, im);
}

}  // namespace fs
}  // namespace tp
