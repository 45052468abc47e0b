// Arithmetic in Fp = Z/(2^61 - 1) and Fp2 = Fp[i]/(i^2 + 1) for sm_100a and host.
//
// Same field and same canonical representation as the reference
// (TruePix-main/native_fp2/fp61.cuh:17-166; Orion's field_element,
// TruePix-main/Orion/Orion_nonzk/include/linear_gkr/prime_field.h:89-176):
// every public value is canonical in [0, p), so any exact implementation gives
// bit-identical results.
//
// Device multiply: the 122-bit product is never formed. With a = a1*2^32 + a0,
// b = b1*2^32 + b0 (a1, b1 < 2^29), and 2^61 == 1, 2^64 == 8 (mod p):
//   a*b == a0*b0 + (a0*b1 + a1*b0)*2^32 + 8*a1*b1
// and (m*2^32) == (m >> 29) + ((m mod 2^29) << 32). Four 32x32->64 IMAD.WIDE
// products and one final Mersenne fold.
#pragma once
#include <stdint.h>

#if defined(__CUDACC__)
#define TP_HD __host__ __device__ __forceinline__
#else
#define TP_HD inline
#endif

namespace tp {

typedef unsigned long long u64;
typedef unsigned int u32;

static constexpr u64 P61 = 0x1FFFFFFFFFFFFFFFull;

struct __align__(16) fp2 {
    u64 re, im;
};

TP_HD u64 canon(u64 x) { return x >= P61 ? x - P61 : x; }
// any 64-bit value -> canonical
TP_HD u64 reduce64(u64 x) { return canon((x & P61) + (x >> 61)); }
TP_HD u64 fadd(u64 a, u64 b) { return canon(a + b); }
TP_HD u64 fsub(u64 a, u64 b) { return canon(a + (P61 - b)); }
TP_HD u64 fneg(u64 a) { return a ? P61 - a : 0; }

TP_HD u64 fmul(u64 a, u64 b)
{
#if defined(__CUDA_ARCH__)
    const u32 a0 = (u32)a, a1 = (u32)(a >> 32);
    const u32 b0 = (u32)b, b1 = (u32)(b >> 32);
    const u64 lo = (u64)a0 * b0;                      // < 2^64
    const u64 mid = (u64)a0 * b1 + (u64)a1 * b0;      // < 2^62
    const u64 hi = (u64)a1 * b1;                      // < 2^58
    u64 s = (lo & P61) + (lo >> 61) + (hi << 3) + (mid >> 29) + ((mid & 0x1FFFFFFFull) << 32);
    s = (s & P61) + (s >> 61);                        // < 2^61 + 4
    return canon(s);
#else
    const unsigned __int128 t = (unsigned __int128)a * b;
    return canon(((u64)t & P61) + (u64)(t >> 61));
#endif
}

// ---- lazy ("nearly canonical") arithmetic --------------------------------
// Values v < 2^61 + 8 stand for v mod p. Inputs of lmul may be < 2^62 + 64,
// so a sum of two nearly canonical values is a valid operand. Nothing is made
// canonical until a value leaves the kernel (canon61).
TP_HD u64 fold61(u64 x) { return (x & P61) + (x >> 61); }   // any x -> < 2^61 + 8
TP_HD u64 canon61(u64 x)
{
    const u64 f = fold61(x);
    return f >= P61 ? f - P61 : f;
}

#if defined(__CUDA_ARCH__)
// a, b < 2^62 + 64  ->  a*b mod p, < 2^61 + 8.
// T = a*b < 2^125 is formed as four 32-bit words with one carry chain, then
// T mod p = (T mod 2^61) + (T >> 61), folded once more.
__device__ __forceinline__ u64 lmul(u64 a, u64 b)
{
    const u32 a0 = (u32)a, a1 = (u32)(a >> 32), b0 = (u32)b, b1 = (u32)(b >> 32);
    const u64 p00 = (u64)a0 * b0;
    const u64 mid = (u64)a0 * b1 + (u64)a1 * b0;   // < 2^64 for these bounds
    const u64 p11 = (u64)a1 * b1;
    u32 w1, w2, w3, q0, q1, s0, s1;
    asm("add.cc.u32 %0, %3, %4;\n\t"
        "addc.cc.u32 %1, %5, %6;\n\t"
        "addc.u32 %2, %7, 0;"
        : "=r"(w1), "=r"(w2), "=r"(w3)
        : "r"((u32)(p00 >> 32)), "r"((u32)mid), "r"((u32)p11), "r"((u32)(mid >> 32)),
          "r"((u32)(p11 >> 32)));
    asm("shf.r.clamp.b32 %0, %1, %2, 29;" : "=r"(q0) : "r"(w1), "r"(w2));
    asm("shf.r.clamp.b32 %0, %1, %2, 29;" : "=r"(q1) : "r"(w2), "r"(w3));
    asm("add.cc.u32 %0, %2, %3;\n\t"
        "addc.u32 %1, %4, %5;"
        : "=r"(s0), "=r"(s1)
        : "r"((u32)p00), "r"(q0), "r"(w1 & 0x1FFFFFFFu), "r"(q1));
    return fold61(((u64)s1 << 32) | s0);
}
#else
inline u64 lmul(u64 a, u64 b)
{
    const unsigned __int128 t = (unsigned __int128)a * b;
    return fold61(((u64)t & P61) + (u64)(t >> 61));
}
#endif
// nearly canonical a, b -> nearly canonical
TP_HD u64 ladd(u64 a, u64 b) { return fold61(a + b); }
TP_HD u64 lsub(u64 a, u64 b) { return fold61(a + (2 * P61 - b)); }   // b <= 2P

TP_HD fp2 mk(u64 re, u64 im) { fp2 r; r.re = re; r.im = im; return r; }
TP_HD fp2 f2zero() { return mk(0, 0); }
TP_HD bool f2is0(fp2 a) { return (a.re | a.im) == 0; }
TP_HD fp2 f2add(fp2 a, fp2 b) { return mk(fadd(a.re, b.re), fadd(a.im, b.im)); }
TP_HD fp2 f2sub(fp2 a, fp2 b) { return mk(fsub(a.re, b.re), fsub(a.im, b.im)); }
TP_HD fp2 f2dbl(fp2 a) { return f2add(a, a); }
// (a + bi)(c + di) = (ac - bd) + ((a + b)(c + d) - ac - bd) i
TP_HD fp2 f2mul(fp2 a, fp2 b)
{
    const u64 ac = fmul(a.re, b.re);
    const u64 bd = fmul(a.im, b.im);
    const u64 s = fmul(fadd(a.re, a.im), fadd(b.re, b.im));
    return mk(fsub(ac, bd), fsub(s, fadd(ac, bd)));
}
// Fp2 times a base-field scalar
TP_HD fp2 f2scale(fp2 a, u64 k) { return mk(fmul(a.re, k), fmul(a.im, k)); }
// line through (0, a) and (1, b) evaluated at r: a + r(b - a)
TP_HD fp2 f2fold(fp2 a, fp2 b, fp2 r) { return f2add(a, f2mul(r, f2sub(b, a))); }
// the same line at -1 and at 2
TP_HD fp2 f2at_m1(fp2 a, fp2 b) { return f2sub(f2dbl(a), b); }
TP_HD fp2 f2at_2(fp2 a, fp2 b) { return f2sub(f2dbl(b), a); }
// lazy Fp2 (limbs nearly canonical in and out)
TP_HD fp2 l2add(fp2 a, fp2 b) { return mk(ladd(a.re, b.re), ladd(a.im, b.im)); }
TP_HD fp2 l2sub(fp2 a, fp2 b) { return mk(lsub(a.re, b.re), lsub(a.im, b.im)); }
TP_HD fp2 l2mul(fp2 a, fp2 b)
{
    const u64 ac = lmul(a.re, b.re);
    const u64 bd = lmul(a.im, b.im);
    const u64 s = lmul(a.re + a.im, b.re + b.im);
    return mk(fold61(ac + (2 * P61 - bd)), fold61(s + (4 * P61 - ac - bd)));
}
TP_HD fp2 l2canon(fp2 a) { return mk(canon61(a.re), canon61(a.im)); }
// a + r (b - a)
TP_HD fp2 l2fold(fp2 a, fp2 b, fp2 r) { return l2add(a, l2mul(r, l2sub(b, a))); }
TP_HD fp2 l2at_m1(fp2 a, fp2 b) { return l2sub(l2add(a, a), b); }
TP_HD fp2 l2at_2(fp2 a, fp2 b) { return l2sub(l2add(b, b), a); }

// small signed integer -> field
TP_HD u64 from_small(int k) { return k >= 0 ? (u64)k : P61 - (u64)(-k); }

TP_HD u64 fpow(u64 a, u64 e)
{
    u64 r = 1;
    while (e) {
        if (e & 1) r = fmul(r, a);
        a = fmul(a, a);
        e >>= 1;
    }
    return r;
}
TP_HD u64 finv(u64 a) { return fpow(a, P61 - 2); }
// 1/(a + bi) = (a - bi)/(a^2 + b^2); zero maps to zero
TP_HD fp2 f2inv(fp2 a)
{
    const u64 n = fadd(fmul(a.re, a.re), fmul(a.im, a.im));
    if (n == 0) return f2zero();
    const u64 ni = finv(n);
    return mk(fmul(a.re, ni), fneg(fmul(a.im, ni)));
}

}  // namespace tp
