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
