// Device arithmetic in GF(M31), GF(M61) and their quadratic extensions with i^2 = -1
// (montmul/src/field.rs:13-42, 131-222). All results are canonical (in [0, p)), so every value
// equals the reference's bit for bit.
//
// Two facts of the reference's tables make the radix-8 butterflies cheap: in both fields the
// primitive 4th root used by the transforms is omega^(n/4) = i, and the primitive 8th root is
// omega^(n/8) = (1 + i) * 2^s with s = 15 (M31) or 30 (M61), so a product with an 8th root is
// one add, one sub and a bit rotation (2^s * x mod 2^b - 1 rotates x by s bits). The host
// checks both facts against its own tables before any launch.
#pragma once
#include "mm_common.h"

namespace mm {

// ---- GF(M31) ----
__device__ __forceinline__ uint32_t add1(uint32_t a, uint32_t b) {
    uint32_t s = a + b;
    return min(s, s - P1);
}
__device__ __forceinline__ uint32_t sub1(uint32_t a, uint32_t b) {
    uint32_t d = a - b;
    return min(d, d + P1);
}
// t mod M31 for t < 2^63.
__device__ __forceinline__ uint32_t red1(uint64_t t) {
    uint64_t u = (t & P1) + (t >> 31);                  // < 2^33
    uint32_t v = (uint32_t)(u & P1) + (uint32_t)(u >> 31);  // < 2^31 + 4
    return min(v, v - P1);
}
__device__ __forceinline__ uint32_t mul1(uint32_t a, uint32_t b) {
    uint64_t t = (uint64_t)a * b;                       // < 2^62
    uint32_t s = (uint32_t)(t & P1) + (uint32_t)(t >> 31);
    return min(s, s - P1);
}
// x * 2^15 mod M31 (rotation of the 31-bit string).
__device__ __forceinline__ uint32_t rot1(uint32_t x) { return ((x << 15) & P1) | (x >> 16); }
// x * 2 mod M31.
__device__ __forceinline__ uint32_t dbl1(uint32_t x) { return ((x << 1) & P1) | (x >> 30); }

// ---- GF(M61) ----
__device__ __forceinline__ uint64_t add2(uint64_t a, uint64_t b) {
    uint64_t s = a + b;
    return min(s, s - P2);
}
__device__ __forceinline__ uint64_t sub2(uint64_t a, uint64_t b) {
    uint64_t d = a - b;
    return min(d, d + P2);
}
// (hi:lo) mod M61 for hi:lo < 2^124.
__device__ __forceinline__ uint64_t red2(uint64_t lo, uint64_t hi) {
    uint64_t t = (lo & P2) + ((hi << 3) | (lo >> 61));  // < 2^61 + 2^63
    uint64_t s = (t & P2) + (t >> 61);                   // < 2^61 + 4
    return min(s, s - P2);
}
__device__ __forceinline__ uint64_t mul2(uint64_t a, uint64_t b) {
    uint64_t lo = a * b, hi = __umul64hi(a, b);
    uint64_t s = (lo & P2) + ((hi << 3) | (lo >> 61));   // <= 2 P2
    return min(s, s - P2);
}
// a*b + c*d mod M61 for canonical inputs (the sum is below 2^123).
__device__ __forceinline__ uint64_t mul2x2(uint64_t a, uint64_t b, uint64_t c, uint64_t d) {
    uint64_t lo1 = a * b, hi1 = __umul64hi(a, b);
    uint64_t lo2 = c * d, hi2 = __umul64hi(c, d);
    uint64_t lo = lo1 + lo2;
    uint64_t hi = hi1 + hi2 + (lo < lo1);
    return red2(lo, hi);
}
__device__ __forceinline__ uint64_t rot2(uint64_t x) { return ((x << 30) & P2) | (x >> 31); }

// ---- GF(M31^2) ----
__device__ __forceinline__ F1 f1(uint32_t re, uint32_t im) { F1 r; r.re = re; r.im = im; return r; }
__device__ __forceinline__ F1 cadd(F1 a, F1 b) { return f1(add1(a.re, b.re), add1(a.im, b.im)); }
__device__ __forceinline__ F1 csub(F1 a, F1 b) { return f1(sub1(a.re, b.re), sub1(a.im, b.im)); }
// (a - b) * i
__device__ __forceinline__ F1 csub_i(F1 a, F1 b) { return f1(sub1(b.im, a.im), sub1(a.re, b.re)); }
// (a - b) * (-i)
__device__ __forceinline__ F1 csub_mi(F1 a, F1 b) { return f1(sub1(a.im, b.im), sub1(b.re, a.re)); }
__device__ __forceinline__ F1 cmul(F1 a, F1 b) {
    uint64_t re = (uint64_t)a.re * b.re + (uint64_t)a.im * (P1 - b.im);
    uint64_t im = (uint64_t)a.re * b.im + (uint64_t)a.im * b.re;
    return f1(red1(re), red1(im));
}
// real * complex
__device__ __forceinline__ F1 cmul_r(uint32_t a, F1 b) { return f1(mul1(a, b.re), mul1(a, b.im)); }
// re(a * b)
__device__ __forceinline__ uint32_t cmul_re(F1 a, F1 b) {
    return red1((uint64_t)a.re * b.re + (uint64_t)a.im * (P1 - b.im));
}
__device__ __forceinline__ F1 csqr(F1 a) {
    uint32_t m = mul1(a.re, a.im);
    return f1(mul1(add1(a.re, a.im), sub1(a.re, a.im)), add1(m, m));
}
__device__ __forceinline__ F1 cscale(F1 a, uint32_t c) {  // c <= 4
    return f1(red1((uint64_t)a.re * c), red1((uint64_t)a.im * c));
}
__device__ __forceinline__ F1 cconj(F1 a) { return f1(a.re, sub1(0, a.im)); }
// x * omega_8 = x * (1 + i) 2^15
__device__ __forceinline__ F1 mul_w8(F1 x) { return f1(rot1(sub1(x.re, x.im)), rot1(add1(x.re, x.im))); }
// x * omega_8^-1 = x * (1 - i) 2^15
__device__ __forceinline__ F1 mul_v8(F1 x) { return f1(rot1(add1(x.re, x.im)), rot1(sub1(x.im, x.re))); }
__device__ __forceinline__ F1 mul_i(F1 x) { return f1(sub1(0, x.im), x.re); }
__device__ __forceinline__ F1 mul_mi(F1 x) { return f1(x.im, sub1(0, x.re)); }

// ---- GF(M61^2) ----
__device__ __forceinline__ F2 f2(uint64_t re, uint64_t im) { F2 r; r.re = re; r.im = im; return r; }
__device__ __forceinline__ F2 cadd(F2 a, F2 b) { return f2(add2(a.re, b.re), add2(a.im, b.im)); }
__device__ __forceinline__ F2 csub(F2 a, F2 b) { return f2(sub2(a.re, b.re), sub2(a.im, b.im)); }
__device__ __forceinline__ F2 csub_i(F2 a, F2 b) { return f2(sub2(b.im, a.im), sub2(a.re, b.re)); }
__device__ __forceinline__ F2 csub_mi(F2 a, F2 b) { return f2(sub2(a.im, b.im), sub2(b.re, a.re)); }
__device__ __forceinline__ F2 cmul(F2 a, F2 b) {
    return f2(mul2x2(a.re, b.re, a.im, P2 - b.im), mul2x2(a.re, b.im, a.im, b.re));
}
__device__ __forceinline__ F2 cmul_r(uint64_t a, F2 b) { return f2(mul2(a, b.re), mul2(a, b.im)); }
__device__ __forceinline__ uint64_t cmul_re(F2 a, F2 b) { return mul2x2(a.re, b.re, a.im, P2 - b.im); }
__device__ __forceinline__ F2 csqr(F2 a) {
    uint64_t m = mul2(a.re, a.im);
    return f2(mul2(add2(a.re, a.im), sub2(a.re, a.im)), add2(m, m));
}
__device__ __forceinline__ uint64_t scale2(uint64_t a, uint32_t c) {   // c <= 4, a < 2^61
    uint64_t t = a * c;                                   // < 2^63
    uint64_t s = (t & P2) + (t >> 61);
    return min(s, s - P2);
}
__device__ __forceinline__ F2 cscale(F2 a, uint32_t c) { return f2(scale2(a.re, c), scale2(a.im, c)); }
__device__ __forceinline__ F2 cconj(F2 a) { return f2(a.re, sub2(0, a.im)); }
__device__ __forceinline__ F2 mul_w8(F2 x) { return f2(rot2(sub2(x.re, x.im)), rot2(add2(x.re, x.im))); }
__device__ __forceinline__ F2 mul_v8(F2 x) { return f2(rot2(add2(x.re, x.im)), rot2(sub2(x.im, x.re))); }
__device__ __forceinline__ F2 mul_i(F2 x) { return f2(sub2(0, x.im), x.re); }
__device__ __forceinline__ F2 mul_mi(F2 x) { return f2(x.im, sub2(0, x.re)); }

// ---- lazy GF(M61) and GF(M61^2) ----
// Values are kept below 2^64 instead of below p; a value is "reduced" when it is below
// ONE = 2^61 + 2^34, the invariant of everything stored between passes. Sums are not reduced;
// a difference a - b becomes a + (K p - b) with K p at least b's bound; lfold brings any u64
// below 2^61 + 8. The radix-8/4/2 butterflies fold where their bounds would pass 2^64; an
// interval model of every operation checks the bounds. Canonical form (lcanon) is needed only
// where the value leaves the transform domain (CRT) or becomes a multiplier constant.
__device__ __forceinline__ uint64_t lfold(uint64_t x) { return (x & P2) + (x >> 61); }
__device__ __forceinline__ uint64_t lcanon(uint64_t x) {
    uint64_t s = lfold(x);
    return min(s, s - P2);
}
template <int K> __device__ __forceinline__ uint64_t lsub(uint64_t a, uint64_t b) { return a + ((uint64_t)K * P2 - b); }
// x 2^30 mod p for any u64 x, below 2^61 + 2^33.
__device__ __forceinline__ uint64_t lrot(uint64_t x) { return ((x << 30) & P2) + (x >> 31); }
// a b mod p below p + (a b >> 61) for a b < 2^125 (one fold of the 128-bit product).
__device__ __forceinline__ uint64_t lmul1(uint64_t a, uint64_t b) {
    uint64_t lo = a * b, hi = __umul64hi(a, b);
    return (lo & P2) + ((hi << 3) | (lo >> 61));
}
__device__ __forceinline__ F2 lcfold(F2 x) { return f2(lfold(x.re), lfold(x.im)); }
__device__ __forceinline__ F2 lccanon(F2 x) { return f2(lcanon(x.re), lcanon(x.im)); }
__device__ __forceinline__ F2 lcadd(F2 a, F2 b) { return f2(a.re + b.re, a.im + b.im); }
template <int K> __device__ __forceinline__ F2 lcsub(F2 a, F2 b) { return f2(lsub<K>(a.re, b.re), lsub<K>(a.im, b.im)); }
// (a - b) i
template <int K> __device__ __forceinline__ F2 lcsub_i(F2 a, F2 b) { return f2(lsub<K>(b.im, a.im), lsub<K>(a.re, b.re)); }
// u + (-i) v and u - (-i) v
template <int K> __device__ __forceinline__ F2 lcadd_mi(F2 u, F2 v) { return f2(u.re + v.im, lsub<K>(u.im, v.re)); }
template <int K> __device__ __forceinline__ F2 lcsub_mi(F2 u, F2 v) { return f2(lsub<K>(u.re, v.im), u.im + v.re); }
// x omega_8 = x (1 + i) 2^30 and x omega_8^-1 = x (1 - i) 2^30, reduced outputs
template <int K> __device__ __forceinline__ F2 lw8(F2 x) { return f2(lrot(lsub<K>(x.re, x.im)), lrot(x.re + x.im)); }
template <int K> __device__ __forceinline__ F2 lv8(F2 x) { return f2(lrot(x.re + x.im), lrot(lsub<K>(x.im, x.re))); }
// x (-i)
template <int K> __device__ __forceinline__ F2 lmi(F2 x) { return f2(x.im, lsub<K>(0, x.re)); }
// x w for reduced x and a twiddle in Karatsuba form: k1 = wr (xr + xi), k2 = xr (wi - wr),
// k3 = xi (wr + wi); re = k1 - k3, im = k1 + k2. Three products instead of four.
__device__ __forceinline__ F2 lkmul(F2 x, const F2K& w) {
    const uint64_t k1 = lmul1(x.re + x.im, w.re), k2 = lmul1(x.re, w.d), k3 = lmul1(x.im, w.s);
    return f2(lfold(lsub<3>(k1, k3)), lfold(k1 + k2));
}
// x w for reduced x and a canonical constant w (its Karatsuba sums formed here).
__device__ __forceinline__ F2 lkmulc(F2 x, F2 w) {
    const uint64_t s = w.re + w.im, d = lsub<1>(w.im, w.re);
    const uint64_t k1 = lmul1(x.re + x.im, w.re), k2 = lmul1(x.re, d), k3 = lmul1(x.im, s);
    return f2(lfold(lsub<4>(k1, k3)), lfold(k1 + k2));
}
// re(x w) for reduced x and a Karatsuba-form twiddle.
__device__ __forceinline__ uint64_t lkmul_re(F2 x, const F2K& w) {
    return lfold(lmul1(x.re, w.re) + lmul1(x.im, P2 - w.im));
}
// v c mod p for a 32-bit v and canonical c, reduced (below 2^61 + 2^32): two 32x32 products.
// v c = p0 + p1 2^32 with p0 = v c_lo, p1 = v c_hi (c_hi < 2^29, so p1 + p0_hi < 2^62).
__device__ __forceinline__ uint64_t lmul32(uint32_t v, uint64_t c) {
    const uint64_t p0 = (uint64_t)v * (uint32_t)c;
    const uint64_t m = (uint64_t)v * (uint32_t)(c >> 32) + (p0 >> 32);   // bits 32.. of v c
    // v c = m 2^32 + p0_lo; mod p: (low 61 bits) + (v c >> 61) = ((m << 32 | p0_lo) & p) + (m >> 29)
    return ((m << 32 | (uint32_t)p0) & P2) + (m >> 29);
}
// real 32-bit limb times a canonical constant, reduced.
__device__ __forceinline__ F2 lreal_times(uint32_t v, const F2K& c) { return f2(lmul32(v, c.re), lmul32(v, c.im)); }
// x^2 c for reduced x and c <= 4, reduced.
__device__ __forceinline__ F2 lsqr_scale(F2 x, uint32_t c) {
    const uint64_t re = lfold(lmul1(x.re + x.im, lsub<2>(x.re, x.im)));
    const uint64_t t = lmul1(x.re, x.im);
    const uint64_t im = lfold(t + t);
    if (c == 1) return f2(re, im);
    return f2(lfold(re * c), lfold(im * c));
}

// ---- CRT (field.rs:288-294) ----
// The unique C < M31 * M61 with C = c1 mod M31 and C = c2 mod M61, as three 32-bit words.
// (M61 mod M31)^-1 = -2 mod M31, so h = 2 (c2 mod M31 - c1) mod M31 and C = c2 + M61 h.
// c2 may be any reduced (lazy) M61 value; it is made canonical first.
__device__ __forceinline__ void crt3(uint32_t c1, uint64_t c2, uint32_t& w0, uint32_t& w1, uint32_t& w2) {
    c2 = lcanon(c2);
    uint32_t c2m = (uint32_t)(c2 & P1) + (uint32_t)(c2 >> 31);   // < 2^31 + 2^30
    c2m = min(c2m, c2m - P1);
    const uint32_t h = dbl1(sub1(c2m, c1));
    // C = c2 - h + h 2^61 = (c2 - h) + (h & 7) 2^61 + (h >> 3) 2^64, with the borrow of c2 - h
    // and the carry of the low 64-bit sum folded into the top word.
    const uint64_t t = c2 - h;
    const uint32_t borrow = c2 < (uint64_t)h;
    const uint64_t lo = t + ((uint64_t)(h & 7) << 61);
    const uint32_t carry = lo < t;
    w0 = (uint32_t)lo;
    w1 = (uint32_t)(lo >> 32);
    w2 = (h >> 3) + carry - borrow;
}

}  // namespace mm
