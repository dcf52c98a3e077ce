// Shared-memory transforms of one vector per thread block: the reference's DIF and DIT
// (montmul/src/cpu.rs:49-115) run as radix-8/4/2 passes, each pass = log2 R radix-2 stages done
// in registers, one barrier per pass.
//
// Radix-R DIF pass with span q on the group b + j + k q (k < R): the R-point butterfly uses only
// the fixed roots i and omega_8 (mm_field.cuh); the remaining factors of the R stages,
// W^(j rev_R(k)) with W a primitive (R q)-th root, are applied to the outputs afterwards (they
// commute with the later butterflies of the same pass). The DIT pass mirrors it: inputs first
// multiplied by V^(j rev_R(k)), V = W^-1, then the inverse butterflies. Either way every
// position ends with exactly the value the reference's radix-2 loops produce.
//
// Shared-memory layout: F2 array (16 B per element) then F1 array (8 B), element e stored at
// swz(e) (swz_c, mm_common.h): conflict-free for every pass and carry of the kernels.
#pragma once
#include "mm_field.cuh"

namespace mm {

// ---- thread groups ----
// One slot is worked on by a group of NT threads (NT a power of two, a multiple of 32). A block
// is one group (the uniform launches, and the mixed launch's wide items) or two (the mixed
// launch's two 256-thread workers). Group 0 synchronizes on hardware barrier 1 and group 1 on
// barrier 2, each with its NT threads only, so the two groups of a block run independently. The
// barrier IDs are immediates: an ID held in a register made the barriers of short steps about
// twice as slow (L = 256: 62 vs 33 ns per slot-step in the uniform launch).
template <int NT> __device__ __forceinline__ int gtid() { return (int)(threadIdx.x & (NT - 1)); }
template <int NT> __device__ __forceinline__ bool group0() { return NT >= 512 || threadIdx.x < NT; }
template <int NT> __device__ __forceinline__ void gsync() {
    if (group0<NT>()) asm volatile("bar.sync 1, %0;" ::"n"(NT) : "memory");
    else asm volatile("bar.sync 2, %0;" ::"n"(NT) : "memory");
}
// Barrier of the group that returns whether `pred` is non-zero on any of its threads.
template <int NT> __device__ __forceinline__ int gsync_or(int pred) {
    int r;
    if (group0<NT>())
        asm volatile("{ .reg .pred p, q; setp.ne.s32 p, %1, 0; bar.red.or.pred q, 1, %2, p; selp.s32 %0, 1, 0, q; }"
                     : "=r"(r) : "r"(pred), "n"(NT) : "memory");
    else
        asm volatile("{ .reg .pred p, q; setp.ne.s32 p, %1, 0; bar.red.or.pred q, 2, %2, p; selp.s32 %0, 1, 0, q; }"
                     : "=r"(r) : "r"(pred), "n"(NT) : "memory");
    return r;
}

__device__ __forceinline__ int swz(int e) { return swz_c(e); }

// ---- in-register butterflies (positions k of one group) ----
// u + (-i) v and u - (-i) v
__device__ __forceinline__ F1 cadd_mi(F1 u, F1 v) { return f1(add1(u.re, v.im), sub1(u.im, v.re)); }
__device__ __forceinline__ F1 csub_mi2(F1 u, F1 v) { return f1(sub1(u.re, v.im), add1(u.im, v.re)); }
__device__ __forceinline__ F2 cadd_mi(F2 u, F2 v) { return f2(add2(u.re, v.im), sub2(u.im, v.re)); }
__device__ __forceinline__ F2 csub_mi2(F2 u, F2 v) { return f2(sub2(u.re, v.im), add2(u.im, v.re)); }

template <int R, typename T> __device__ __forceinline__ void bf_dif(T* x);
template <int R, typename T> __device__ __forceinline__ void bf_dit(T* x);

template <> __device__ __forceinline__ void bf_dif<2, F1>(F1* x) { F1 u = x[0]; x[0] = cadd(u, x[1]); x[1] = csub(u, x[1]); }
template <> __device__ __forceinline__ void bf_dif<2, F2>(F2* x) { F2 u = x[0]; x[0] = cadd(u, x[1]); x[1] = csub(u, x[1]); }
template <> __device__ __forceinline__ void bf_dit<2, F1>(F1* x) { bf_dif<2, F1>(x); }
template <> __device__ __forceinline__ void bf_dit<2, F2>(F2* x) { bf_dif<2, F2>(x); }

template <typename T> __device__ __forceinline__ void bf_dif4(T* x) {
    T a0 = cadd(x[0], x[2]), b0 = csub(x[0], x[2]);
    T a1 = cadd(x[1], x[3]), b1 = csub_i(x[1], x[3]);
    x[0] = cadd(a0, a1); x[1] = csub(a0, a1);
    x[2] = cadd(b0, b1); x[3] = csub(b0, b1);
}
template <typename T> __device__ __forceinline__ void bf_dit4(T* x) {
    T c0 = cadd(x[0], x[1]), c1 = csub(x[0], x[1]);
    T c2 = cadd(x[2], x[3]), c3 = csub(x[2], x[3]);
    x[0] = cadd(c0, c2); x[2] = csub(c0, c2);
    x[1] = cadd_mi(c1, c3); x[3] = csub_mi2(c1, c3);
}
template <typename T> __device__ __forceinline__ void bf_dif8(T* x) {
    T a0 = cadd(x[0], x[4]), b0 = csub(x[0], x[4]);
    T a1 = cadd(x[1], x[5]), b1 = mul_w8(csub(x[1], x[5]));
    T a2 = cadd(x[2], x[6]), b2 = csub_i(x[2], x[6]);
    T a3 = cadd(x[3], x[7]), b3 = mul_w8(csub_i(x[3], x[7]));
    T c0 = cadd(a0, a2), c2 = csub(a0, a2);
    T c1 = cadd(a1, a3), c3 = csub_i(a1, a3);
    T d0 = cadd(b0, b2), d2 = csub(b0, b2);
    T d1 = cadd(b1, b3), d3 = csub_i(b1, b3);
    x[0] = cadd(c0, c1); x[1] = csub(c0, c1);
    x[2] = cadd(c2, c3); x[3] = csub(c2, c3);
    x[4] = cadd(d0, d1); x[5] = csub(d0, d1);
    x[6] = cadd(d2, d3); x[7] = csub(d2, d3);
}
template <typename T> __device__ __forceinline__ void bf_dit8(T* x) {
    T c0 = cadd(x[0], x[1]), c1 = csub(x[0], x[1]);
    T c2 = cadd(x[2], x[3]), c3 = csub(x[2], x[3]);
    T c4 = cadd(x[4], x[5]), c5 = csub(x[4], x[5]);
    T c6 = cadd(x[6], x[7]), c7 = csub(x[6], x[7]);
    T a0 = cadd(c0, c2), a2 = csub(c0, c2);
    T a1 = cadd_mi(c1, c3), a3 = csub_mi2(c1, c3);
    T b0 = cadd(c4, c6), b2 = csub(c4, c6);
    T b1 = cadd_mi(c5, c7), b3 = csub_mi2(c5, c7);
    // stage with span 4: factors nu8^k on b_k, nu8 = omega_8^-1, nu8^2 = -i, nu8^3 = nu8 (-i)
    T v1 = mul_v8(b1), v2 = mul_mi(b2), v3 = mul_mi(mul_v8(b3));
    x[0] = cadd(a0, b0); x[4] = csub(a0, b0);
    x[1] = cadd(a1, v1); x[5] = csub(a1, v1);
    x[2] = cadd(a2, v2); x[6] = csub(a2, v2);
    x[3] = cadd(a3, v3); x[7] = csub(a3, v3);
}
// ---- lazy GF(M61^2) butterflies (inputs reduced, below 2^61 + 2^34) ----
// DIF: outputs below 8 * 2^61, not reduced (the pass folds them or feeds them to a twiddle
// product after a fold). DIT: outputs reduced. Offsets K p and fold points follow the interval
// model of these exact operation sequences.
__device__ __forceinline__ void ldif2(F2* x) { F2 u = x[0]; x[0] = lcadd(u, x[1]); x[1] = lcsub<2>(u, x[1]); }
__device__ __forceinline__ void ldit2(F2* x) { F2 u = x[0]; x[0] = lcfold(lcadd(u, x[1])); x[1] = lcfold(lcsub<2>(u, x[1])); }
__device__ __forceinline__ void ldif4(F2* x) {
    const F2 a0 = lcadd(x[0], x[2]), b0 = lcsub<2>(x[0], x[2]);
    const F2 a1 = lcadd(x[1], x[3]), b1 = lcsub_i<2>(x[1], x[3]);
    x[0] = lcadd(a0, a1); x[1] = lcsub<3>(a0, a1);
    x[2] = lcadd(b0, b1); x[3] = lcsub<4>(b0, b1);
}
__device__ __forceinline__ void ldit4(F2* x) {
    const F2 c0 = lcadd(x[0], x[1]), c1 = lcsub<2>(x[0], x[1]);
    const F2 c2 = lcadd(x[2], x[3]), c3 = lcsub<2>(x[2], x[3]);
    x[0] = lcfold(lcadd(c0, c2)); x[2] = lcfold(lcsub<3>(c0, c2));
    x[1] = lcfold(lcadd_mi<4>(c1, c3)); x[3] = lcfold(lcsub_mi<4>(c1, c3));
}
__device__ __forceinline__ void ldif8(F2* x) {
    const F2 a0 = lcfold(lcadd(x[0], x[4])), b0 = lcfold(lcsub<2>(x[0], x[4]));
    const F2 a1 = lcfold(lcadd(x[1], x[5])), b1 = lw8<4>(lcsub<2>(x[1], x[5]));
    const F2 a2 = lcfold(lcadd(x[2], x[6])), b2 = lcfold(lcsub_i<2>(x[2], x[6]));
    const F2 a3 = lcfold(lcadd(x[3], x[7])), b3 = lw8<4>(lcsub_i<2>(x[3], x[7]));
    const F2 c0 = lcadd(a0, a2), c2 = lcsub<2>(a0, a2);
    const F2 c1 = lcadd(a1, a3), c3 = lcsub_i<2>(a1, a3);
    const F2 d0 = lcadd(b0, b2), d2 = lcsub<2>(b0, b2);
    const F2 d1 = lcadd(b1, b3), d3 = lcsub_i<2>(b1, b3);
    x[0] = lcadd(c0, c1); x[1] = lcsub<3>(c0, c1);
    x[2] = lcadd(c2, c3); x[3] = lcsub<4>(c2, c3);
    x[4] = lcadd(d0, d1); x[5] = lcsub<3>(d0, d1);
    x[6] = lcadd(d2, d3); x[7] = lcsub<4>(d2, d3);
}
__device__ __forceinline__ void ldit8(F2* x) {
    const F2 c0 = lcfold(lcadd(x[0], x[1])), c1 = lcfold(lcsub<2>(x[0], x[1]));
    const F2 c2 = lcfold(lcadd(x[2], x[3])), c3 = lcfold(lcsub<2>(x[2], x[3]));
    const F2 c4 = lcfold(lcadd(x[4], x[5])), c5 = lcfold(lcsub<2>(x[4], x[5]));
    const F2 c6 = lcfold(lcadd(x[6], x[7])), c7 = lcfold(lcsub<2>(x[6], x[7]));
    const F2 a0 = lcadd(c0, c2), a2 = lcsub<2>(c0, c2);
    const F2 a1 = lcadd_mi<2>(c1, c3), a3 = lcsub_mi<2>(c1, c3);
    const F2 b0 = lcadd(c4, c6), b2 = lcsub<2>(c4, c6);
    const F2 b1 = lcadd_mi<2>(c5, c7), b3 = lcsub_mi<2>(c5, c7);
    const F2 v1 = lv8<4>(b1), v3 = lv8<4>(lmi<4>(b3));
    x[0] = lcfold(lcadd(a0, b0)); x[4] = lcfold(lcsub<3>(a0, b0));
    x[1] = lcfold(lcadd(a1, v1)); x[5] = lcfold(lcsub<2>(a1, v1));
    x[2] = lcfold(f2(a2.re + b2.im, lsub<4>(a2.im, b2.re)));
    x[6] = lcfold(f2(lsub<4>(a2.re, b2.im), a2.im + b2.re));
    x[3] = lcfold(lcadd(a3, v3)); x[7] = lcfold(lcsub<2>(a3, v3));
}
template <int R> __device__ __forceinline__ void ldif(F2* x) { if (R == 2) ldif2(x); else if (R == 4) ldif4(x); else ldif8(x); }
template <int R> __device__ __forceinline__ void ldit(F2* x) { if (R == 2) ldit2(x); else if (R == 4) ldit4(x); else ldit8(x); }

template <> __device__ __forceinline__ void bf_dif<4, F1>(F1* x) { bf_dif4(x); }
template <> __device__ __forceinline__ void bf_dif<4, F2>(F2* x) { bf_dif4(x); }
template <> __device__ __forceinline__ void bf_dit<4, F1>(F1* x) { bf_dit4(x); }
template <> __device__ __forceinline__ void bf_dit<4, F2>(F2* x) { bf_dit4(x); }
template <> __device__ __forceinline__ void bf_dif<8, F1>(F1* x) { bf_dif8(x); }
template <> __device__ __forceinline__ void bf_dif<8, F2>(F2* x) { bf_dif8(x); }
template <> __device__ __forceinline__ void bf_dit<8, F1>(F1* x) { bf_dit8(x); }
template <> __device__ __forceinline__ void bf_dit<8, F2>(F2* x) { bf_dit8(x); }

// ---- one pass over the shared vector ----
// A radix-R pass with span q = 2^LQ over G = n/R groups, twiddles `t2`/`t1` laid out
// [k-1][j] (TW) or none (span 1). One non-inlined function per (R, direction, TW) with a
// runtime span serves every pass of every transform: the smaller code measured faster than one
// instance per span, because the step loop's code then stays within the instruction cache.
template <int R, bool FWD, int NT, bool TW>
__device__ __noinline__ void pass_rt(F2* s2, F1* s1, const F2K* __restrict__ t2, const F1* __restrict__ t1, int LQ, int G) {
    const int q = 1 << LQ;
    // swz(k q) for k < R: swz is linear over XOR, so the offsets are XORs of those of the
    // span's powers of two q, 2q, 4q (three registers instead of R).
    const int kb0 = swz(q), kb1 = R > 2 ? swz(2 * q) : 0, kb2 = R > 4 ? swz(4 * q) : 0;
#define MM_KO(k) ((((k) & 1) ? kb0 : 0) ^ (((k) & 2) ? kb1 : 0) ^ (((k) & 4) ? kb2 : 0))
#pragma unroll 1
    for (int g = gtid<NT>(); g < G; g += NT) {
        const int j = g & (q - 1);
        // b + k q has disjoint bits: swz(b + k q) = swz(b) ^ swz(k q).
        const int sb = swz(((g >> LQ) << (LQ + ilog2c(R))) + j);
        {
            F2 x[R];
#pragma unroll
            for (int k = 0; k < R; ++k) x[k] = s2[sb ^ MM_KO(k)];
            if (FWD) {
                ldif<R>(x);
                x[0] = lcfold(x[0]);
#pragma unroll
                for (int k = 1; k < R; ++k) x[k] = TW ? lkmul(lcfold(x[k]), t2[(k - 1) * q + j]) : lcfold(x[k]);
            } else {
                if (TW) {
#pragma unroll
                    for (int k = 1; k < R; ++k) x[k] = lkmul(x[k], t2[(k - 1) * q + j]);
                }
                ldit<R>(x);
            }
#pragma unroll
            for (int k = 0; k < R; ++k) s2[sb ^ MM_KO(k)] = x[k];
        }
        {
            F1 x[R];
#pragma unroll
            for (int k = 0; k < R; ++k) x[k] = s1[sb ^ MM_KO(k)];
            if (FWD) {
                bf_dif<R, F1>(x);
                if (TW) {
#pragma unroll
                    for (int k = 1; k < R; ++k) x[k] = cmul(x[k], t1[(k - 1) * q + j]);
                }
            } else {
                if (TW) {
#pragma unroll
                    for (int k = 1; k < R; ++k) x[k] = cmul(x[k], t1[(k - 1) * q + j]);
                }
                bf_dit<R, F1>(x);
            }
#pragma unroll
            for (int k = 0; k < R; ++k) s1[sb ^ MM_KO(k)] = x[k];
        }
    }
#undef MM_KO
    gsync<NT>();
}

// Pass I (DIF order) of the length-2^M transform; its table follows mm_common.h's layout.
template <int M, int I, bool FWD, int NT, bool WEIGHTED>
__device__ __forceinline__ void smem_pass(F2* s2, F1* s1, const F2K* tab2, const F1* tab1) {
    constexpr int R = sched_radix(M, I), Q = sched_q(M, I);
    constexpr int toff = FWD ? tab_fwd_off(M, I, WEIGHTED) : tab_inv_off(M, I, WEIGHTED);
    pass_rt<R, FWD, NT, (Q > 1)>(s2, s1, tab2 + toff, tab1 + toff, ilog2c(Q), (1 << M) / R);
}

// ---- the weighted first DIF pass, straight from real limbs in global memory ----
// Element j + k q of the input is (v, 0) with v the 32-bit limb (0 beyond `cnt`); its weight
// zeta^(j + k q) = zeta^j zeta^(q k) splits into the pass constant zeta^(q k) on the input and
// zeta^j folded into the output factors of the table.
template <typename T> __device__ __forceinline__ T real_times(uint32_t v, T c);
template <> __device__ __forceinline__ F1 real_times<F1>(uint32_t v, F1 c) {
    uint32_t s = (v & P1) + (v >> 31);
    s = min(s, s - P1);
    return cmul_r(s, c);
}

template <int M, int NT>
__device__ __noinline__ void dif_first_from_limbs(const uint32_t* __restrict__ lim, int cnt, F2* s2, F1* s1,
                                                     const F2K* tab2, const F1* tab1) {
    constexpr int R = sched_radix(M, 0), Q = sched_q(M, 0);
    static_assert(Q > 1, "single-pass transforms use the fused pass");
    constexpr int toff = tab_fwd_off(M, 0, true), coff = tab_in_const_off(M, true);
#pragma unroll 1
    for (int j = gtid<NT>(); j < Q; j += NT) {
        const int sj = swz(j);   // j < Q: swz(j + k Q) = swz(j) ^ swz(k Q)
        uint32_t v[R];
#pragma unroll
        for (int k = 0; k < R; ++k) v[k] = (j + k * Q < cnt) ? lim[j + k * Q] : 0u;
        {
            F2 x[R];
#pragma unroll
            for (int k = 0; k < R; ++k) x[k] = lreal_times(v[k], tab2[coff + k]);
            ldif<R>(x);
#pragma unroll
            for (int k = 0; k < R; ++k) s2[(sj ^ swz_c(k * Q))] = lkmul(lcfold(x[k]), tab2[toff + k * Q + j]);
        }
        {
            F1 x[R];
#pragma unroll
            for (int k = 0; k < R; ++k) x[k] = real_times<F1>(v[k], tab1[coff + k]);
            bf_dif<R, F1>(x);
#pragma unroll
            for (int k = 0; k < R; ++k) s1[(sj ^ swz_c(k * Q))] = cmul(x[k], tab1[toff + k * Q + j]);
        }
    }
    gsync<NT>();
}

// ---- the weighted last DIT pass: unweights by zeta^-(j + k q) / n into natural order ----
// REAL_ONLY: only the real parts are needed (the low half of the product, coefficients < n).
template <int M, int NT, bool REAL_ONLY>
__device__ __noinline__ void dit_last_weighted(F2* s2, F1* s1, const F2K* tab2, const F1* tab1) {
    constexpr int R = sched_radix(M, 0), Q = sched_q(M, 0);
    static_assert(Q > 1, "single-pass transforms use the fused pass");
    constexpr int toff = tab_inv_off(M, 0, true), coff = tab_out_const_off(M, true);
#pragma unroll 1
    for (int j = gtid<NT>(); j < Q; j += NT) {
        const int sj = swz(j);   // j < Q: swz(j + k Q) = swz(j) ^ swz(k Q)
        {
            F2 x[R];
#pragma unroll
            for (int k = 0; k < R; ++k) x[k] = lkmul(s2[(sj ^ swz_c(k * Q))], tab2[toff + k * Q + j]);
            ldit<R>(x);
#pragma unroll
            for (int k = 0; k < R; ++k) {
                if (REAL_ONLY) s2[(sj ^ swz_c(k * Q))].re = lkmul_re(x[k], tab2[coff + k]);
                else s2[(sj ^ swz_c(k * Q))] = lkmul(x[k], tab2[coff + k]);
            }
        }
        {
            F1 x[R];
#pragma unroll
            for (int k = 0; k < R; ++k) x[k] = cmul(s1[(sj ^ swz_c(k * Q))], tab1[toff + k * Q + j]);
            bf_dit<R, F1>(x);
#pragma unroll
            for (int k = 0; k < R; ++k) {
                if (REAL_ONLY) s1[(sj ^ swz_c(k * Q))].re = cmul_re(x[k], tab1[coff + k]);
                else s1[(sj ^ swz_c(k * Q))] = cmul(x[k], tab1[coff + k]);
            }
        }
    }
    gsync<NT>();
}

// ---- the Transform trait's weighted passes on complex elements (cpu.rs:86-103) ----
// Forward: element j + k q times zeta^(q k) before the butterfly; zeta^j and the pass twiddles
// after it, from the table (none when the transform is this single pass, q = 1). The vector is
// in shared memory at swz positions, canonical or reduced.
template <int M, int NT>
__device__ __noinline__ void dif_first_complex(F2* s2, F1* s1, const F2K* tab2, const F1* tab1) {
    constexpr int R = sched_radix(M, 0), Q = sched_q(M, 0);
    constexpr int toff = tab_fwd_off(M, 0, true), coff = tab_in_const_off(M, true);
#pragma unroll 1
    for (int j = gtid<NT>(); j < Q; j += NT) {
        const int sj = swz(j);   // j < Q: swz(j + k Q) = swz(j) ^ swz(k Q)
        {
            F2 x[R];
#pragma unroll
            for (int k = 0; k < R; ++k) x[k] = lkmul(s2[(sj ^ swz_c(k * Q))], tab2[coff + k]);
            ldif<R>(x);
#pragma unroll
            for (int k = 0; k < R; ++k)
                s2[(sj ^ swz_c(k * Q))] = Q > 1 ? lkmul(lcfold(x[k]), tab2[toff + k * Q + j]) : lcfold(x[k]);
        }
        {
            F1 x[R];
#pragma unroll
            for (int k = 0; k < R; ++k) x[k] = cmul(s1[(sj ^ swz_c(k * Q))], tab1[coff + k]);
            bf_dif<R, F1>(x);
#pragma unroll
            for (int k = 0; k < R; ++k) s1[(sj ^ swz_c(k * Q))] = Q > 1 ? cmul(x[k], tab1[toff + k * Q + j]) : x[k];
        }
    }
    gsync<NT>();
}

// Inverse: the pass twiddles (with zeta^-j) before the butterfly, zeta^-(q k) / n after it.
template <int M, int NT>
__device__ __noinline__ void dit_last_complex(F2* s2, F1* s1, const F2K* tab2, const F1* tab1) {
    constexpr int R = sched_radix(M, 0), Q = sched_q(M, 0);
    constexpr int toff = tab_inv_off(M, 0, true), coff = tab_out_const_off(M, true);
#pragma unroll 1
    for (int j = gtid<NT>(); j < Q; j += NT) {
        const int sj = swz(j);   // j < Q: swz(j + k Q) = swz(j) ^ swz(k Q)
        {
            F2 x[R];
#pragma unroll
            for (int k = 0; k < R; ++k)
                x[k] = Q > 1 ? lkmul(s2[(sj ^ swz_c(k * Q))], tab2[toff + k * Q + j]) : s2[(sj ^ swz_c(k * Q))];
            ldit<R>(x);
#pragma unroll
            for (int k = 0; k < R; ++k) s2[(sj ^ swz_c(k * Q))] = lkmul(x[k], tab2[coff + k]);
        }
        {
            F1 x[R];
#pragma unroll
            for (int k = 0; k < R; ++k) x[k] = Q > 1 ? cmul(s1[(sj ^ swz_c(k * Q))], tab1[toff + k * Q + j]) : s1[(sj ^ swz_c(k * Q))];
            bf_dit<R, F1>(x);
#pragma unroll
            for (int k = 0; k < R; ++k) s1[(sj ^ swz_c(k * Q))] = cmul(x[k], tab1[coff + k]);
        }
    }
    gsync<NT>();
}

// ---- the fused middle: last DIF pass (span 1), a pointwise operation, first DIT pass ----
// OP::apply2/apply1(x, g) transforms the R spectrum values of group g (positions R g + k).
// With a single pass (M <= 3) the same pass is also the weighted first/last pass.
template <int M, int NT, bool REAL_ONLY, class OP>
__device__ __noinline__ void fused_mid(const uint32_t* __restrict__ lim, int cnt, F2* s2, F1* s1,
                                          const F2K* tab2, const F1* tab1, const OP& op) {
    constexpr int P = sched_passes(M);
    constexpr int R = sched_radix(M, P - 1);
    constexpr int G = (1 << M) / R;
    constexpr bool single = (P == 1);
    constexpr int cin = tab_in_const_off(M, true), cout = tab_out_const_off(M, true);
#pragma unroll 1
    for (int g = gtid<NT>(); g < G; g += NT) {
        const int sg = swz(R * g);   // swz(R g + k) = swz(R g) ^ k for k < R <= 8
        {
            F2 x[R];
            if (single) {
#pragma unroll
                for (int k = 0; k < R; ++k) x[k] = lreal_times(k < cnt ? lim[k] : 0u, tab2[cin + k]);
            } else {
#pragma unroll
                for (int k = 0; k < R; ++k) x[k] = s2[(sg ^ k)];
            }
            ldif<R>(x);
#pragma unroll
            for (int k = 0; k < R; ++k) x[k] = lcfold(x[k]);
            if (!op.template apply2<R>(x, g)) {
                ldit<R>(x);
#pragma unroll
                for (int k = 0; k < R; ++k) {
                    if (single) {
                        if (REAL_ONLY) s2[k].re = lkmul_re(x[k], tab2[cout + k]);
                        else s2[k] = lkmul(x[k], tab2[cout + k]);
                    } else {
                        s2[(sg ^ k)] = x[k];
                    }
                }
            }
        }
        {
            F1 x[R];
            if (single) {
#pragma unroll
                for (int k = 0; k < R; ++k) x[k] = real_times<F1>(k < cnt ? lim[k] : 0u, tab1[cin + k]);
            } else {
#pragma unroll
                for (int k = 0; k < R; ++k) x[k] = s1[(sg ^ k)];
            }
            bf_dif<R, F1>(x);
            if (!op.template apply1<R>(x, g)) {
                bf_dit<R, F1>(x);
#pragma unroll
                for (int k = 0; k < R; ++k) {
                    if (single) {
                        if (REAL_ONLY) s1[k].re = cmul_re(x[k], tab1[cout + k]);
                        else s1[k] = cmul(x[k], tab1[cout + k]);
                    } else {
                        s1[(sg ^ k)] = x[k];
                    }
                }
            }
        }
    }
    gsync<NT>();
}

// ---- whole transforms ----
// Forward weighted transform of real limbs up to (not including) the last pass.
template <int M, int NT>
__device__ __forceinline__ void fwd_limbs(const uint32_t* __restrict__ lim, int cnt, F2* s2, F1* s1,
                                          const F2K* t2, const F1* t1) {
    constexpr int P = sched_passes(M);
    if constexpr (P >= 2) {
        dif_first_from_limbs<M, NT>(lim, cnt, s2, s1, t2, t1);
        if constexpr (P >= 3) smem_pass<M, 1, true, NT, true>(s2, s1, t2, t1);
        if constexpr (P >= 4) smem_pass<M, 2, true, NT, true>(s2, s1, t2, t1);
        if constexpr (P >= 5) smem_pass<M, 3, true, NT, true>(s2, s1, t2, t1);
        static_assert(P <= 5, "schedule longer than the shared-memory lengths need");
    }
}

// Inverse weighted transform from after the fused pass down to natural order.
template <int M, int NT, bool REAL_ONLY>
__device__ __forceinline__ void inv_to_natural(F2* s2, F1* s1, const F2K* t2, const F1* t1) {
    constexpr int P = sched_passes(M);
    if constexpr (P >= 2) {
        if constexpr (P >= 5) smem_pass<M, 3, false, NT, true>(s2, s1, t2, t1);
        if constexpr (P >= 4) smem_pass<M, 2, false, NT, true>(s2, s1, t2, t1);
        if constexpr (P >= 3) smem_pass<M, 1, false, NT, true>(s2, s1, t2, t1);
        dit_last_weighted<M, NT, REAL_ONLY>(s2, s1, t2, t1);
    }
}

// Unweighted transforms of the first 2^M elements (the wraparound path's length h), all in smem.
template <int M, int NT>
__device__ __forceinline__ void dif_unweighted(F2* s2, F1* s1, const F2K* t2, const F1* t1) {
    constexpr int P = sched_passes(M);
    smem_pass<M, 0, true, NT, false>(s2, s1, t2, t1);
    if constexpr (P >= 2) smem_pass<M, 1, true, NT, false>(s2, s1, t2, t1);
    if constexpr (P >= 3) smem_pass<M, 2, true, NT, false>(s2, s1, t2, t1);
    if constexpr (P >= 4) smem_pass<M, 3, true, NT, false>(s2, s1, t2, t1);
    if constexpr (P >= 5) smem_pass<M, 4, true, NT, false>(s2, s1, t2, t1);
    static_assert(P <= 5, "schedule longer than the shared-memory lengths need");
}
template <int M, int NT>
__device__ __forceinline__ void dit_unweighted(F2* s2, F1* s1, const F2K* t2, const F1* t1) {
    constexpr int P = sched_passes(M);
    if constexpr (P >= 5) smem_pass<M, 4, false, NT, false>(s2, s1, t2, t1);
    if constexpr (P >= 4) smem_pass<M, 3, false, NT, false>(s2, s1, t2, t1);
    if constexpr (P >= 3) smem_pass<M, 2, false, NT, false>(s2, s1, t2, t1);
    if constexpr (P >= 2) smem_pass<M, 1, false, NT, false>(s2, s1, t2, t1);
    smem_pass<M, 0, false, NT, false>(s2, s1, t2, t1);
}

}  // namespace mm
