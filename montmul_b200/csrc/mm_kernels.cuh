// The fused modular step and its set-up, one thread block per slot with the whole vector in
// shared memory (n <= 8192 elements of 24 bytes).
//
// One step (montmul/src/cpu.rs:486-497 with redc 452-484, wraparound path):
//   T = c x^2:       forward(x) -> square * c -> inverse -> carry into T (2k limbs, global)
//   m = T N' mod R:  forward(T mod R) -> * F(N') -> inverse -> carry (low k limbs), packed
//   m N mod (R-1):   half-length DIF -> e A + d B (cpu.rs:261-284) -> half-length DIT
//   x = T/R + ((m N + T mod R) mod (R - 1))  with the end-around carry, then + T high half.
// The exponent bit of every step is read on the device (transform.rs:67).
#pragma once
#include "mm_abi.h"
#include "mm_carry.cuh"

namespace mm {

// ---- pointwise operations of the fused pass (positions R g + k) ----
// apply2/apply1 transform the R values of group g in place; returning true stops the pass
// before the inverse butterflies (the spectrum was consumed).
struct SquareOp {
    uint32_t c;
    template <int R> __device__ __forceinline__ bool apply2(F2* x, int) const {
#pragma unroll
        for (int k = 0; k < R; ++k) x[k] = lsqr_scale(x[k], c);
        return false;
    }
    template <int R> __device__ __forceinline__ bool apply1(F1* x, int) const {
#pragma unroll
        for (int k = 0; k < R; ++k) { x[k] = csqr(x[k]); if (c != 1) x[k] = cscale(x[k], c); }
        return false;
    }
};

// Multiplies by a spectrum stored in fused-pass order (element k * (n / R) + g).
template <int M> struct SpecMulOp {
    const F2* b2; const F1* b1;
    template <int R> __device__ __forceinline__ bool apply2(F2* x, int g) const {
#pragma unroll
        for (int k = 0; k < R; ++k) x[k] = lkmulc(x[k], b2[k * ((1 << M) / R) + g]);
        return false;
    }
    template <int R> __device__ __forceinline__ bool apply1(F1* x, int g) const {
#pragma unroll
        for (int k = 0; k < R; ++k) x[k] = cmul(x[k], b1[k * ((1 << M) / R) + g]);
        return false;
    }
};

// Stores the spectrum (canonical, as every multiplier constant is) in fused-pass order and
// stops (no inverse).
template <int M> struct SpecStoreOp {
    F2* b2; F1* b1;
    template <int R> __device__ __forceinline__ bool apply2(F2* x, int g) const {
#pragma unroll
        for (int k = 0; k < R; ++k) b2[k * ((1 << M) / R) + g] = lccanon(x[k]);
        return true;
    }
    template <int R> __device__ __forceinline__ bool apply1(F1* x, int g) const {
#pragma unroll
        for (int k = 0; k < R; ++k) b1[k * ((1 << M) / R) + g] = x[k];
        return true;
    }
};

// ---- the wraparound half-pointwise step (cpu.rs:221-237, 261-284) ----
// out_p = (z_p + conj z_q) A_p + (z_p - conj z_q) B_p with q = partner(p), the position of
// index (h - rev(p)) mod h; in place, one thread per pair {p, q} (q = 3 * 2^a - 1 - p for p in
// octave [2^a, 2^(a+1)), q = p for p < 2). The vector (h elements at swz(p)) may be in shared
// or global memory.
__device__ __forceinline__ void half_pointwise_pair(F2* s2, F1* s1, int H, const F2* __restrict__ ab2,
                                                    const F1* __restrict__ ab1, int tau) {
    const int p = tau < 2 ? tau : tau - 1 + (1 << (31 - __clz(tau - 1)));
    const int q = p == 0 ? 0 : (3 << (31 - __clz(p))) - 1 - p;
    {
        // e = z_p + conj z_q, d = z_p - conj z_q on reduced values, then e A + d B.
        const F2 zp = s2[swz(p)], zq = s2[swz(q)];
        const F2 e = lcfold(f2(zp.re + zq.re, zp.im + lsub<2>(0, zq.im)));
        const F2 d = lcfold(f2(lsub<2>(zp.re, zq.re), zp.im + zq.im));
        const F2 op = lcfold(lcadd(lkmulc(e, ab2[p]), lkmulc(d, ab2[H + p])));
        if (q != p) {
            const F2 e2 = lcfold(f2(zq.re + zp.re, zq.im + lsub<2>(0, zp.im)));
            const F2 d2 = lcfold(f2(lsub<2>(zq.re, zp.re), zq.im + zp.im));
            s2[swz(q)] = lcfold(lcadd(lkmulc(e2, ab2[q]), lkmulc(d2, ab2[H + q])));
        }
        s2[swz(p)] = op;
    }
    {
        const F1 zp = s1[swz(p)], zq = s1[swz(q)];
        const F1 e = cadd(zp, cconj(zq)), d = csub(zp, cconj(zq));
        const F1 op = cadd(cmul(e, ab1[p]), cmul(d, ab1[H + p]));
        if (q != p) {
            const F1 e2 = cadd(zq, cconj(zp)), d2 = csub(zq, cconj(zp));
            s1[swz(q)] = cadd(cmul(e2, ab1[q]), cmul(d2, ab1[H + q]));
        }
        s1[swz(p)] = op;
    }
}

template <int MH, int NT>
__device__ __noinline__ void half_pointwise(F2* s2, F1* s1, const F2* __restrict__ ab2, const F1* __restrict__ ab1) {
    constexpr int H = 1 << MH;
#pragma unroll 1
    for (int tau = gtid<NT>(); tau < H / 2 + 1; tau += NT) half_pointwise_pair(s2, s1, H, ab2, ab1, tau);
    gsync<NT>();
}

// half_forward's packing (cpu.rs:286-295): z_j = v_2j + i v_2j+1 for j < h, at swz(j). Ends
// with a barrier.
__device__ __forceinline__ void pack_pairs(const uint32_t* __restrict__ v, F2* s2, F1* s1, int H, int nt) {
    for (int j = threadIdx.x; j < H; j += nt) {
        const uint32_t v0 = v[2 * j], v1 = v[2 * j + 1];
        F2 z2; z2.re = v0; z2.im = v1;
        const uint32_t r0 = (v0 & P1) + (v0 >> 31), r1 = (v1 & P1) + (v1 >> 31);
        F1 z1; z1.re = min(r0, r0 - P1); z1.im = min(r1, r1 - P1);
        s2[swz(j)] = z2;
        s1[swz(j)] = z1;
    }
    __syncthreads();
}

// ---- wraparound factors of one modulus from the half transform of N (cpu.rs:239-284) ----
// In: the unweighted length-h DIF of z_j = N_2j + i N_2j+1 in elements [0, h) (at swz). Writes
// half_nhat into elements [h, 2h), then A (ab[p]) and B (ab[h + p]). u: unpack roots w^rev(p)
// (p < h) and w^-rev(p) (h + p). inv8h = (8 h)^-1. Ends with a barrier.
__device__ __forceinline__ void half_factors_block(F2* s2, F1* s1, int H, const F2K* u2, const F1* u1, F2* ab2, F1* ab1,
                                                   F2 inv8h2, F1 inv8h1, int nt) {
    // half_nhat (cpu.rs:239-249) into elements h..2h.
    for (int p = threadIdx.x; p < H; p += nt) {
        const int q = p < 2 ? p : (3 << (31 - __clz(p))) - 1 - p;
        {
            const F2 zk = lccanon(s2[swz(p)]), zj = cconj(lccanon(s2[swz(q)]));
            const F2 e = cadd(zk, zj), wo = cmul(mul_mi(csub(zk, zj)), f2(u2[p].re, u2[p].im));
            const F2 xx = cadd(e, wo), yy = csub(e, wo);
            s2[swz(H + p)] = p == 0 ? cadd(cmul(xx, inv8h2), mul_i(cmul(yy, inv8h2))) : cmul(xx, inv8h2);
        }
        {
            const F1 zk = s1[swz(p)], zj = cconj(s1[swz(q)]);
            const F1 e = cadd(zk, zj), wo = cmul(mul_mi(csub(zk, zj)), u1[p]);
            const F1 xx = cadd(e, wo), yy = csub(e, wo);
            s1[swz(H + p)] = p == 0 ? cadd(cmul(xx, inv8h1), mul_i(cmul(yy, inv8h1))) : cmul(xx, inv8h1);
        }
    }
    __syncthreads();
    // half_factors (cpu.rs:265-277): A at offset 0, B at h.
    for (int p = threadIdx.x; p < H; p += nt) {
        const int q = p < 2 ? p : (3 << (31 - __clz(p))) - 1 - p;
        {
            const F2 sp = s2[swz(H + p)], sq = s2[swz(H + q)];
            const F2 nx = p == 0 ? f2(sp.re, 0) : sp, ny = p == 0 ? f2(sp.im, 0) : cconj(sq);
            const F2 iu = f2(u2[H + p].re, u2[H + p].im), iiu = mul_i(iu);
            const F2 X = cmul(nx, f2(add2(1, iiu.re), iiu.im)), Y = cmul(ny, f2(sub2(1, iiu.re), sub2(0, iiu.im)));
            ab2[p] = cadd(X, Y);
            ab2[H + p] = cmul(mul_mi(csub(X, Y)), f2(u2[p].re, u2[p].im));
        }
        {
            const F1 sp = s1[swz(H + p)], sq = s1[swz(H + q)];
            const F1 nx = p == 0 ? f1(sp.re, 0) : sp, ny = p == 0 ? f1(sp.im, 0) : cconj(sq);
            const F1 iu = u1[H + p], iiu = mul_i(iu);
            const F1 X = cmul(nx, f1(add1(1, iiu.re), iiu.im)), Y = cmul(ny, f1(sub1(1, iiu.re), sub1(0, iiu.im)));
            ab1[p] = cadd(X, Y);
            ab1[H + p] = cmul(mul_mi(csub(X, Y)), u1[p]);
        }
    }
    __syncthreads();
}

// The Transform trait's forward (weight by zeta^j, DIF) or inverse (DIT, unweight by
// zeta^-j / n) of vector first + blockIdx.x, in place in a device buffer whose element order is
// the kernels' (element j at swz(j)); the result is canonical (cpu.rs:86-103, 349-407).
template <int M, int NT>
__global__ void __launch_bounds__(NT) transform_kernel(F2* v2, F1* v1, const F2K* tab2, const F1* tab1, uint32_t first,
                                                       int inverse) {
    constexpr int N = 1 << M, P = sched_passes(M);
    extern __shared__ __align__(16) unsigned char smem_raw[];
    F2* s2 = reinterpret_cast<F2*>(smem_raw);
    F1* s1 = reinterpret_cast<F1*>(smem_raw + 16 * N);
    F2* g2 = v2 + (size_t)(first + blockIdx.x) * N;
    F1* g1 = v1 + (size_t)(first + blockIdx.x) * N;
    for (int e = gtid<NT>(); e < N; e += NT) {
        s2[e] = g2[e];
        s1[e] = g1[e];
    }
    gsync<NT>();
    if (!inverse) {
        dif_first_complex<M, NT>(s2, s1, tab2, tab1);
        if constexpr (P >= 2) smem_pass<M, (P >= 2 ? 1 : 0), true, NT, true>(s2, s1, tab2, tab1);
        if constexpr (P >= 3) smem_pass<M, (P >= 3 ? 2 : 0), true, NT, true>(s2, s1, tab2, tab1);
        if constexpr (P >= 4) smem_pass<M, (P >= 4 ? 3 : 0), true, NT, true>(s2, s1, tab2, tab1);
        if constexpr (P >= 5) smem_pass<M, (P >= 5 ? 4 : 0), true, NT, true>(s2, s1, tab2, tab1);
    } else {
        if constexpr (P >= 5) smem_pass<M, (P >= 5 ? 4 : 0), false, NT, true>(s2, s1, tab2, tab1);
        if constexpr (P >= 4) smem_pass<M, (P >= 4 ? 3 : 0), false, NT, true>(s2, s1, tab2, tab1);
        if constexpr (P >= 3) smem_pass<M, (P >= 3 ? 2 : 0), false, NT, true>(s2, s1, tab2, tab1);
        if constexpr (P >= 2) smem_pass<M, (P >= 2 ? 1 : 0), false, NT, true>(s2, s1, tab2, tab1);
        dit_last_complex<M, NT>(s2, s1, tab2, tab1);
    }
    for (int e = gtid<NT>(); e < N; e += NT) {
        g2[e] = lccanon(s2[e]);
        g1[e] = s1[e];
    }
}

// Shared memory of one block: F2 vector (16 n B), F1 vector (8 n B).
template <int M> constexpr int smem_bytes() { return 24 << M; }

// REDC from T (in tl, 2n limbs) into x (n limbs), wraparound path. Returns false on a carry
// out that must vanish.
template <int M, int NT>
__device__ __noinline__ bool redc_wrap(F2* s2, F1* s1, const uint32_t* tl, uint32_t* x, const F2* cc2, const F1* cc1,
                                          const F2K* tab2, const F1* tab1, uint64_t* sc) {
    constexpr int N = 1 << M;
    const F2K* ht2 = tab2 + lt_half_off(M);
    const F1* ht1 = tab1 + lt_half_off(M);
    fwd_limbs<M, NT>(tl, N, s2, s1, tab2, tab1);
    fused_mid<M, NT, true>(tl, N, s2, s1, tab2, tab1, SpecMulOp<M>{cc2, cc1});
    inv_to_natural<M, NT, true>(s2, s1, tab2, tab1);
    carry_low_and_pack<M, NT>(s2, s1, sc);
    dif_unweighted<M - 1, NT>(s2, s1, ht2, ht1);
    half_pointwise<M - 1, NT>(s2, s1, cc2 + N, cc1 + N);
    dit_unweighted<M - 1, NT>(s2, s1, ht2, ht1);
    return wrap_combine<M, NT>(s2, s1, tl, x, sc);
}

// REDC without the wraparound path (cpu.rs:453-484 with half = None), k <= n limbs: m = (T mod R)
// N' mod R through F(N'), then m N through F(N) (both in cc, fused-pass order), and
// x = T_high + (m N)_high + [T mod R != 0]. m overwrites x, which the step no longer needs.
template <int M, int NT>
__device__ __noinline__ bool redc_plain(F2* s2, F1* s1, const uint32_t* tl, uint32_t* x, const F2* cc2, const F1* cc1,
                                        const F2K* tab2, const F1* tab1, uint64_t* sc, int k) {
    constexpr int N = 1 << M;
    int nz = 0;
    for (int q = gtid<NT>(); q < k; q += NT) nz |= tl[q] != 0;
    const uint32_t flag = gsync_or<NT>(nz) ? 1u : 0u;
    fwd_limbs<M, NT>(tl, k, s2, s1, tab2, tab1);
    fused_mid<M, NT, true>(tl, k, s2, s1, tab2, tab1, SpecMulOp<M>{cc2, cc1});
    inv_to_natural<M, NT, true>(s2, s1, tab2, tab1);
    carry_low_to<M, NT>(s2, s1, x, k, sc);
    fwd_limbs<M, NT>(x, k, s2, s1, tab2, tab1);
    fused_mid<M, NT, false>(x, k, s2, s1, tab2, tab1, SpecMulOp<M>{cc2 + N, cc1 + N});
    inv_to_natural<M, NT, false>(s2, s1, tab2, tab1);
    return carry_shift_add<M, NT>(s2, s1, tl, x, k, flag, sc);
}

// Up to `bits` steps x <- x^2 c^bit R^-1 on one slot (cpu.rs:543-556), the whole block, the
// vector in `smem_raw` (24 n bytes). Used by the uniform launch and the mixed-length launch.
// With a.bare each step ends after T = c x^2 and x stays as it was (the reference's run_bare,
// lib.rs:883-927, which times the squaring alone).
template <int M, int NT>
__device__ __forceinline__ void step_slot(const SlotArgs& a, uint32_t slot, uint32_t bits, unsigned char* smem_raw,
                                          uint64_t* sc) {
    constexpr int N = 1 << M;
    F2* s2 = reinterpret_cast<F2*>(smem_raw);
    F1* s1 = reinterpret_cast<F1*>(smem_raw + 16 * N);
    const int k = (int)a.k;
    uint32_t* x = a.x + (size_t)slot * k;
    uint32_t* tl = a.tbuf + (size_t)slot * 2 * N;
    const F2* cc2 = a.c2 + (size_t)slot * 2 * N;
    const F1* cc1 = a.c1 + (size_t)slot * 2 * N;
    const uint32_t* ex = a.exp + (size_t)slot * a.ew;
    const uint32_t nb = a.nbits[slot];
    uint32_t pos = a.pos[slot];
    bool ok = true;
    for (uint32_t it = 0; it < bits && pos < nb; ++it, ++pos) {
        const uint32_t bit = (ex[pos >> 5] >> (31 - (pos & 31))) & 1;
        const uint32_t c = bit ? a.base : 1;
        fwd_limbs<M, NT>(x, k, s2, s1, a.tab2, a.tab1);
        fused_mid<M, NT, false>(x, k, s2, s1, a.tab2, a.tab1, SquareOp{c});
        inv_to_natural<M, NT, false>(s2, s1, a.tab2, a.tab1);
        ok &= carry_product<M, NT>(s2, s1, tl, sc) == 0;
        if (a.bare) continue;
        if (a.plain) ok &= redc_plain<M, NT>(s2, s1, tl, x, cc2, cc1, a.tab2, a.tab1, sc, k);
        else ok &= redc_wrap<M, NT>(s2, s1, tl, x, cc2, cc1, a.tab2, a.tab1, sc);
    }
    gsync<NT>();   // every thread has read pos before it is written
    if (gtid<NT>() == 0) {
        a.pos[slot] = pos;
        if (!ok) a.err[slot] = 1;
    }
}

// The uniform launch: one block per slot first + blockIdx.x, `bits` steps each; or, with an item
// list, one block per item (slot, steps) of the list (a serving tick's launch over the busy slots
// of a batch; each slot at most once).
template <int M, int NT, int MINB = (M <= 12 ? 2 : 1)>
__global__ void __launch_bounds__(NT, MINB)
    step_kernel(SlotArgs a, uint32_t first, uint32_t bits, const uint2* __restrict__ items) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ uint64_t sc[CarryScratch<NT>::words];
    if (items) {
        const uint2 it = items[blockIdx.x];
        step_slot<M, NT>(a, it.x, it.y, smem_raw, sc);
    } else {
        step_slot<M, NT>(a, first + blockIdx.x, bits, smem_raw, sc);
    }
}

// x[out] <- x[ia] x[ib] R^-1 with slot out's modulus (cpu.rs:558-571), one block. spec: n
// elements of scratch for F(x[ib]).
template <int M, int NT>
__global__ void __launch_bounds__(NT) mul_kernel(SlotArgs a, uint32_t out, uint32_t ia, uint32_t ib, F2* spec2, F1* spec1) {
    constexpr int N = 1 << M;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    F2* s2 = reinterpret_cast<F2*>(smem_raw);
    F1* s1 = reinterpret_cast<F1*>(smem_raw + 16 * N);
    __shared__ uint64_t sc[CarryScratch<NT>::words];
    const int k = (int)a.k;
    const uint32_t* xb = a.x + (size_t)ib * k;
    const uint32_t* xa = a.x + (size_t)ia * k;
    fwd_limbs<M, NT>(xb, k, s2, s1, a.tab2, a.tab1);
    fused_mid<M, NT, false>(xb, k, s2, s1, a.tab2, a.tab1, SpecStoreOp<M>{spec2, spec1});
    gsync<NT>();
    fwd_limbs<M, NT>(xa, k, s2, s1, a.tab2, a.tab1);
    fused_mid<M, NT, false>(xa, k, s2, s1, a.tab2, a.tab1, SpecMulOp<M>{spec2, spec1});
    inv_to_natural<M, NT, false>(s2, s1, a.tab2, a.tab1);
    uint32_t* tl = a.tbuf + (size_t)out * 2 * N;
    bool ok = carry_product<M, NT>(s2, s1, tl, sc) == 0;
    uint32_t* xo = a.x + (size_t)out * k;
    if (a.plain)
        ok &= redc_plain<M, NT>(s2, s1, tl, xo, a.c2 + (size_t)out * 2 * N, a.c1 + (size_t)out * 2 * N, a.tab2, a.tab1,
                                sc, k);
    else
        ok &= redc_wrap<M, NT>(s2, s1, tl, xo, a.c2 + (size_t)out * 2 * N, a.c1 + (size_t)out * 2 * N, a.tab2, a.tab1, sc);
    if (gtid<NT>() == 0 && !ok) a.err[out] = 1;
}

// Per-slot constants of slot first + blockIdx.x (or slots[blockIdx.x]) from its N and N' limbs
// (k = n each):
// F(N') in fused-pass order (cpu.rs:518), then the wraparound factors A | B from the half
// transform of N (cpu.rs:239-284; computed on the host by the reference's GPU backend).
// inv8h = (8 h)^-1 in each field.
template <int M, int NT>
__global__ void __launch_bounds__(NT) setup_kernel(const uint32_t* nl, const uint32_t* npl, F2* c2, F1* c1, const F2K* tab2,
                                                   const F1* tab1, F2 inv8h2, F1 inv8h1, uint32_t first,
                                                   const uint32_t* slots, uint32_t k, int plain) {
    constexpr int N = 1 << M, H = N / 2;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    F2* s2 = reinterpret_cast<F2*>(smem_raw);
    F1* s1 = reinterpret_cast<F1*>(smem_raw + 16 * N);
    // Rows of nl / npl (k limbs each): all slots from `first` on, or (with a slot list) one row
    // per listed slot.
    const uint32_t slot = slots ? slots[blockIdx.x] : first + blockIdx.x;
    const size_t row = slots ? blockIdx.x : slot;
    const uint32_t* np = npl + row * k;
    const uint32_t* nn = nl + row * k;
    F2* o2 = c2 + (size_t)slot * 2 * N;
    F1* o1 = c1 + (size_t)slot * 2 * N;
    fwd_limbs<M, NT>(np, (int)k, s2, s1, tab2, tab1);
    fused_mid<M, NT, false>(np, (int)k, s2, s1, tab2, tab1, SpecStoreOp<M>{o2, o1});
    gsync<NT>();
    if (plain) {
        // F(N) in the second half (cpu.rs:518-521), in fused-pass order.
        fwd_limbs<M, NT>(nn, (int)k, s2, s1, tab2, tab1);
        fused_mid<M, NT, false>(nn, (int)k, s2, s1, tab2, tab1, SpecStoreOp<M>{o2 + N, o1 + N});
        return;
    }
    pack_pairs(nn, s2, s1, H, NT);
    const F2K* ht2 = tab2 + lt_half_off(M);
    const F1* ht1 = tab1 + lt_half_off(M);
    dif_unweighted<M - 1, NT>(s2, s1, ht2, ht1);
    half_factors_block(s2, s1, H, tab2 + lt_unpack_off(M), tab1 + lt_unpack_off(M), o2 + N, o1 + N, inv8h2, inv8h1, NT);
}

}  // namespace mm
