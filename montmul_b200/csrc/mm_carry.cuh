// CRT and carry propagation for one vector per thread block (montmul/src/cpu.rs:117-129,
// 297-328; field.rs:288-294).
//
// A product's coefficients C_q < M31*M61 < 2^92 are summed as sum C_q 2^(32 q). Each thread
// owns E consecutive coefficients ("segment"), sums them locally into E limbs plus a carry
// c < 2^62 out of the segment, and block_resolve() finishes the sum: thread t adds c_(t-1),
// which leaves a carry of 0 or 1 out of each segment (a segment holds at least 64 bits), and
// those 0/1 carries are resolved at once by carry-lookahead: per warp, generate and propagate
// ballots G and Y = G | P give every lane's carry-in as the bits of (G + Y + cin) ^ G ^ Y; the
// same identity over the per-warp summaries gives each warp's carry-in.
#pragma once
#include "mm_ntt.cuh"

namespace mm {

MM_HD constexpr int cmax(int a, int b) { return a > b ? a : b; }

// Scratch words block_resolve needs: per-warp carries, the top carry, per-warp summaries.
template <int NT> struct CarryScratch { static constexpr int words = 2 * ((NT + 31) / 32) + 1; };

// Segments of E limbs on threads t < TA. `c` is the carry out of this thread's segment, `cin0`
// an extra carry into limb 0 of thread 0. Returns the carry out of the top segment, the same
// value on every thread; ends with a barrier so the scratch can be reused at once.
template <int E, int TA, int NT>
__device__ __forceinline__ uint64_t block_resolve(uint32_t (&L)[E], uint64_t c, uint64_t cin0, uint64_t* sc) {
    static_assert(E >= 2, "a segment must hold at least 64 bits");
    constexpr int W = (NT + 31) / 32;
    const int t = gtid<NT>(), lane = t & 31, w = t >> 5;
    const bool act = t < TA;
    if (lane == 31) sc[w] = c;
    if (t == TA - 1) sc[W] = c;
    gsync<NT>();
    const uint64_t up = __shfl_up_sync(0xffffffffu, c, 1);
    const uint64_t cin = (t == 0) ? cin0 : (lane == 0 ? sc[w - 1] : up);
    uint32_t r = 0;
    bool ones = true;
    if (act) {
        uint64_t acc = cin;
#pragma unroll
        for (int e = 0; e < E; ++e) {
            acc += L[e];
            L[e] = (uint32_t)acc;
            acc >>= 32;
            ones &= (L[e] == 0xffffffffu);
        }
        r = (uint32_t)acc;   // 0 or 1
    }
    const uint32_t G = __ballot_sync(0xffffffffu, r != 0);
    const uint32_t Y = G | __ballot_sync(0xffffffffu, ones);
    const uint64_t s = (uint64_t)G + Y;
    const uint32_t wgen = (uint32_t)(s >> 32);
    const uint32_t wprop = (Y == 0xffffffffu) && !wgen;
    uint64_t* summ = sc + W + 1;
    if (lane == 0) summ[w] = wgen | (wprop << 1);
    gsync<NT>();
    const uint64_t f = lane < W ? summ[lane] : 0;
    const uint32_t gw = __ballot_sync(0xffffffffu, f & 1);
    const uint32_t yw = gw | __ballot_sync(0xffffffffu, (f >> 1) & 1);
    const uint64_t sw = (uint64_t)gw + yw;
    const uint32_t cw = (uint32_t)sw ^ gw ^ yw;
    const uint32_t cl = (uint32_t)((uint64_t)G + Y + ((cw >> w) & 1)) ^ G ^ Y;
    if (act && ((cl >> lane) & 1)) {
        uint32_t b = 1;
#pragma unroll
        for (int e = 0; e < E; ++e) {
            uint32_t v = L[e] + b;
            b = b & (v == 0);
            L[e] = v;
        }
    }
    const uint64_t top = sc[W] + ((sw >> W) & 1);
    gsync<NT>();
    return top;
}

// 96-bit accumulate of a CRT value into the running segment sum.
struct Acc96 {
    uint32_t a0 = 0, a1 = 0, a2 = 0;   // running value (bits 0..95)
    __device__ __forceinline__ uint32_t add_shift(uint32_t w0, uint32_t w1, uint32_t w2) {
        unsigned __int128 v = ((unsigned __int128)a2 << 64) | ((uint64_t)a1 << 32) | a0;
        v += ((unsigned __int128)w2 << 64) | ((uint64_t)w1 << 32) | w0;
        uint32_t out = (uint32_t)v;
        v >>= 32;
        a0 = (uint32_t)v; a1 = (uint32_t)(v >> 32); a2 = (uint32_t)(v >> 64);
        return out;
    }
    __device__ __forceinline__ uint64_t rest() const { return ((uint64_t)a1 << 32) | a0; }  // a2 == 0 here
};

// T = sum C_q 2^(32 q) over the 2n coefficients of a product in natural order (coefficient q < n
// is re of element q, q >= n is im of element q - n), written to `out` (2n limbs, global).
// Returns the carry out of the top, which must be 0 for a product that fits.
template <int M, int NT>
__device__ __noinline__ uint64_t carry_product(const F2* s2, const F1* s1, uint32_t* __restrict__ out, uint64_t* sc) {
    constexpr int N = 1 << M, COUNT = 2 * N;
    constexpr int E = cmax(2, COUNT / NT), TA = COUNT / E;
    const int t = gtid<NT>();
    uint32_t L[E];
    uint64_t c = 0;
    const int q0 = t * E;
    if (t < TA) {
        const bool hi = q0 >= N;
        const int j0 = hi ? q0 - N : q0;
        Acc96 acc;
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const F2 a2 = s2[(swz(j0) ^ swz_c(e))];
            const F1 a1 = s1[(swz(j0) ^ swz_c(e))];
            uint32_t w0, w1, w2;
            crt3(hi ? a1.im : a1.re, hi ? a2.im : a2.re, w0, w1, w2);
            L[e] = acc.add_shift(w0, w1, w2);
        }
        c = acc.rest();
    } else {
#pragma unroll
        for (int e = 0; e < E; ++e) L[e] = 0;
    }
    const uint64_t top = block_resolve<E, TA, NT>(L, c, 0, sc);
    if (t < TA) {
#pragma unroll
        for (int e = 0; e < E; ++e) out[q0 + e] = L[e];
    }
    gsync<NT>();
    return top;
}

// m = low n limbs of the product in natural order (coefficients q < n: re of element q), then
// packed in place for the wraparound path as z_j = m_2j + i m_2j+1, j < n/2 (cpu.rs:286-295).
template <int M, int NT>
__device__ __noinline__ void carry_low_and_pack(F2* s2, F1* s1, uint64_t* sc) {
    constexpr int N = 1 << M, COUNT = N;
    constexpr int E = cmax(2, COUNT / NT), TA = COUNT / E;
    const int t = gtid<NT>();
    uint32_t L[E];
    uint64_t c = 0;
    const int q0 = t * E;
    if (t < TA) {
        Acc96 acc;
#pragma unroll
        for (int e = 0; e < E; ++e) {
            uint32_t w0, w1, w2;
            crt3(s1[(swz(q0) ^ swz_c(e))].re, s2[(swz(q0) ^ swz_c(e))].re, w0, w1, w2);
            L[e] = acc.add_shift(w0, w1, w2);
        }
        c = acc.rest();
    } else {
#pragma unroll
        for (int e = 0; e < E; ++e) L[e] = 0;
    }
    block_resolve<E, TA, NT>(L, c, 0, sc);   // the carry out of the top is dropped (mod R)
    if (t < TA) {
#pragma unroll
        for (int e = 0; e < E; e += 2) {
            // (q0 + e) / 2, q0 / 2 a multiple of E / 2: swz of the sum is the XOR of the parts
            const int sj = swz(q0 >> 1) ^ swz_c(e >> 1);
            F2 z2; z2.re = L[e]; z2.im = L[e + 1];
            uint32_t r0 = (L[e] & P1) + (L[e] >> 31), r1 = (L[e + 1] & P1) + (L[e + 1] >> 31);
            F1 z1; z1.re = min(r0, r0 - P1); z1.im = min(r1, r1 - P1);
            s2[sj] = z2;
            s1[sj] = z1;
        }
    }
    gsync<NT>();
}

// m = the low k limbs of a product whose low n coefficients are the real parts of the first n
// elements (k <= n), written to `out` (global); the REDC without the wraparound path
// (cpu.rs:459-462).
template <int M, int NT>
__device__ __noinline__ void carry_low_to(const F2* s2, const F1* s1, uint32_t* __restrict__ out, int k, uint64_t* sc) {
    constexpr int N = 1 << M, COUNT = N;
    constexpr int E = cmax(2, COUNT / NT), TA = COUNT / E;
    const int t = gtid<NT>();
    uint32_t L[E];
    uint64_t c = 0;
    const int q0 = t * E;
    if (t < TA) {
        Acc96 acc;
#pragma unroll
        for (int e = 0; e < E; ++e) {
            uint32_t w0, w1, w2;
            crt3(s1[(swz(q0) ^ swz_c(e))].re, s2[(swz(q0) ^ swz_c(e))].re, w0, w1, w2);
            L[e] = acc.add_shift(w0, w1, w2);
        }
        c = acc.rest();
    } else {
#pragma unroll
        for (int e = 0; e < E; ++e) L[e] = 0;
    }
    block_resolve<E, TA, NT>(L, c, 0, sc);   // limbs from k on are dropped (mod R)
    if (t < TA) {
#pragma unroll
        for (int e = 0; e < E; ++e)
            if (q0 + e < k) out[q0 + e] = L[e];
    }
    gsync<NT>();
}

// x = (T + m N) / R without the wraparound path (cpu.rs:470-481): the product m N in natural
// order (coefficient q < n in the real part of element q, q >= n in the imaginary part of element
// q - n) plus T's high half from limb k, plus `flag` (T mod R != 0: the low halves sum to R
// then) at limb k; limbs k .. 2k - 1 into x. Returns false when anything remains above them.
template <int M, int NT>
__device__ __noinline__ bool carry_shift_add(const F2* s2, const F1* s1, const uint32_t* __restrict__ tl,
                                             uint32_t* __restrict__ x, int k, uint32_t flag, uint64_t* sc) {
    constexpr int N = 1 << M, COUNT = 2 * N;
    constexpr int E = cmax(2, COUNT / NT), TA = COUNT / E;
    const int t = gtid<NT>();
    uint32_t L[E];
    uint64_t c = 0;
    const int q0 = t * E;
    if (t < TA) {
        const bool hi = q0 >= N;
        const int j0 = hi ? q0 - N : q0;
        Acc96 acc;
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const int q = q0 + e;
            const F2 a2 = s2[(swz(j0) ^ swz_c(e))];
            const F1 a1 = s1[(swz(j0) ^ swz_c(e))];
            uint32_t w0, w1, w2;
            crt3(hi ? a1.im : a1.re, hi ? a2.im : a2.re, w0, w1, w2);
            const uint64_t add = (q >= k && q < 2 * k ? (uint64_t)tl[q] : 0u) + (q == k ? flag : 0u);
            const uint64_t lo = (((uint64_t)w1 << 32) | w0) + add;
            w2 += lo < add;
            L[e] = acc.add_shift((uint32_t)lo, (uint32_t)(lo >> 32), w2);
        }
        c = acc.rest();
    } else {
#pragma unroll
        for (int e = 0; e < E; ++e) L[e] = 0;
    }
    const uint64_t top = block_resolve<E, TA, NT>(L, c, 0, sc);
    int stray = 0;
    if (t < TA) {
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const int q = q0 + e;
            if (q >= k && q < 2 * k) x[q - k] = L[e];
            else if (q >= 2 * k) stray |= L[e] != 0;
        }
    }
    return !gsync_or<NT>(stray) && top == 0;
}

// x = floor(T / R) + ((cyclic + T mod R) mod (R - 1)) with the cyclic product m N mod (R - 1)
// packed in the first n/2 elements (coefficient q: element q/2, re for even q, im for odd q),
// T (2n limbs) in global memory; writes x (n limbs). cpu.rs:297-328. Returns false when the
// final carry out is not 0 (a product that did not fit).
template <int M, int NT>
__device__ __noinline__ bool wrap_combine(const F2* s2, const F1* s1, const uint32_t* __restrict__ tl,
                                             uint32_t* __restrict__ x, uint64_t* sc) {
    constexpr int K = 1 << M, COUNT = K;
    constexpr int E = cmax(2, COUNT / NT), TA = COUNT / E;
    const int t = gtid<NT>();
    uint32_t L[E];
    uint64_t c = 0;
    const int q0 = t * E;
    if (t < TA) {
        Acc96 acc;
#pragma unroll
        for (int e = 0; e < E; e += 2) {
            // (q0 + e) / 2, q0 / 2 a multiple of E / 2: swz of the sum is the XOR of the parts
            const int sj = swz(q0 >> 1) ^ swz_c(e >> 1);
            const F2 a2 = s2[sj];
            const F1 a1 = s1[sj];
            uint32_t w0, w1, w2;
            crt3(a1.re, a2.re, w0, w1, w2);
            uint64_t lo = (((uint64_t)w1 << 32) | w0) + tl[q0 + e];
            w2 += lo < (uint64_t)tl[q0 + e];
            L[e] = acc.add_shift((uint32_t)lo, (uint32_t)(lo >> 32), w2);
            crt3(a1.im, a2.im, w0, w1, w2);
            lo = (((uint64_t)w1 << 32) | w0) + tl[q0 + e + 1];
            w2 += lo < (uint64_t)tl[q0 + e + 1];
            L[e + 1] = acc.add_shift((uint32_t)lo, (uint32_t)(lo >> 32), w2);
        }
        c = acc.rest();
    } else {
#pragma unroll
        for (int e = 0; e < E; ++e) L[e] = 0;
    }
    uint64_t top = block_resolve<E, TA, NT>(L, c, 0, sc);
    // End-around carry: 2^(32 k) = 1 mod R - 1.
    while (top != 0) top = block_resolve<E, TA, NT>(L, 0, top, sc);
    c = 0;
    if (t < TA) {
        uint64_t acc = 0;
#pragma unroll
        for (int e = 0; e < E; ++e) {
            acc += (uint64_t)L[e] + tl[K + q0 + e];
            L[e] = (uint32_t)acc;
            acc >>= 32;
        }
        c = acc;
    }
    top = block_resolve<E, TA, NT>(L, c, 0, sc);
    if (t < TA) {
#pragma unroll
        for (int e = 0; e < E; ++e) x[q0 + e] = L[e];
    }
    gsync<NT>();
    return top == 0;
}

}  // namespace mm
