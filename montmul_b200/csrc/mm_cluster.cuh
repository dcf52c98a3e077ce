// Cluster mode: lengths whose vector exceeds one SM's shared memory but fits a thread-block
// cluster's. n = 2^M elements (M = 14, 15: L = 32768, 65536) are spread over C = n / 8192 CTAs
// of one cluster, 8,192 elements (192 KiB, the F2 then F1 arrays at swz positions) in each CTA's
// shared memory; the CTAs reach each other's chunks through distributed shared memory. The
// reference runs these lengths in global memory (kernels/src/lib.rs:455-511); here nothing of
// the vector leaves the chip:
//   - every pass whose groups stay inside 8,192 elements (all but the first radix pass of each
//     transform, for these lengths) is the shared-mode pass on the CTA's own chunk;
//   - the first DIF pass and the last DIT pass of each transform, and the wraparound
//     half-pointwise step, read and write across CTAs, then the cluster synchronizes;
//   - carries run over the whole cluster: each CTA owns a contiguous piece of the coefficient
//     chain, and the 0/1 carries left after the segment sums resolve by lookahead at three
//     levels: lanes (ballots), warps (per-warp summaries) and CTAs (per-CTA summaries exchanged
//     through distributed shared memory).
// The per-slot constants, x, T and the exponent state are global mode's, so a batch switches
// between global and cluster mode at any time.
#pragma once
#include <cooperative_groups.h>

#include "mm_global.cuh"

namespace mm {

namespace cgx = cooperative_groups;

constexpr int kChunkLog = kClusterChunkLog;     // elements per CTA by default: 2^13
constexpr int kChunk = 1 << kChunkLog;
constexpr int kClusterThreads = 512;
constexpr int kClusterSmem = 24 * kChunk;      // 192 KiB

// The chunks of every CTA of the cluster, as generic pointers (the own chunk included).
template <int C> struct Chunks {
    F2* c2[C];
    F1* c1[C];
    // Element e of a vector spread in chunks of 2^LOG elements.
    template <int LOG> __device__ __forceinline__ F2& e2(int e) const { return c2[e >> LOG][swz(e & ((1 << LOG) - 1))]; }
    template <int LOG> __device__ __forceinline__ F1& e1(int e) const { return c1[e >> LOG][swz(e & ((1 << LOG) - 1))]; }
};

// Element j + k Q of a vector spread in chunks of 2^LOG elements, for j < Q where Q divides the
// chunk length: its chunk, (k Q) >> LOG, and its position's swz offset, swz((k Q) mod 2^LOG), are
// fixed by k, so an unrolled loop over k addresses it with the chunk pointers in registers and
// swz(j) ^ a constant (swz is linear over XOR, and j and (k Q) mod 2^LOG have disjoint bits).
template <int LOG, int Q> __device__ __forceinline__ constexpr int kchunk(int k) { return (k * Q) >> LOG; }
template <int LOG, int Q> __device__ __forceinline__ constexpr int koff(int k) { return swz_c((k * Q) & ((1 << LOG) - 1)); }
template <int C> struct ChunkRegs {
    F2* c2[C];
    F1* c1[C];
    __device__ __forceinline__ explicit ChunkRegs(const Chunks<C>& ch) {
#pragma unroll
        for (int d = 0; d < C; ++d) { c2[d] = ch.c2[d]; c1[d] = ch.c1[d]; }
    }
};

// Per-CTA scratch of the cluster carry (each CTA's own copy; peers write into it).
struct ClusterCarry {
    uint64_t cin_prev;   // segment carry of the previous CTA's last thread
    uint64_t top;        // the chain's carry out, from the last CTA
    uint32_t summ[8];    // per CTA: bit 0 generates a carry, bit 1 propagates one
};

// The 0/1-carry resolution of block_resolve (mm_carry.cuh) over a chain spread across the
// cluster: CTA r owns the chain piece after CTA r - 1's, every thread of it a segment of E limbs
// with segment carry c; cin0 enters limb 0 of CTA 0's thread 0. Returns the carry out of the
// top of the chain on every thread of every CTA; ends with a cluster barrier.
template <int E, int NT, int C>
__device__ __forceinline__ uint64_t cluster_resolve(uint32_t (&L)[E], uint64_t c, uint64_t cin0, uint64_t* sc,
                                                    ClusterCarry* cc, const cgx::cluster_group& cl) {
    static_assert(E >= 2 && C <= 8, "segments of 64 bits or more, at most 8 CTAs");
    constexpr int W = NT / 32;
    constexpr uint32_t kWarpMask = W == 32 ? 0xffffffffu : ((1u << W) - 1u);
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    const int r = (int)cl.block_rank();
    if (lane == 31) sc[w] = c;
    if (t == NT - 1) {
        sc[W] = c;
        if (r + 1 < C) cl.map_shared_rank(cc, r + 1)->cin_prev = c;
    }
    cl.sync();
    const uint64_t up = __shfl_up_sync(0xffffffffu, c, 1);
    const uint64_t cin = t == 0 ? (r == 0 ? cin0 : cc->cin_prev) : (lane == 0 ? sc[w - 1] : up);
    uint64_t acc = cin;
    bool ones = true;
#pragma unroll
    for (int e = 0; e < E; ++e) {
        acc += L[e];
        L[e] = (uint32_t)acc;
        acc >>= 32;
        ones &= (L[e] == 0xffffffffu);
    }
    const uint32_t rb = (uint32_t)acc;   // 0 or 1
    const uint32_t G = __ballot_sync(0xffffffffu, rb != 0);
    const uint32_t Y = G | __ballot_sync(0xffffffffu, ones);
    const uint64_t s = (uint64_t)G + Y;
    uint64_t* summ = sc + W + 1;
    if (lane == 0) summ[w] = (uint32_t)(s >> 32) | (uint32_t)((Y == 0xffffffffu) && !(s >> 32)) << 1;
    __syncthreads();
    const uint64_t f = lane < W ? summ[lane] : 0;
    const uint32_t gw = __ballot_sync(0xffffffffu, f & 1);
    const uint32_t yw = gw | __ballot_sync(0xffffffffu, (f >> 1) & 1);
    if (t == 0) {
        const uint32_t gen = (uint32_t)((((uint64_t)gw + yw) >> W) & 1);
        const uint32_t prop = (yw == kWarpMask) && !gen;
        for (int d = 0; d < C; ++d) cl.map_shared_rank(cc, d)->summ[r] = gen | prop << 1;
    }
    cl.sync();
    uint32_t ccin = 0;   // carry into this CTA's piece from the pieces below
#pragma unroll
    for (int d = 0; d < C - 1; ++d) {
        if (d < r) {
            const uint32_t sd = cc->summ[d];
            ccin = (sd & 1) | ((sd >> 1) & ccin);
        }
    }
    const uint64_t sw = (uint64_t)gw + yw + ccin;
    const uint32_t cw = (uint32_t)sw ^ gw ^ yw;
    const uint32_t cl_in = (uint32_t)((uint64_t)G + Y + ((cw >> w) & 1)) ^ G ^ Y;
    if ((cl_in >> lane) & 1) {
        uint32_t b = 1;
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const uint32_t v = L[e] + b;
            b = b & (v == 0);
            L[e] = v;
        }
    }
    if (r == C - 1 && t == 0) {
        const uint64_t top = sc[W] + ((sw >> W) & 1);
        for (int d = 0; d < C; ++d) cl.map_shared_rank(cc, d)->top = top;
    }
    cl.sync();
    return cc->top;
}

// ---- passes that cross CTAs ----
// The weighted first DIF pass of the length-2^M transform straight from real limbs (as
// dif_first_from_limbs): CTA r does groups [r Q / C, (r + 1) Q / C) and writes every CTA's chunk.
template <int M, int NT, int C>
__device__ __noinline__ void cl_dif_first(const uint32_t* __restrict__ lim, int cnt, const Chunks<C>& ch, const F2K* tab2,
                                          const F1* tab1, const cgx::cluster_group& cl) {
    constexpr int R = sched_radix(M, 0), Q = (1 << M) / R, QC = Q / C, CL = M - ilog2c(C);
    constexpr int toff = tab_fwd_off(M, 0, true), coff = tab_in_const_off(M, true);
    // Every CTA has started, the limbs other CTAs wrote (x, T) are visible, and no CTA still
    // reads the chunks this pass overwrites.
    cl.sync();
    const int j0 = (int)cl.block_rank() * QC;
    const ChunkRegs<C> cr(ch);
    static_assert((1 << CL) % Q == 0, "the passes' spans divide the chunk length");
#pragma unroll 1
    for (int j = j0 + (int)threadIdx.x; j < j0 + QC; j += NT) {
        const int sj = swz(j);
        uint32_t v[R];
#pragma unroll
        for (int k = 0; k < R; ++k) v[k] = (j + k * Q < cnt) ? lim[j + k * Q] : 0u;
        {
            F2 x[R];
#pragma unroll
            for (int k = 0; k < R; ++k) x[k] = lreal_times(v[k], tab2[coff + k]);
            ldif<R>(x);
#pragma unroll
            for (int k = 0; k < R; ++k) cr.c2[kchunk<CL, Q>(k)][sj ^ koff<CL, Q>(k)] = lkmul(lcfold(x[k]), tab2[toff + k * Q + j]);
        }
        {
            F1 x[R];
#pragma unroll
            for (int k = 0; k < R; ++k) x[k] = real_times<F1>(v[k], tab1[coff + k]);
            bf_dif<R, F1>(x);
#pragma unroll
            for (int k = 0; k < R; ++k) cr.c1[kchunk<CL, Q>(k)][sj ^ koff<CL, Q>(k)] = cmul(x[k], tab1[toff + k * Q + j]);
        }
    }
    cl.sync();
}

// The weighted last DIT pass (as dit_last_weighted), into natural order across the chunks.
template <int M, int NT, int C, bool REAL_ONLY>
__device__ __noinline__ void cl_dit_last(const Chunks<C>& ch, const F2K* tab2, const F1* tab1, const cgx::cluster_group& cl) {
    constexpr int R = sched_radix(M, 0), Q = (1 << M) / R, QC = Q / C, CL = M - ilog2c(C);
    constexpr int toff = tab_inv_off(M, 0, true), coff = tab_out_const_off(M, true);
    cl.sync();   // the local passes before this one wrote every chunk
    const int j0 = (int)cl.block_rank() * QC;
    const ChunkRegs<C> cr(ch);
    static_assert((1 << CL) % Q == 0, "the passes' spans divide the chunk length");
#pragma unroll 1
    for (int j = j0 + (int)threadIdx.x; j < j0 + QC; j += NT) {
        const int sj = swz(j);
        {
            F2 x[R];
#pragma unroll
            for (int k = 0; k < R; ++k) x[k] = lkmul(cr.c2[kchunk<CL, Q>(k)][sj ^ koff<CL, Q>(k)], tab2[toff + k * Q + j]);
            ldit<R>(x);
#pragma unroll
            for (int k = 0; k < R; ++k) {
                if (REAL_ONLY) cr.c2[kchunk<CL, Q>(k)][sj ^ koff<CL, Q>(k)].re = lkmul_re(x[k], tab2[coff + k]);
                else cr.c2[kchunk<CL, Q>(k)][sj ^ koff<CL, Q>(k)] = lkmul(x[k], tab2[coff + k]);
            }
        }
        {
            F1 x[R];
#pragma unroll
            for (int k = 0; k < R; ++k) x[k] = cmul(cr.c1[kchunk<CL, Q>(k)][sj ^ koff<CL, Q>(k)], tab1[toff + k * Q + j]);
            bf_dit<R, F1>(x);
#pragma unroll
            for (int k = 0; k < R; ++k) {
                if (REAL_ONLY) cr.c1[kchunk<CL, Q>(k)][sj ^ koff<CL, Q>(k)].re = cmul_re(x[k], tab1[coff + k]);
                else cr.c1[kchunk<CL, Q>(k)][sj ^ koff<CL, Q>(k)] = cmul(x[k], tab1[coff + k]);
            }
        }
    }
    cl.sync();
}

// The first (DIF) or last (DIT) pass of the unweighted half-length transform (length 2^MH over
// chunks of 2^MH / C elements per CTA), across CTAs.
template <int MH, bool FWD, int NT, int C>
__device__ __noinline__ void cl_half_pass0(const Chunks<C>& ch, const F2K* ht2, const F1* ht1, const cgx::cluster_group& cl) {
    constexpr int R = sched_radix(MH, 0), Q = (1 << MH) / R, QC = Q / C, LOG = MH - ilog2c(C);
    constexpr int toff = FWD ? tab_fwd_off(MH, 0, false) : tab_inv_off(MH, 0, false);
    static_assert(Q > 1, "the half transform has more than one pass");
    if (!FWD) cl.sync();
    const int j0 = (int)cl.block_rank() * QC;
    const ChunkRegs<C> cr(ch);
    static_assert((1 << LOG) % Q == 0, "the passes' spans divide the chunk length");
#pragma unroll 1
    for (int j = j0 + (int)threadIdx.x; j < j0 + QC; j += NT) {
        const int sj = swz(j);
        {
            F2 x[R];
#pragma unroll
            for (int k = 0; k < R; ++k) x[k] = cr.c2[kchunk<LOG, Q>(k)][sj ^ koff<LOG, Q>(k)];
            if (FWD) {
                ldif<R>(x);
                x[0] = lcfold(x[0]);
#pragma unroll
                for (int k = 1; k < R; ++k) x[k] = lkmul(lcfold(x[k]), ht2[toff + (k - 1) * Q + j]);
            } else {
#pragma unroll
                for (int k = 1; k < R; ++k) x[k] = lkmul(x[k], ht2[toff + (k - 1) * Q + j]);
                ldit<R>(x);
            }
#pragma unroll
            for (int k = 0; k < R; ++k) cr.c2[kchunk<LOG, Q>(k)][sj ^ koff<LOG, Q>(k)] = x[k];
        }
        {
            F1 x[R];
#pragma unroll
            for (int k = 0; k < R; ++k) x[k] = cr.c1[kchunk<LOG, Q>(k)][sj ^ koff<LOG, Q>(k)];
            if (FWD) {
                bf_dif<R, F1>(x);
#pragma unroll
                for (int k = 1; k < R; ++k) x[k] = cmul(x[k], ht1[toff + (k - 1) * Q + j]);
            } else {
#pragma unroll
                for (int k = 1; k < R; ++k) x[k] = cmul(x[k], ht1[toff + (k - 1) * Q + j]);
                bf_dit<R, F1>(x);
            }
#pragma unroll
            for (int k = 0; k < R; ++k) cr.c1[kchunk<LOG, Q>(k)][sj ^ koff<LOG, Q>(k)] = x[k];
        }
    }
    cl.sync();
}

// The wraparound half-pointwise step (as half_pointwise_pair) over the half vector in chunks.
template <int MH, int NT, int C>
__device__ __noinline__ void cl_half_pointwise(const Chunks<C>& ch, const F2* __restrict__ ab2, const F1* __restrict__ ab1,
                                               const cgx::cluster_group& cl) {
    constexpr int H = 1 << MH, PAIRS = H / 2 + 1, PC = (PAIRS + C - 1) / C, LOG = MH - ilog2c(C);
    cl.sync();
    const int r = (int)cl.block_rank();
    const int t1 = min(PAIRS, (r + 1) * PC);
#pragma unroll 1
    for (int tau = r * PC + (int)threadIdx.x; tau < t1; tau += NT) {
        const int p = tau < 2 ? tau : tau - 1 + (1 << (31 - __clz(tau - 1)));
        const int q = p == 0 ? 0 : (3 << (31 - __clz(p))) - 1 - p;
        {
            F2& rp = ch.template e2<LOG>(p);
            F2& rq = ch.template e2<LOG>(q);
            const F2 zp = rp, zq = rq;
            const F2 e = lcfold(f2(zp.re + zq.re, zp.im + lsub<2>(0, zq.im)));
            const F2 d = lcfold(f2(lsub<2>(zp.re, zq.re), zp.im + zq.im));
            const F2 op = lcfold(lcadd(lkmulc(e, ab2[p]), lkmulc(d, ab2[H + p])));
            if (q != p) {
                const F2 e2v = lcfold(f2(zq.re + zp.re, zq.im + lsub<2>(0, zp.im)));
                const F2 d2 = lcfold(f2(lsub<2>(zq.re, zp.re), zq.im + zp.im));
                rq = lcfold(lcadd(lkmulc(e2v, ab2[q]), lkmulc(d2, ab2[H + q])));
            }
            rp = op;
        }
        {
            F1& rp = ch.template e1<LOG>(p);
            F1& rq = ch.template e1<LOG>(q);
            const F1 zp = rp, zq = rq;
            const F1 e = cadd(zp, cconj(zq)), d = csub(zp, cconj(zq));
            const F1 op = cadd(cmul(e, ab1[p]), cmul(d, ab1[H + p]));
            if (q != p) {
                const F1 e2v = cadd(zq, cconj(zp)), d2 = csub(zq, cconj(zp));
                rq = cadd(cmul(e2v, ab1[q]), cmul(d2, ab1[H + q]));
            }
            rp = op;
        }
    }
    cl.sync();
}

// ---- local passes of a transform on the CTA's own chunk ----
// Passes 1 .. P - 2 of the length-2^M weighted transform (DIF) or P - 2 .. 1 (DIT); each stays
// inside 8,192 elements for these lengths.
template <int M, int NT, bool FWD, int CL>
__device__ __forceinline__ void cl_local_full(F2* s2, F1* s1, const F2K* tab2, const F1* tab1) {
    constexpr int P = sched_passes(M);
    static_assert(sched_radix(M, 1) * sched_q(M, 1) <= (1 << CL), "only the first pass may cross chunks");
    if (FWD) {
#pragma unroll
        for (int i = 1; i < P - 1; ++i) {
            const int R = sched_radix(M, i);
            const F2K* t2 = tab2 + tab_fwd_off(M, i, true);
            const F1* t1 = tab1 + tab_fwd_off(M, i, true);
            if (R == 8) pass_rt<8, true, NT, true>(s2, s1, t2, t1, ilog2c(sched_q(M, i)), (1 << CL) / 8);
            else pass_rt<4, true, NT, true>(s2, s1, t2, t1, ilog2c(sched_q(M, i)), (1 << CL) / 4);
        }
    } else {
#pragma unroll
        for (int i = P - 2; i >= 1; --i) {
            const int R = sched_radix(M, i);
            const F2K* t2 = tab2 + tab_inv_off(M, i, true);
            const F1* t1 = tab1 + tab_inv_off(M, i, true);
            if (R == 8) pass_rt<8, false, NT, true>(s2, s1, t2, t1, ilog2c(sched_q(M, i)), (1 << CL) / 8);
            else pass_rt<4, false, NT, true>(s2, s1, t2, t1, ilog2c(sched_q(M, i)), (1 << CL) / 4);
        }
    }
}

// Passes 1 .. P - 1 (DIF) or P - 1 .. 1 (DIT) of the unweighted half-length transform on the
// CTA's chunk of 2^(CL - 1) elements.
template <int MH, int NT, bool FWD, int CL>
__device__ __forceinline__ void cl_local_half(F2* s2, F1* s1, const F2K* ht2, const F1* ht1) {
    constexpr int P = sched_passes(MH), HC = (1 << CL) / 2;
    static_assert(sched_radix(MH, 1) * sched_q(MH, 1) <= HC, "only the first half pass may cross chunks");
    if (FWD) {
#pragma unroll
        for (int i = 1; i < P; ++i) {
            const int R = sched_radix(MH, i), q = sched_q(MH, i);
            const F2K* t2 = ht2 + tab_fwd_off(MH, i, false);
            const F1* t1 = ht1 + tab_fwd_off(MH, i, false);
            if (R == 8) {
                if (q > 1) pass_rt<8, true, NT, true>(s2, s1, t2, t1, ilog2c(q), HC / 8);
                else pass_rt<8, true, NT, false>(s2, s1, t2, t1, 0, HC / 8);
            } else {
                pass_rt<4, true, NT, true>(s2, s1, t2, t1, ilog2c(q), HC / 4);
            }
        }
    } else {
#pragma unroll
        for (int i = P - 1; i >= 1; --i) {
            const int R = sched_radix(MH, i), q = sched_q(MH, i);
            const F2K* t2 = ht2 + tab_inv_off(MH, i, false);
            const F1* t1 = ht1 + tab_inv_off(MH, i, false);
            if (R == 8) {
                if (q > 1) pass_rt<8, false, NT, true>(s2, s1, t2, t1, ilog2c(q), HC / 8);
                else pass_rt<8, false, NT, false>(s2, s1, t2, t1, 0, HC / 8);
            } else {
                pass_rt<4, false, NT, true>(s2, s1, t2, t1, ilog2c(q), HC / 4);
            }
        }
    }
}

// ---- carries over the cluster ----
// T = c x^2 (2n limbs to `out`): CTA r owns coefficients [r 2n / C, (r + 1) 2n / C) of the
// chain, E = 2 n / (C NT) per thread; coefficient q < n is re of element q, q >= n im of q - n.
template <int M, int NT, int C>
__device__ __noinline__ uint64_t cl_carry_product(const Chunks<C>& ch, uint32_t* __restrict__ out, uint64_t* sc,
                                                  ClusterCarry* cc, const cgx::cluster_group& cl) {
    constexpr int N = 1 << M, CL = M - ilog2c(C), E = 2 * (1 << CL) / NT;
    const int q0 = (int)cl.block_rank() * (2 * N / C) + (int)threadIdx.x * E;
    const bool hi = q0 >= N;
    const int j0 = hi ? q0 - N : q0;
    // The run [j0, j0 + E) lies in one chunk (E divides the chunk length).
    const F2* b2 = ch.c2[j0 >> CL];
    const F1* b1 = ch.c1[j0 >> CL];
    const int sb = swz(j0 & ((1 << CL) - 1));
    uint32_t L[E];
    Acc96 acc;
#pragma unroll
    for (int e = 0; e < E; ++e) {
        const F2 a2 = b2[sb ^ swz_c(e)];
        const F1 a1 = b1[sb ^ swz_c(e)];
        uint32_t w0, w1, w2;
        crt3(hi ? a1.im : a1.re, hi ? a2.im : a2.re, w0, w1, w2);
        L[e] = acc.add_shift(w0, w1, w2);
    }
    const uint64_t top = cluster_resolve<E, NT, C>(L, acc.rest(), 0, sc, cc, cl);
#pragma unroll
    for (int e = 0; e < E; ++e) out[q0 + e] = L[e];
    return top;
}

// m = the low n limbs of the product (real parts), packed into the half vector as
// z_j = m_2j + i m_2j+1: CTA r owns coefficients [r n / C, (r + 1) n / C), all in its own
// chunk, and its packed elements are its own half-vector chunk.
template <int M, int NT, int C>
__device__ __noinline__ void cl_carry_low_and_pack(F2* s2, F1* s1, uint64_t* sc, ClusterCarry* cc,
                                                   const cgx::cluster_group& cl) {
    constexpr int E = (1 << (M - ilog2c(C))) / NT;
    const int l0 = (int)threadIdx.x * E;   // local coefficient index
    uint32_t L[E];
    Acc96 acc;
#pragma unroll
    for (int e = 0; e < E; ++e) {
        uint32_t w0, w1, w2;
        crt3(s1[(swz(l0) ^ swz_c(e))].re, s2[(swz(l0) ^ swz_c(e))].re, w0, w1, w2);
        L[e] = acc.add_shift(w0, w1, w2);
    }
    cluster_resolve<E, NT, C>(L, acc.rest(), 0, sc, cc, cl);   // the carry out of the top is dropped (mod R)
#pragma unroll
    for (int e = 0; e < E; e += 2) {
        const int sj = swz(l0 >> 1) ^ swz_c(e >> 1);   // (l0 + e) / 2, l0 / 2 a multiple of E / 2
        F2 z2; z2.re = L[e]; z2.im = L[e + 1];
        const uint32_t r0 = (L[e] & P1) + (L[e] >> 31), r1 = (L[e + 1] & P1) + (L[e + 1] >> 31);
        F1 z1; z1.re = min(r0, r0 - P1); z1.im = min(r1, r1 - P1);
        s2[sj] = z2;
        s1[sj] = z1;
    }
    cl.sync();
}

// x = floor(T / R) + ((cyclic + T mod R) mod (R - 1)) as wrap_combine: CTA r owns limbs
// [r n / C, (r + 1) n / C), the cyclic product's coefficients packed in its half chunk.
template <int M, int NT, int C>
__device__ __noinline__ bool cl_wrap_combine(const F2* s2, const F1* s1, const uint32_t* __restrict__ tl,
                                             uint32_t* __restrict__ x, uint64_t* sc, ClusterCarry* cc,
                                             const cgx::cluster_group& cl) {
    constexpr int K = 1 << M, CL = M - ilog2c(C), E = (1 << CL) / NT;
    const int l0 = (int)threadIdx.x * E;
    const int q0 = (int)cl.block_rank() * (1 << CL) + l0;
    uint32_t L[E];
    Acc96 acc;
#pragma unroll
    for (int e = 0; e < E; e += 2) {
        const int sj = swz(l0 >> 1) ^ swz_c(e >> 1);   // (l0 + e) / 2, l0 / 2 a multiple of E / 2
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
    uint64_t top = cluster_resolve<E, NT, C>(L, acc.rest(), 0, sc, cc, cl);
    // End-around carry: 2^(32 k) = 1 mod R - 1; `top` is the same on every CTA.
    while (top != 0) top = cluster_resolve<E, NT, C>(L, 0, top, sc, cc, cl);
    uint64_t a2 = 0;
#pragma unroll
    for (int e = 0; e < E; ++e) {
        a2 += (uint64_t)L[e] + tl[K + q0 + e];
        L[e] = (uint32_t)a2;
        a2 >>= 32;
    }
    top = cluster_resolve<E, NT, C>(L, a2, 0, sc, cc, cl);
#pragma unroll
    for (int e = 0; e < E; ++e) x[q0 + e] = L[e];
    return top == 0;
}

// ---- the step ----
// Up to `bits` steps x <- x^2 c^bit R^-1 on one slot, the cluster's CTAs together (as step_slot,
// wraparound path). Every CTA runs the same steps; CTA 0 writes pos and the error word.
template <int M, int NT, int C>
__device__ __forceinline__ void cl_step_slot(const SlotArgs& a, uint32_t slot, uint32_t bits, unsigned char* smem_raw,
                                             uint64_t* sc, ClusterCarry* cc) {
    constexpr int N = 1 << M, MH = M - 1, CL = M - ilog2c(C), CH = 1 << CL;
    static_assert(CH * C == N, "C chunks of 2^CL elements hold the vector");
    const cgx::cluster_group cl = cgx::this_cluster();
    F2* s2 = reinterpret_cast<F2*>(smem_raw);
    F1* s1 = reinterpret_cast<F1*>(smem_raw + 16 * CH);
    Chunks<C> ch;
#pragma unroll
    for (int d = 0; d < C; ++d) {
        ch.c2[d] = cl.map_shared_rank(s2, d);
        ch.c1[d] = cl.map_shared_rank(s1, d);
    }
    const int r = (int)cl.block_rank();
    uint32_t* x = a.x + (size_t)slot * N;
    uint32_t* tl = a.tbuf + (size_t)slot * 2 * N;
    const F2* cc2 = a.c2 + (size_t)slot * 2 * N;
    const F1* cc1 = a.c1 + (size_t)slot * 2 * N;
    const uint32_t* ex = a.exp + (size_t)slot * a.ew;
    const F2K* ht2 = a.tab2 + lt_half_off(M);
    const F1* ht1 = a.tab1 + lt_half_off(M);
    const uint32_t nb = a.nbits[slot];
    uint32_t pos = a.pos[slot];
    const int gbase = r * (CH / 8);   // this CTA's first group of the span-1 pass
    bool ok = true;
    for (uint32_t it = 0; it < bits && pos < nb; ++it, ++pos) {
        const uint32_t bit = (ex[pos >> 5] >> (31 - (pos & 31))) & 1;
        const uint32_t c = bit ? a.base : 1;
        // T = c x^2
        cl_dif_first<M, NT, C>(x, N, ch, a.tab2, a.tab1, cl);
        cl_local_full<M, NT, true, CL>(s2, s1, a.tab2, a.tab1);
        fused_mid<CL, NT, false>(nullptr, 0, s2, s1, a.tab2, a.tab1, TileOp<SquareOp>{SquareOp{c}, gbase});
        cl_local_full<M, NT, false, CL>(s2, s1, a.tab2, a.tab1);
        cl_dit_last<M, NT, C, false>(ch, a.tab2, a.tab1, cl);
        ok &= cl_carry_product<M, NT, C>(ch, tl, sc, cc, cl) == 0;
        if (a.bare) continue;
        // m = (T mod R) N' mod R
        cl_dif_first<M, NT, C>(tl, N, ch, a.tab2, a.tab1, cl);
        cl_local_full<M, NT, true, CL>(s2, s1, a.tab2, a.tab1);
        fused_mid<CL, NT, true>(nullptr, 0, s2, s1, a.tab2, a.tab1,
                                       TileOp<SpecMulRT>{SpecMulRT{cc2, cc1, N / 8}, gbase});
        cl_local_full<M, NT, false, CL>(s2, s1, a.tab2, a.tab1);
        cl_dit_last<M, NT, C, true>(ch, a.tab2, a.tab1, cl);
        cl_carry_low_and_pack<M, NT, C>(s2, s1, sc, cc, cl);
        // m N mod (R - 1) through the half-length transform of the packed limbs
        cl_half_pass0<MH, true, NT, C>(ch, ht2, ht1, cl);
        cl_local_half<MH, NT, true, CL>(s2, s1, ht2, ht1);
        cl_half_pointwise<MH, NT, C>(ch, cc2 + N, cc1 + N, cl);
        cl_local_half<MH, NT, false, CL>(s2, s1, ht2, ht1);
        cl_half_pass0<MH, false, NT, C>(ch, ht2, ht1, cl);
        ok &= cl_wrap_combine<M, NT, C>(s2, s1, tl, x, sc, cc, cl);
    }
    cl.sync();   // every thread of every CTA has read pos before it is written
    if (r == 0 && threadIdx.x == 0) {
        a.pos[slot] = pos;
        if (!ok) a.err[slot] = 1;
    }
}

// The uniform cluster launch: cluster i (C = 2^(M - CL) consecutive blocks of 2^CL elements)
// steps slot first + i. CL = 13: one block of 192 KiB per SM; CL = 12 (L = 32768 only): two
// blocks of 96 KiB per SM, so twice the warps hide the latency of the cross-block accesses, at
// 64 registers per thread and with more of each cross-block pass remote.
template <int M, int CL>
__global__ void __launch_bounds__(kClusterThreads, kChunkLog - CL + 1)
    cluster_step_kernel(SlotArgs a, uint32_t first, uint32_t bits) {
    constexpr int C = 1 << (M - CL);
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ uint64_t sc[CarryScratch<kClusterThreads>::words];
    __shared__ ClusterCarry cc;
    cl_step_slot<M, kClusterThreads, C>(a, first + blockIdx.x / C, bits, smem_raw, sc, &cc);
}

// ---- host side: launch and shared-memory opt-in of one instantiation ----
template <int M, int CL>
cudaError_t launch_cluster_m(const SlotArgs& a, uint32_t slots, uint32_t bits, cudaStream_t s) {
    constexpr int C = 1 << (M - CL);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(C * slots, 1, 1);
    cfg.blockDim = dim3(kClusterThreads, 1, 1);
    cfg.dynamicSmemBytes = 24 << CL;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = C;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, cluster_step_kernel<M, CL>, a, 0u, bits);
}

template <int M, int CL>
cudaError_t configure_cluster_m() {
    return cudaFuncSetAttribute((const void*)cluster_step_kernel<M, CL>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                24 << CL);
}

// The 4,096-element-chunk instantiation at L = 32768 (mm_cluster_half.cu).
cudaError_t cluster_half_chunk_configure();
cudaError_t cluster_half_chunk_launch(const SlotArgs& a, uint32_t slots, uint32_t bits, cudaStream_t s);

}  // namespace mm
