// Shared host/device definitions of the B200 MontMul backend: field constants, element types,
// the per-length transform schedule (radix of every pass) and the layout of the twiddle tables.
//
// The transform is the reference's right-angle NTT over GF(M31^2) x GF(M61^2)
// (montmul/src/field.rs, cpu.rs:49-115): a length-n complex DIF (natural order in, bit-reversed
// order out) and DIT (bit-reversed in, natural out), n = L/2. Here it runs as radix-8/4/2
// passes; a radix-R pass is exactly R' = log2 R consecutive radix-2 stages of the reference,
// so every spectrum position holds the same value as in the reference.
#pragma once
#include <stdint.h>

#if defined(__CUDACC__)
#define MM_HD __host__ __device__ __forceinline__
#else
#define MM_HD inline
#ifndef __align__
#define __align__(n) __attribute__((aligned(n)))   // host-only builds of this header
#endif
#endif

namespace mm {

constexpr uint32_t P1 = 0x7fffffffu;             // M31
constexpr uint64_t P2 = 0x1fffffffffffffffull;   // M61

struct __align__(8) F1 { uint32_t re, im; };
struct __align__(16) F2 { uint64_t re, im; };
// A GF(M61^2) twiddle in the form the Karatsuba product reads: re, im, re + im, im - re (mod p).
struct __align__(16) F2K { uint64_t re, im, s, d; };

// Largest transform length handled with the whole vector in shared memory: n = 8192
// (L = 16384) needs 24 n = 196,608 B of the 227 KB a B200 block may opt into.
constexpr int kMaxSharedLogN = 13;
constexpr int kMinLogN = 2;   // L = 8

// Dynamic shared memory of one block at length 2^(m+1): F2 vector (16 n B), F1 vector (8 n B).
MM_HD constexpr int smem_bytes_host(int m) { return 24 << m; }

// Position of element e in shared memory (and in global mode's work vectors): e with its low
// four bits flipped by a linear function of bits 3-8,
//   bit 0 ^= e3 ^ e6 ^ e8,  bit 1 ^= e4 ^ e6 ^ e7,  bit 2 ^= e5,  bit 3 ^= e4 ^ e5 ^ e6.
// Chosen by simulating every shared-memory access pattern of the kernels (each radix-8 and
// radix-4 pass of both transforms at every span; the carries' runs of 2 to 32 consecutive
// elements per thread and their pair-packed reads and writes; 16-B F2 and 8-B F1 accesses; 32 to
// 1,024 threads per slot): every warp access of n >= 64 elements takes the minimum number of
// wavefronts (tests/test_swizzle.py). Flipping the low bits by bits 3-6 alone left the carries'
// runs of 16 and 32 elements 2- and 4-way conflicted. swz is linear over XOR,
// swz(a ^ b) = swz(a) ^ swz(b), and permutes each aligned run of 16 elements.
MM_HD constexpr int swz_c(int e) {
    const int h = e >> 3, u = (h >> 3) & 7;   // h: bits 3.., u: bits 6-8
    const int lo = (h ^ ((u ^ (u << 1) ^ (u >> 2)) & 3)) & 7;
    const int b3 = ((h >> 1) ^ (h >> 2) ^ (h >> 3)) & 1;
    return e ^ lo ^ (b3 << 3);
}

// ---- pass schedule: radices, DIF order ----
// m = log2 n. m = 3a -> [8]*a; m = 3a + 1 -> [4, 4, 8*(a-1)]; m = 3a + 2 -> [4, 8*a];
// m = 1 -> [2], m = 2 -> [4]. Radix-8 passes dominate; the last DIF pass (span 1) carries no
// twiddles, so it is kept at radix 8 whenever m >= 3.
MM_HD constexpr int sched_passes(int m) {
    return m <= 3 ? 1 : (m % 3 == 0 ? m / 3 : (m % 3 == 1 ? m / 3 + 1 : m / 3 + 1));
}
MM_HD constexpr int sched_radix(int m, int i) {
    return m == 1 ? 2 : m == 2 ? 4 : m == 3 ? 8
         : (m % 3 == 0 ? 8 : (m % 3 == 1 ? (i < 2 ? 4 : 8) : (i < 1 ? 4 : 8)));
}
MM_HD constexpr int ilog2c(int v) { return v <= 1 ? 0 : 1 + ilog2c(v / 2); }
// Span q of the last radix-2 stage of DIF pass i (also the first span of the DIT pass i).
MM_HD constexpr int sched_q(int m, int i) {
    int lq = m;
    for (int p = 0; p <= i; ++p) lq -= ilog2c(sched_radix(m, p));
    return 1 << lq;
}

// ---- twiddle table layout for one transform (m, weighted) ----
// Elements (F1 and F2 arrays use the same indices):
//   forward pass i with q_i > 1:  weighted pass 0: R*q entries [k][j] = zeta^j W^(j rev_R(k));
//                                 other passes:    (R-1)*q entries [k-1][j] = W^(j rev_R(k)).
//   inverse pass i with q_i > 1:  same shapes with V = W^-1 (and zeta^-j for weighted pass 0).
//   weighted transforms then hold R_0 input constants zeta^(q_0 k) and R_0 output constants
//   zeta^(-q_0 k) / n.
// W is the primitive (R q)-th root omega_n^(n/(R q)) of the reference's tables (field.rs:243).
MM_HD constexpr int tab_pass_size(int m, int i, bool weighted) {
    int R = sched_radix(m, i), q = sched_q(m, i);
    return q <= 1 ? 0 : (weighted && i == 0 ? R * q : (R - 1) * q);
}
MM_HD constexpr int tab_fwd_off(int m, int i, bool weighted) {
    int o = 0;
    for (int p = 0; p < i; ++p) o += tab_pass_size(m, p, weighted);
    return o;
}
MM_HD constexpr int tab_fwd_size(int m, bool weighted) { return tab_fwd_off(m, sched_passes(m), weighted); }
MM_HD constexpr int tab_inv_off(int m, int i, bool weighted) {
    return tab_fwd_size(m, weighted) + tab_fwd_off(m, i, weighted);
}
MM_HD constexpr int tab_in_const_off(int m, bool weighted) { return 2 * tab_fwd_size(m, weighted); }
MM_HD constexpr int tab_out_const_off(int m, bool weighted) {
    return tab_in_const_off(m, weighted) + (weighted ? sched_radix(m, 0) : 0);
}
MM_HD constexpr int tab_size(int m, bool weighted) {
    return tab_out_const_off(m, weighted) + (weighted ? sched_radix(m, 0) : 0);
}

// Tables of one transform length L = 2^(m+1): the weighted length-n transform (m = log2 n)
// followed by the unweighted length-h transform of the wraparound path (h = n/2), then the
// wraparound set-up tables u[p] = w^rev(p), iu[p] = w^-rev(p) over h positions (cpu.rs:165-179).
MM_HD constexpr int lt_full_off(int) { return 0; }
MM_HD constexpr int lt_half_off(int m) { return tab_size(m, true); }
MM_HD constexpr int lt_unpack_off(int m) { return lt_half_off(m) + (m >= 2 ? tab_size(m - 1, false) : 0); }
MM_HD constexpr int lt_size(int m) { return lt_unpack_off(m) + 2 * (1 << (m - 1)); }

// Per-slot constants in the order the fused pointwise step reads them: the spectrum position
// p = R*g + k of the last DIF pass (radix R = sched_radix(m, last)) is stored at k*(n/R) + g,
// so the R loads of one group are coalesced across a warp. n elements hold N^' = F(N'); the
// next n hold the wraparound factors A (positions p < h) and B (h + p), in natural position
// order (cpu.rs:265-284).
MM_HD constexpr int const_index(int m, int p) {
    int R = sched_radix(m, sched_passes(m) - 1);
    int n = 1 << m;
    return (p % R) * (n / R) + p / R;
}

}  // namespace mm

namespace mm {

// ---- global mode: the vector in HBM, transformed through shared-memory tiles ----
// Lengths n = 2^m > kMaxSharedLogN. DIF stages whose span reaches a tile (2^kTileLog elements)
// run as passes over global memory; the remaining kTileLog stages are, on every tile, exactly a
// complete length-2^kTileLog transform (the twiddles of a stage depend only on its span), so the
// tiles reuse one unweighted length-2^kTileLog table. DIT mirrors this.
constexpr int kTileLog = 11;                  // 2,048-element tiles (48 KiB of F2 + F1)
constexpr int kMaxGlobalLogN = 23;            // L = 2^24, the reference's largest length

// Global passes of a length-2^m transform: the schedule of its G = m - kTileLog global stages.
MM_HD int gl_stages(int m) { return m - kTileLog; }
MM_HD int gl_passes(int m) { return sched_passes(gl_stages(m)); }
MM_HD int gl_radix(int m, int i) { return sched_radix(gl_stages(m), i); }
MM_HD int gl_lq(int m, int i) {
    int lq = m;
    for (int p = 0; p <= i; ++p) lq -= ilog2c(gl_radix(m, p));
    return lq;
}
MM_HD int gl_pass_size(int m, int i, bool weighted) {
    const int R = gl_radix(m, i), q = 1 << gl_lq(m, i);
    return weighted && i == 0 ? R * q : (R - 1) * q;
}
MM_HD int gl_fwd_off(int m, int i, bool weighted) {
    int o = 0;
    for (int p = 0; p < i; ++p) o += gl_pass_size(m, p, weighted);
    return o;
}
MM_HD int gl_fwd_size(int m, bool weighted) { return gl_fwd_off(m, gl_passes(m), weighted); }
MM_HD int gl_inv_off(int m, int i, bool weighted) { return gl_fwd_size(m, weighted) + gl_fwd_off(m, i, weighted); }
MM_HD int gl_in_const_off(int m, bool weighted) { return 2 * gl_fwd_size(m, weighted); }
MM_HD int gl_out_const_off(int m, bool weighted) { return gl_in_const_off(m, weighted) + (weighted ? gl_radix(m, 0) : 0); }
MM_HD int gl_tab_size(int m, bool weighted) { return gl_out_const_off(m, weighted) + (weighted ? gl_radix(m, 0) : 0); }

// Tables of global-mode length L = 2^(m+1): the weighted full transform's global passes, the
// tile transform (unweighted, length 2^kTileLog), the half transform's global passes (or none
// when the half length fits one tile), then the wraparound unpack roots over h positions.
MM_HD int glt_tile_off(int m) { return gl_tab_size(m, true); }
MM_HD int glt_half_off(int m) { return glt_tile_off(m) + tab_size(kTileLog, false); }
MM_HD int glt_unpack_off(int m) { return glt_half_off(m) + (m - 1 > kTileLog ? gl_tab_size(m - 1, false) : 0); }
MM_HD int glt_size(int m) { return glt_unpack_off(m) + 2 * (1 << (m - 1)); }

}  // namespace mm
