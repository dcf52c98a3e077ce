// Global mode: lengths n = 2^m, kMaxSharedLogN < m <= kMaxGlobalLogN, one thread block per slot
// with the slot's vector in HBM (a per-slot work buffer, F2 then F1, element e at swz(e) as in
// shared memory). The reference runs these lengths with its global-memory kernels and 2,048-
// element shared tiles (kernels/src/lib.rs:455-511); here:
//   - DIF stages whose span reaches a tile run as passes straight over global memory (the same
//     runtime-span pass functions as shared mode, on global pointers; warps read consecutive j,
//     so every access is coalesced);
//   - the remaining kTileLog stages are, on each tile, a complete length-2^kTileLog transform;
//     tiles stream through shared memory with 1-D bulk copies (cp.async.bulk, no multicast),
//     double-buffered: while one tile is transformed the next is loading and the previous is
//     storing. The pointwise operation runs inside the tile, between its last DIF and first
//     DIT pass, so the middle of a step costs one read and one write of the vector;
//   - carries run in chunks of 16 coefficients per thread.
// Every wait on a bulk copy is bounded; a wait that runs out sets the slot's error word to 2.
#pragma once
#include "mm_abi.h"
#include "mm_kernels.cuh"

namespace mm {

constexpr int kTile = 1 << kTileLog;
constexpr int kTileBytes2 = 16 * kTile, kTileBytes1 = 8 * kTile;
constexpr int kGlobalSmem = 2 * (kTileBytes2 + kTileBytes1);   // two tile buffers: 96 KiB
constexpr int kChunkE = 16;                                    // coefficients per thread per carry chunk
constexpr int kErrTimeout = 2;
constexpr uint64_t kWaitLimitNs = 100000000ull;                // bound of every wait on a bulk copy

// ---- bulk copies and mbarriers (PTX) ----
__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bar)) : "memory");
}
__device__ __forceinline__ void mbar_expect(uint64_t* bar, uint32_t bytes) {
    asm volatile("{ .reg .b64 st; mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1; }" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}
// Waits for phase `parity` of the barrier; gives up after about `limit_ns` of global time
// (checked every 256 polls) or 2^26 polls, whichever comes first.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint64_t limit_ns = kWaitLimitNs) {
    const uint32_t a = smem_addr(bar);
    uint64_t t0;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
    for (uint32_t it = 0; it < (1u << 26); ++it) {
        uint32_t done;
        asm volatile("{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
                     : "=r"(done)
                     : "r"(a), "r"(parity)
                     : "memory");
        if (done) return true;
        if ((it & 255) == 255) {
            uint64_t t;
            asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
            if (t - t0 > limit_ns) return false;
        }
    }
    return false;
}
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}
__device__ __forceinline__ void bulk_store(void* dst, const void* src, uint32_t bytes) {
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst), "r"(smem_addr(src)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_read() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }
// Orders this thread's generic-proxy accesses of global (or shared) memory before later
// async-proxy (bulk copy) accesses, and the async proxy's completed writes before later reads.
__device__ __forceinline__ void fence_async_global() { asm volatile("fence.proxy.async.global;" ::: "memory"); }
__device__ __forceinline__ void fence_async_shared() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// ---- pointwise operations with a runtime length (index k (n/8) + g of the last radix-8 pass) ----
struct SpecMulRT {
    const F2* b2; const F1* b1; int nr;   // nr = n / 8
    template <int R> __device__ __forceinline__ bool apply2(F2* x, int g) const {
#pragma unroll
        for (int k = 0; k < R; ++k) x[k] = lkmulc(x[k], b2[k * nr + g]);
        return false;
    }
    template <int R> __device__ __forceinline__ bool apply1(F1* x, int g) const {
#pragma unroll
        for (int k = 0; k < R; ++k) x[k] = cmul(x[k], b1[k * nr + g]);
        return false;
    }
};
struct SpecStoreRT {
    F2* b2; F1* b1; int nr;
    template <int R> __device__ __forceinline__ bool apply2(F2* x, int g) const {
#pragma unroll
        for (int k = 0; k < R; ++k) b2[k * nr + g] = lccanon(x[k]);
        return true;
    }
    template <int R> __device__ __forceinline__ bool apply1(F1* x, int g) const {
#pragma unroll
        for (int k = 0; k < R; ++k) b1[k * nr + g] = x[k];
        return true;
    }
};
// Shifts a tile-local group index to the global one.
template <class OP> struct TileOp {
    OP op; int gbase;
    template <int R> __device__ __forceinline__ bool apply2(F2* x, int g) const { return op.template apply2<R>(x, gbase + g); }
    template <int R> __device__ __forceinline__ bool apply1(F1* x, int g) const { return op.template apply1<R>(x, gbase + g); }
};

// ---- global passes with a runtime radix ----
template <int NT>
__device__ __forceinline__ void g_pass(int R, bool fwd, F2* v2, F1* v1, const F2K* t2, const F1* t1, int lq, int n) {
    if (R == 8) {
        if (fwd) pass_rt<8, true, NT, true>(v2, v1, t2, t1, lq, n / 8);
        else pass_rt<8, false, NT, true>(v2, v1, t2, t1, lq, n / 8);
    } else if (R == 4) {
        if (fwd) pass_rt<4, true, NT, true>(v2, v1, t2, t1, lq, n / 4);
        else pass_rt<4, false, NT, true>(v2, v1, t2, t1, lq, n / 4);
    } else {
        if (fwd) pass_rt<2, true, NT, true>(v2, v1, t2, t1, lq, n / 2);
        else pass_rt<2, false, NT, true>(v2, v1, t2, t1, lq, n / 2);
    }
}

// Weighted first global pass from real limbs (runtime span), as dif_first_from_limbs.
template <int R, int NT>
__device__ __noinline__ void g_dif_first(const uint32_t* __restrict__ lim, int cnt, F2* v2, F1* v1, const F2K* t2,
                                         const F1* t1, const F2K* cin2, const F1* cin1, int lq) {
    const int q = 1 << lq;
#pragma unroll 1
    for (int j = gtid<NT>(); j < q; j += NT) {
        uint32_t v[R];
#pragma unroll
        for (int k = 0; k < R; ++k) v[k] = (j + k * q < cnt) ? lim[j + k * q] : 0u;
        {
            F2 x[R];
#pragma unroll
            for (int k = 0; k < R; ++k) x[k] = lreal_times(v[k], cin2[k]);
            ldif<R>(x);
#pragma unroll
            for (int k = 0; k < R; ++k) v2[swz(j + k * q)] = lkmul(lcfold(x[k]), t2[k * q + j]);
        }
        {
            F1 x[R];
#pragma unroll
            for (int k = 0; k < R; ++k) x[k] = real_times<F1>(v[k], cin1[k]);
            bf_dif<R, F1>(x);
#pragma unroll
            for (int k = 0; k < R; ++k) v1[swz(j + k * q)] = cmul(x[k], t1[k * q + j]);
        }
    }
    gsync<NT>();
}

// Weighted last global DIT pass into natural order (runtime span), as dit_last_weighted.
template <int R, int NT, bool REAL_ONLY>
__device__ __noinline__ void g_dit_last(F2* v2, F1* v1, const F2K* t2, const F1* t1, const F2K* cout2,
                                        const F1* cout1, int lq) {
    const int q = 1 << lq;
#pragma unroll 1
    for (int j = gtid<NT>(); j < q; j += NT) {
        {
            F2 x[R];
#pragma unroll
            for (int k = 0; k < R; ++k) x[k] = lkmul(v2[swz(j + k * q)], t2[k * q + j]);
            ldit<R>(x);
#pragma unroll
            for (int k = 0; k < R; ++k) {
                if (REAL_ONLY) v2[swz(j + k * q)].re = lkmul_re(x[k], cout2[k]);
                else v2[swz(j + k * q)] = lkmul(x[k], cout2[k]);
            }
        }
        {
            F1 x[R];
#pragma unroll
            for (int k = 0; k < R; ++k) x[k] = cmul(v1[swz(j + k * q)], t1[k * q + j]);
            bf_dit<R, F1>(x);
#pragma unroll
            for (int k = 0; k < R; ++k) {
                if (REAL_ONLY) v1[swz(j + k * q)].re = cmul_re(x[k], cout1[k]);
                else v1[swz(j + k * q)] = cmul(x[k], cout1[k]);
            }
        }
    }
    gsync<NT>();
}

// Weighted first global pass of complex elements in place (the Transform trait's forward, as
// dif_first_complex).
template <int R, int NT>
__device__ __noinline__ void g_dif_first_complex(F2* v2, F1* v1, const F2K* t2, const F1* t1, const F2K* cin2,
                                                 const F1* cin1, int lq) {
    const int q = 1 << lq;
#pragma unroll 1
    for (int j = gtid<NT>(); j < q; j += NT) {
        {
            F2 x[R];
#pragma unroll
            for (int k = 0; k < R; ++k) x[k] = lkmul(v2[swz(j + k * q)], cin2[k]);
            ldif<R>(x);
#pragma unroll
            for (int k = 0; k < R; ++k) v2[swz(j + k * q)] = lkmul(lcfold(x[k]), t2[k * q + j]);
        }
        {
            F1 x[R];
#pragma unroll
            for (int k = 0; k < R; ++k) x[k] = cmul(v1[swz(j + k * q)], cin1[k]);
            bf_dif<R, F1>(x);
#pragma unroll
            for (int k = 0; k < R; ++k) v1[swz(j + k * q)] = cmul(x[k], t1[k * q + j]);
        }
    }
    gsync<NT>();
}

template <int NT>
__device__ __forceinline__ void g_dif_first_rt(int R, const uint32_t* lim, int cnt, F2* v2, F1* v1, const F2K* t2,
                                               const F1* t1, const F2K* c2, const F1* c1, int lq) {
    if (R == 8) g_dif_first<8, NT>(lim, cnt, v2, v1, t2, t1, c2, c1, lq);
    else if (R == 4) g_dif_first<4, NT>(lim, cnt, v2, v1, t2, t1, c2, c1, lq);
    else g_dif_first<2, NT>(lim, cnt, v2, v1, t2, t1, c2, c1, lq);
}
template <int NT, bool REAL_ONLY>
__device__ __forceinline__ void g_dit_last_rt(int R, F2* v2, F1* v1, const F2K* t2, const F1* t1, const F2K* c2,
                                              const F1* c1, int lq) {
    if (R == 8) g_dit_last<8, NT, REAL_ONLY>(v2, v1, t2, t1, c2, c1, lq);
    else if (R == 4) g_dit_last<4, NT, REAL_ONLY>(v2, v1, t2, t1, c2, c1, lq);
    else g_dit_last<2, NT, REAL_ONLY>(v2, v1, t2, t1, c2, c1, lq);
}

// Global passes of a length-2^m transform: DIF from real limbs (weighted) or of the vector
// already in place (unweighted), and DIT down to natural order.
template <int NT>
__device__ __forceinline__ void g_fwd(int m, bool weighted, const uint32_t* lim, F2* v2, F1* v1, const F2K* tab2,
                                      const F1* tab1, int cnt = 0) {
    const int P = gl_passes(m), n = 1 << m;
    int i = 0;
    if (weighted) {
        g_dif_first_rt<NT>(gl_radix(m, 0), lim, cnt ? cnt : n, v2, v1, tab2 + gl_fwd_off(m, 0, true), tab1 + gl_fwd_off(m, 0, true),
                           tab2 + gl_in_const_off(m, true), tab1 + gl_in_const_off(m, true), gl_lq(m, 0));
        i = 1;
    }
    for (; i < P; ++i)
        g_pass<NT>(gl_radix(m, i), true, v2, v1, tab2 + gl_fwd_off(m, i, weighted), tab1 + gl_fwd_off(m, i, weighted),
                   gl_lq(m, i), n);
}
template <int NT, bool REAL_ONLY>
__device__ __forceinline__ void g_inv(int m, bool weighted, F2* v2, F1* v1, const F2K* tab2, const F1* tab1) {
    const int P = gl_passes(m), n = 1 << m;
    for (int i = P - 1; i >= (weighted ? 1 : 0); --i)
        g_pass<NT>(gl_radix(m, i), false, v2, v1, tab2 + gl_inv_off(m, i, weighted), tab1 + gl_inv_off(m, i, weighted),
                   gl_lq(m, i), n);
    if (weighted)
        g_dit_last_rt<NT, REAL_ONLY>(gl_radix(m, 0), v2, v1, tab2 + gl_inv_off(m, 0, true), tab1 + gl_inv_off(m, 0, true),
                                     tab2 + gl_out_const_off(m, true), tab1 + gl_out_const_off(m, true), gl_lq(m, 0));
}

// ---- the tile phase ----
enum { kTileFull = 0, kTileDif = 1, kTileDit = 2, kTileDifOp = 3 };

struct TileSmem {
    unsigned char* base;   // two buffers of kTileBytes2 + kTileBytes1
    uint64_t* bar;         // one mbarrier per buffer
    __device__ F2* b2(int b) const { return reinterpret_cast<F2*>(base + b * (kTileBytes2 + kTileBytes1)); }
    __device__ F1* b1(int b) const { return reinterpret_cast<F1*>(base + b * (kTileBytes2 + kTileBytes1) + kTileBytes2); }
};

// Once per kernel, all threads of the group.
template <int NT>
__device__ __forceinline__ void tile_init(const TileSmem& sm) {
    if (gtid<NT>() == 0) {
        mbar_init(&sm.bar[0]);
        mbar_init(&sm.bar[1]);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    gsync<NT>();
}

// The mbarrier phases: bit b of `par` is the parity of the next phase of barrier b. Tile c uses
// barrier c & 1, so a phase over t tiles completes ceil(t/2) phases of barrier 0 and floor(t/2)
// of barrier 1.
__device__ __forceinline__ uint32_t tile_par_next(uint32_t par, int n) {
    const int tiles = n >> kTileLog;
    return par ^ (((tiles + 1) >> 1) & 1) ^ (((tiles >> 1) & 1) << 1);
}

// Runs the tile part of a transform on every tile of the n-element vector (v2, v1) in global
// memory: full (DIF, op, DIT), DIF only, DIT only, or DIF then op (the op consumes the
// spectrum: nothing is stored back). Returns false, the same on every thread, when a bulk copy
// did not complete in time. It then gives the loads of tiles c and c + 1 one more bounded wait
// before returning, so a late copy normally lands before the block moves on; if that wait also
// runs out (a copy stalled for over 200 ms, which no healthy GPU does), the block returns with
// the load possibly still pending, the slot's error word reports the time-out, and the caller
// must treat the batch's results as lost.
template <int NT, class OP>
__device__ __noinline__ bool tile_phase(F2* v2, F1* v1, int n, const F2K* tt2, const F1* tt1, const OP& op, int mode,
                                        const TileSmem& sm, uint32_t par) {
    const int tiles = n >> kTileLog;
    const bool store = mode != kTileDifOp;
    constexpr uint32_t kBytes = kTileBytes2 + kTileBytes1;
    // This thread's generic writes of the vector (earlier passes) before the bulk loads read it,
    // and its generic accesses of the tile buffers (a shared-mode item of the mixed launch may
    // have used them) before the bulk loads overwrite them.
    fence_async_global();
    fence_async_shared();
    gsync<NT>();
    if (gtid<NT>() == 0) {
        mbar_expect(&sm.bar[0], kBytes);
        bulk_load(sm.b2(0), v2, kTileBytes2, &sm.bar[0]);
        bulk_load(sm.b1(0), v1, kTileBytes1, &sm.bar[0]);
    }
    bool ok = true;
#pragma unroll 1
    for (int c = 0; c < tiles; ++c) {
        const int b = c & 1;
        const uint32_t ph = ((par >> b) ^ (uint32_t)(c >> 1)) & 1;
        if (gtid<NT>() == 0 && c + 1 < tiles) {
            // The other buffer's store (tile c - 1) must have read its data out first.
            bulk_wait_read();
            mbar_expect(&sm.bar[b ^ 1], kBytes);
            bulk_load(sm.b2(b ^ 1), v2 + ((size_t)(c + 1) << kTileLog), kTileBytes2, &sm.bar[b ^ 1]);
            bulk_load(sm.b1(b ^ 1), v1 + ((size_t)(c + 1) << kTileLog), kTileBytes1, &sm.bar[b ^ 1]);
        }
        const bool got = mbar_wait(&sm.bar[b], ph);
        if (gsync_or<NT>(!got)) {
            // Give the copies of tiles c and c + 1 one more bounded wait before leaving.
            if (gtid<NT>() == 0) {
                mbar_wait(&sm.bar[b], ph);
                if (c + 1 < tiles) mbar_wait(&sm.bar[b ^ 1], ((par >> (b ^ 1)) ^ (uint32_t)((c + 1) >> 1)) & 1);
            }
            ok = false;
            break;
        }
        F2* s2 = sm.b2(b);
        F1* s1 = sm.b1(b);
        const TileOp<OP> top{op, c * (kTile / 8)};
        if (mode == kTileFull || mode == kTileDifOp) {
            smem_pass<kTileLog, 0, true, NT, false>(s2, s1, tt2, tt1);
            smem_pass<kTileLog, 1, true, NT, false>(s2, s1, tt2, tt1);
            smem_pass<kTileLog, 2, true, NT, false>(s2, s1, tt2, tt1);
            fused_mid<kTileLog, NT, false>(nullptr, 0, s2, s1, tt2, tt1, top);
            if (mode == kTileFull) {
                smem_pass<kTileLog, 2, false, NT, false>(s2, s1, tt2, tt1);
                smem_pass<kTileLog, 1, false, NT, false>(s2, s1, tt2, tt1);
                smem_pass<kTileLog, 0, false, NT, false>(s2, s1, tt2, tt1);
            }
        } else if (mode == kTileDif) {
            dif_unweighted<kTileLog, NT>(s2, s1, tt2, tt1);
        } else {
            dit_unweighted<kTileLog, NT>(s2, s1, tt2, tt1);
        }
        // Generic accesses of this buffer before the async proxy reads (store) or rewrites
        // (the load of tile c + 2) it.
        fence_async_shared();
        gsync<NT>();
        if (store && gtid<NT>() == 0) {
            bulk_store(v2 + ((size_t)c << kTileLog), s2, kTileBytes2);
            bulk_store(v1 + ((size_t)c << kTileLog), s1, kTileBytes1);
            bulk_commit();
        }
    }
    if (gtid<NT>() == 0) {
        bulk_wait_all();
        fence_async_global();
    }
    gsync<NT>();
    return ok;
}

// ---- chunked carries over global vectors ----
// Sums coefficient(q) (three 32-bit words, < 2^93) over q < count into out[q], 16 per thread per
// chunk, the carry of each chunk entering the next; returns the carry out of the top.
template <int NT, class COEF>
__device__ __forceinline__ uint64_t chunked_sum(const COEF& coef, int count, uint32_t* out, uint64_t cin, uint64_t* sc) {
#pragma unroll 1
    for (int base = 0; base < count; base += kChunkE * NT) {
        const int q0 = base + gtid<NT>() * kChunkE;
        uint32_t L[kChunkE];
        Acc96 acc;
#pragma unroll
        for (int e = 0; e < kChunkE; ++e) {
            uint32_t w0, w1, w2;
            coef(q0 + e, w0, w1, w2);
            L[e] = acc.add_shift(w0, w1, w2);
        }
        cin = block_resolve<kChunkE, NT, NT>(L, acc.rest(), cin, sc);
#pragma unroll
        for (int e = 0; e < kChunkE; ++e) out[q0 + e] = L[e];
    }
    gsync<NT>();
    return cin;
}

template <int NT>
__device__ __noinline__ uint64_t g_carry_product(const F2* v2, const F1* v1, int n, uint32_t* out, uint64_t* sc) {
    auto coef = [&](int q, uint32_t& w0, uint32_t& w1, uint32_t& w2) {
        const bool hi = q >= n;
        const int e = swz(hi ? q - n : q);
        const F2 a2 = v2[e];
        const F1 a1 = v1[e];
        crt3(hi ? a1.im : a1.re, hi ? a2.im : a2.re, w0, w1, w2);
    };
    return chunked_sum<NT>(coef, 2 * n, out, 0, sc);
}

template <int NT>
__device__ __noinline__ void g_carry_low_and_pack(F2* v2, F1* v1, int n, uint64_t* sc) {
    uint64_t cin = 0;
#pragma unroll 1
    for (int base = 0; base < n; base += kChunkE * NT) {
        const int q0 = base + gtid<NT>() * kChunkE;
        uint32_t L[kChunkE];
        Acc96 acc;
#pragma unroll
        for (int e = 0; e < kChunkE; ++e) {
            uint32_t w0, w1, w2;
            const int el = swz(q0 + e);
            crt3(v1[el].re, v2[el].re, w0, w1, w2);
            L[e] = acc.add_shift(w0, w1, w2);
        }
        cin = block_resolve<kChunkE, NT, NT>(L, acc.rest(), cin, sc);
#pragma unroll
        for (int e = 0; e < kChunkE; e += 2) {
            const int j = swz((q0 + e) >> 1);
            F2 z2; z2.re = L[e]; z2.im = L[e + 1];
            const uint32_t r0 = (L[e] & P1) + (L[e] >> 31), r1 = (L[e + 1] & P1) + (L[e + 1] >> 31);
            F1 z1; z1.re = min(r0, r0 - P1); z1.im = min(r1, r1 - P1);
            v2[j] = z2;
            v1[j] = z1;
        }
    }
    gsync<NT>();
}

template <int NT>
__device__ __noinline__ bool g_wrap_combine(const F2* v2, const F1* v1, int n, const uint32_t* tl, uint32_t* x, uint64_t* sc) {
    auto first = [&](int q, uint32_t& w0, uint32_t& w1, uint32_t& w2) {
        const int el = swz(q >> 1);
        if (q & 1) crt3(v1[el].im, v2[el].im, w0, w1, w2);
        else crt3(v1[el].re, v2[el].re, w0, w1, w2);
        const uint64_t lo = (((uint64_t)w1 << 32) | w0) + tl[q];
        w2 += lo < (uint64_t)tl[q];
        w0 = (uint32_t)lo;
        w1 = (uint32_t)(lo >> 32);
    };
    uint64_t top = chunked_sum<NT>(first, n, x, 0, sc);
    auto again = [&](int q, uint32_t& w0, uint32_t& w1, uint32_t& w2) { w0 = x[q]; w1 = 0; w2 = 0; };
    while (top != 0) top = chunked_sum<NT>(again, n, x, top, sc);   // end-around carry
    auto high = [&](int q, uint32_t& w0, uint32_t& w1, uint32_t& w2) {
        const uint64_t s = (uint64_t)x[q] + tl[n + q];
        w0 = (uint32_t)s; w1 = (uint32_t)(s >> 32); w2 = 0;
    };
    return chunked_sum<NT>(high, n, x, 0, sc) == 0;
}

// The half-pointwise step over the h-element vector in global memory (pairs cross tiles).
template <int NT>
__device__ __noinline__ void half_pointwise_rt(F2* v2, F1* v1, int H, const F2* __restrict__ ab2, const F1* __restrict__ ab1) {
#pragma unroll 1
    for (int tau = gtid<NT>(); tau < H / 2 + 1; tau += NT) half_pointwise_pair(v2, v1, H, ab2, ab1, tau);
    gsync<NT>();
}

// ---- the REDC without the wraparound path on global vectors ----
// m = the low k limbs of the product's real parts (k <= n) into out, as carry_low_to.
template <int NT>
__device__ __noinline__ void g_carry_low_to(const F2* v2, const F1* v1, int n, uint32_t* out, int k, uint64_t* sc) {
    uint64_t cin = 0;
#pragma unroll 1
    for (int base = 0; base < k; base += kChunkE * NT) {
        const int q0 = base + gtid<NT>() * kChunkE;
        uint32_t L[kChunkE];
        Acc96 acc;
#pragma unroll
        for (int e = 0; e < kChunkE; ++e) {
            uint32_t w0 = 0, w1 = 0, w2 = 0;
            if (q0 + e < n) {
                const int el = swz(q0 + e);
                crt3(v1[el].re, v2[el].re, w0, w1, w2);
            }
            L[e] = acc.add_shift(w0, w1, w2);
        }
        cin = block_resolve<kChunkE, NT, NT>(L, acc.rest(), cin, sc);
#pragma unroll
        for (int e = 0; e < kChunkE; ++e)
            if (q0 + e < k) out[q0 + e] = L[e];
    }
    gsync<NT>();
}

// x = (T + m N) / R, as carry_shift_add, in chunks over the 2n coefficients of m N.
template <int NT>
__device__ __noinline__ bool g_carry_shift_add(const F2* v2, const F1* v1, int n, const uint32_t* tl, uint32_t* x, int k,
                                               uint32_t flag, uint64_t* sc) {
    int stray = 0;
    uint64_t cin = 0;
#pragma unroll 1
    for (int base = 0; base < 2 * n; base += kChunkE * NT) {
        const int q0 = base + gtid<NT>() * kChunkE;
        uint32_t L[kChunkE];
        Acc96 acc;
#pragma unroll
        for (int e = 0; e < kChunkE; ++e) {
            const int q = q0 + e;
            const bool hi = q >= n;
            const int el = swz(hi ? q - n : q);
            uint32_t w0, w1, w2;
            crt3(hi ? v1[el].im : v1[el].re, hi ? v2[el].im : v2[el].re, w0, w1, w2);
            const uint64_t add = (q >= k && q < 2 * k ? (uint64_t)tl[q] : 0u) + (q == k ? flag : 0u);
            const uint64_t lo = (((uint64_t)w1 << 32) | w0) + add;
            w2 += lo < add;
            L[e] = acc.add_shift((uint32_t)lo, (uint32_t)(lo >> 32), w2);
        }
        cin = block_resolve<kChunkE, NT, NT>(L, acc.rest(), cin, sc);
#pragma unroll
        for (int e = 0; e < kChunkE; ++e) {
            const int q = q0 + e;
            if (q >= k && q < 2 * k) x[q - k] = L[e];
            else if (q >= 2 * k) stray |= L[e] != 0;
        }
    }
    return !gsync_or<NT>(stray) && cin == 0;
}

// ---- the wraparound steps on global vectors ----
enum { kStepOk = 0, kStepCarry = 1, kStepTimeout = 2 };

// REDC from T (tl, 2n limbs) into x, wraparound path, as redc_wrap. Returns a kStep* status
// (the same on every thread) and advances the mbarrier parities.
template <int NT>
__device__ __forceinline__ int g_redc_wrap(F2* w2, F1* w1, int m, const uint32_t* tl, uint32_t* x, const F2* cc2,
                                           const F1* cc1, const F2K* tab2, const F1* tab1, uint64_t* sc,
                                           const TileSmem& sm, uint32_t& par) {
    const int n = 1 << m, h = n / 2;
    const F2K* tt2 = tab2 + glt_tile_off(m);
    const F1* tt1 = tab1 + glt_tile_off(m);
    g_fwd<NT>(m, true, tl, w2, w1, tab2, tab1);
    if (!tile_phase<NT>(w2, w1, n, tt2, tt1, SpecMulRT{cc2, cc1, n / 8}, kTileFull, sm, par)) return kStepTimeout;
    par = tile_par_next(par, n);
    g_inv<NT, true>(m, true, w2, w1, tab2, tab1);
    g_carry_low_and_pack<NT>(w2, w1, n, sc);
    // Cyclic m N mod (R - 1) through the half-length transform of the packed limbs.
    const F2K* ht2 = tab2 + glt_half_off(m);
    const F1* ht1 = tab1 + glt_half_off(m);
    const bool half_global = m - 1 > kTileLog;
    if (half_global) g_fwd<NT>(m - 1, false, nullptr, w2, w1, ht2, ht1);
    if (!tile_phase<NT>(w2, w1, h, tt2, tt1, SquareOp{1}, kTileDif, sm, par)) return kStepTimeout;
    par = tile_par_next(par, h);
    half_pointwise_rt<NT>(w2, w1, h, cc2 + n, cc1 + n);
    if (!tile_phase<NT>(w2, w1, h, tt2, tt1, SquareOp{1}, kTileDit, sm, par)) return kStepTimeout;
    par = tile_par_next(par, h);
    if (half_global) g_inv<NT, false>(m - 1, false, w2, w1, ht2, ht1);
    return g_wrap_combine<NT>(w2, w1, n, tl, x, sc) ? kStepOk : kStepCarry;
}

// REDC without the wraparound path in global mode (as redc_plain). Returns a kStep* status.
template <int NT>
__device__ __forceinline__ int g_redc_plain(F2* w2, F1* w1, int m, const uint32_t* tl, uint32_t* x, const F2* cc2,
                                            const F1* cc1, const F2K* tab2, const F1* tab1, uint64_t* sc,
                                            const TileSmem& sm, uint32_t& par, int k) {
    const int n = 1 << m;
    const F2K* tt2 = tab2 + glt_tile_off(m);
    const F1* tt1 = tab1 + glt_tile_off(m);
    int nz = 0;
    for (int q = gtid<NT>(); q < k; q += NT) nz |= tl[q] != 0;
    const uint32_t flag = gsync_or<NT>(nz) ? 1u : 0u;
    g_fwd<NT>(m, true, tl, w2, w1, tab2, tab1, k);
    if (!tile_phase<NT>(w2, w1, n, tt2, tt1, SpecMulRT{cc2, cc1, n / 8}, kTileFull, sm, par)) return kStepTimeout;
    par = tile_par_next(par, n);
    g_inv<NT, true>(m, true, w2, w1, tab2, tab1);
    g_carry_low_to<NT>(w2, w1, n, x, k, sc);
    g_fwd<NT>(m, true, x, w2, w1, tab2, tab1, k);
    if (!tile_phase<NT>(w2, w1, n, tt2, tt1, SpecMulRT{cc2 + n, cc1 + n, n / 8}, kTileFull, sm, par)) return kStepTimeout;
    par = tile_par_next(par, n);
    g_inv<NT, false>(m, true, w2, w1, tab2, tab1);
    return g_carry_shift_add<NT>(w2, w1, n, tl, x, k, flag, sc) ? kStepOk : kStepCarry;
}

// Up to `bits` steps on one slot, global mode (as step_slot). `par` carries the mbarrier
// parities from one call to the next. Returns false (on every thread) after a bulk copy that did
// not complete in time; the parities are then no longer usable.
template <int NT>
__device__ __forceinline__ bool gstep_slot(const GArgs& g, uint32_t slot, uint32_t bits, const TileSmem& sm, uint64_t* sc,
                                           uint32_t& par) {
    const SlotArgs& a = g.a;
    const int m = g.m, n = 1 << m, k = (int)a.k;
    uint32_t* x = a.x + (size_t)slot * k;
    uint32_t* tl = a.tbuf + (size_t)slot * 2 * n;
    const F2* cc2 = a.c2 + (size_t)slot * 2 * n;
    const F1* cc1 = a.c1 + (size_t)slot * 2 * n;
    F2* w2 = g.w2 + (size_t)slot * n;
    F1* w1 = g.w1 + (size_t)slot * n;
    const uint32_t* ex = a.exp + (size_t)slot * a.ew;
    const uint32_t nb = a.nbits[slot];
    uint32_t pos = a.pos[slot];
    const F2K* tt2 = a.tab2 + glt_tile_off(m);
    const F1* tt1 = a.tab1 + glt_tile_off(m);
    int st = kStepOk;
    bool carry_ok = true;
    for (uint32_t it = 0; it < bits && pos < nb; ++it, ++pos) {
        const uint32_t bit = (ex[pos >> 5] >> (31 - (pos & 31))) & 1;
        const uint32_t c = bit ? a.base : 1;
        g_fwd<NT>(m, true, x, w2, w1, a.tab2, a.tab1, k);
        if (!tile_phase<NT>(w2, w1, n, tt2, tt1, SquareOp{c}, kTileFull, sm, par)) { st = kStepTimeout; break; }
        par = tile_par_next(par, n);
        g_inv<NT, false>(m, true, w2, w1, a.tab2, a.tab1);
        carry_ok &= g_carry_product<NT>(w2, w1, n, tl, sc) == 0;
        if (a.bare) continue;
        st = a.plain ? g_redc_plain<NT>(w2, w1, m, tl, x, cc2, cc1, a.tab2, a.tab1, sc, sm, par, k)
                     : g_redc_wrap<NT>(w2, w1, m, tl, x, cc2, cc1, a.tab2, a.tab1, sc, sm, par);
        if (st == kStepTimeout) break;
        carry_ok &= st == kStepOk;
    }
    gsync<NT>();   // every thread has read pos before it is written
    if (gtid<NT>() == 0) {
        a.pos[slot] = pos;
        if (st == kStepTimeout) a.err[slot] = kErrTimeout;
        else if (!carry_ok) a.err[slot] = 1;
    }
    return st != kStepTimeout;
}

// The uniform launch, global mode: one block per slot first + blockIdx.x.
template <int NT>
__global__ void __launch_bounds__(NT, 2) gstep_kernel(GArgs g, uint32_t first, uint32_t bits) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ uint64_t sc[CarryScratch<NT>::words];
    __shared__ uint64_t bars[2];
    const TileSmem sm{smem_raw, bars};
    tile_init<NT>(sm);
    uint32_t par = 0;
    gstep_slot<NT>(g, first + blockIdx.x, bits, sm, sc, par);
}

// x[out] <- x[ia] x[ib] R^-1, global mode; spec: n-element scratch for F(x[ib]).
template <int NT>
__global__ void __launch_bounds__(NT, 2) gmul_kernel(GArgs g, uint32_t out, uint32_t ia, uint32_t ib, F2* spec2, F1* spec1) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ uint64_t sc[CarryScratch<NT>::words];
    __shared__ uint64_t bars[2];
    const TileSmem sm{smem_raw, bars};
    tile_init<NT>(sm);
    const SlotArgs& a = g.a;
    const int m = g.m, n = 1 << m;
    F2* w2 = g.w2 + (size_t)out * n;
    F1* w1 = g.w1 + (size_t)out * n;
    const F2K* tt2 = a.tab2 + glt_tile_off(m);
    const F1* tt1 = a.tab1 + glt_tile_off(m);
    uint32_t par = 0;
    int st = kStepTimeout;
    const int k = (int)a.k;
    g_fwd<NT>(m, true, a.x + (size_t)ib * k, w2, w1, a.tab2, a.tab1, k);
    if (tile_phase<NT>(w2, w1, n, tt2, tt1, SpecStoreRT{spec2, spec1, n / 8}, kTileDifOp, sm, par)) {
        par = tile_par_next(par, n);
        g_fwd<NT>(m, true, a.x + (size_t)ia * k, w2, w1, a.tab2, a.tab1, k);
        if (tile_phase<NT>(w2, w1, n, tt2, tt1, SpecMulRT{spec2, spec1, n / 8}, kTileFull, sm, par)) {
            par = tile_par_next(par, n);
            g_inv<NT, false>(m, true, w2, w1, a.tab2, a.tab1);
            uint32_t* tl = a.tbuf + (size_t)out * 2 * n;
            const bool fits = g_carry_product<NT>(w2, w1, n, tl, sc) == 0;
            uint32_t* xo = a.x + (size_t)out * k;
            const F2* oc2 = a.c2 + (size_t)out * 2 * n;
            const F1* oc1 = a.c1 + (size_t)out * 2 * n;
            st = a.plain ? g_redc_plain<NT>(w2, w1, m, tl, xo, oc2, oc1, a.tab2, a.tab1, sc, sm, par, k)
                         : g_redc_wrap<NT>(w2, w1, m, tl, xo, oc2, oc1, a.tab2, a.tab1, sc, sm, par);
            if (st == kStepOk && !fits) st = kStepCarry;
        }
    }
    if (gtid<NT>() == 0 && st != kStepOk) a.err[out] = st == kStepTimeout ? kErrTimeout : 1;
}

// Per-slot constants in global mode (as setup_kernel): F(N') through the global passes and the
// tile DIF, then the wraparound factors from the half transform of N.
template <int NT>
__global__ void __launch_bounds__(NT, 2) gsetup_kernel(GArgs g, const uint32_t* nl, const uint32_t* npl, F2* c2, F1* c1,
                                                       F2 inv8h2, F1 inv8h1, uint32_t first, const uint32_t* slots) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ uint64_t bars[2];
    const TileSmem sm{smem_raw, bars};
    tile_init<NT>(sm);
    const SlotArgs& a = g.a;
    const int m = g.m, n = 1 << m, h = n / 2;
    const uint32_t slot = slots ? slots[blockIdx.x] : first + blockIdx.x;
    const size_t row = slots ? blockIdx.x : slot;
    F2* w2 = g.w2 + (size_t)slot * n;
    F1* w1 = g.w1 + (size_t)slot * n;
    F2* o2 = c2 + (size_t)slot * 2 * n;
    F1* o1 = c1 + (size_t)slot * 2 * n;
    const F2K* tt2 = a.tab2 + glt_tile_off(m);
    const F1* tt1 = a.tab1 + glt_tile_off(m);
    uint32_t par = 0;
    bool ok = false;
    const int k = (int)a.k;
    g_fwd<NT>(m, true, npl + row * k, w2, w1, a.tab2, a.tab1, k);
    if (a.plain) {
        // F(N) in the second half (cpu.rs:518-521).
        if (tile_phase<NT>(w2, w1, n, tt2, tt1, SpecStoreRT{o2, o1, n / 8}, kTileDifOp, sm, par)) {
            par = tile_par_next(par, n);
            g_fwd<NT>(m, true, nl + row * k, w2, w1, a.tab2, a.tab1, k);
            ok = tile_phase<NT>(w2, w1, n, tt2, tt1, SpecStoreRT{o2 + n, o1 + n, n / 8}, kTileDifOp, sm, par);
        }
        if (gtid<NT>() == 0 && !ok) a.err[slot] = kErrTimeout;
        return;
    }
    if (tile_phase<NT>(w2, w1, n, tt2, tt1, SpecStoreRT{o2, o1, n / 8}, kTileDifOp, sm, par)) {
        par = tile_par_next(par, n);
        pack_pairs(nl + row * k, w2, w1, h, NT);
        const F2K* ht2 = a.tab2 + glt_half_off(m);
        const F1* ht1 = a.tab1 + glt_half_off(m);
        if (m - 1 > kTileLog) g_fwd<NT>(m - 1, false, nullptr, w2, w1, ht2, ht1);
        if (tile_phase<NT>(w2, w1, h, tt2, tt1, SquareOp{1}, kTileDif, sm, par)) {
            half_factors_block(w2, w1, h, a.tab2 + glt_unpack_off(m), a.tab1 + glt_unpack_off(m), o2 + n, o1 + n, inv8h2,
                               inv8h1, NT);
            ok = true;
        }
    }
    if (gtid<NT>() == 0 && !ok) a.err[slot] = kErrTimeout;
}

// The Transform trait's forward or inverse of vector first + blockIdx.x in global mode, in place
// in a device buffer in the kernels' element order; the result is canonical. A bulk copy that
// does not complete in time sets err[0] to 2.
template <int NT>
__global__ void __launch_bounds__(NT, 2) gtransform_kernel(F2* v2, F1* v1, const F2K* tab2, const F1* tab1, int m,
                                                           uint32_t first, int inverse, uint32_t* err) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ uint64_t bars[2];
    const TileSmem sm{smem_raw, bars};
    tile_init<NT>(sm);
    const int n = 1 << m, P = gl_passes(m);
    F2* w2 = v2 + (size_t)(first + blockIdx.x) * n;
    F1* w1 = v1 + (size_t)(first + blockIdx.x) * n;
    const F2K* tt2 = tab2 + glt_tile_off(m);
    const F1* tt1 = tab1 + glt_tile_off(m);
    bool ok;
    if (!inverse) {
        const int R0 = gl_radix(m, 0), lq0 = gl_lq(m, 0);
        const F2K* t2 = tab2 + gl_fwd_off(m, 0, true);
        const F1* t1 = tab1 + gl_fwd_off(m, 0, true);
        const F2K* c2 = tab2 + gl_in_const_off(m, true);
        const F1* c1 = tab1 + gl_in_const_off(m, true);
        if (R0 == 8) g_dif_first_complex<8, NT>(w2, w1, t2, t1, c2, c1, lq0);
        else if (R0 == 4) g_dif_first_complex<4, NT>(w2, w1, t2, t1, c2, c1, lq0);
        else g_dif_first_complex<2, NT>(w2, w1, t2, t1, c2, c1, lq0);
        for (int i = 1; i < P; ++i)
            g_pass<NT>(gl_radix(m, i), true, w2, w1, tab2 + gl_fwd_off(m, i, true), tab1 + gl_fwd_off(m, i, true),
                       gl_lq(m, i), n);
        ok = tile_phase<NT>(w2, w1, n, tt2, tt1, SquareOp{1}, kTileDif, sm, 0);
    } else {
        ok = tile_phase<NT>(w2, w1, n, tt2, tt1, SquareOp{1}, kTileDit, sm, 0);
        if (ok) g_inv<NT, false>(m, true, w2, w1, tab2, tab1);
    }
    if (ok)
        for (int e = gtid<NT>(); e < n; e += NT) w2[e] = lccanon(w2[e]);
    if (gtid<NT>() == 0 && !ok) *err = kErrTimeout;
}

}  // namespace mm
