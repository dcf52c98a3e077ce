// Host-side field arithmetic and table generation of the B200 backend: the reference's
// GF(M31^2) x GF(M61^2) tables (montmul/src/field.rs:224-281) rearranged into the per-pass
// layouts of mm_common.h, plus the wraparound path's unpack roots (cpu.rs:165-179).
#pragma once
#include <cstdint>
#include <stdexcept>
#include <vector>

#include "mm_common.h"

namespace mm {
namespace host {

typedef unsigned __int128 u128;

inline uint32_t add1(uint32_t a, uint32_t b) { uint32_t s = a + b; return s >= P1 ? s - P1 : s; }
inline uint32_t sub1(uint32_t a, uint32_t b) { return a >= b ? a - b : a + P1 - b; }
inline uint32_t mul1(uint32_t a, uint32_t b) {
    uint64_t t = (uint64_t)a * b;
    uint32_t s = (uint32_t)((t & P1) + (t >> 31));
    return s >= P1 ? s - P1 : s;
}
inline uint64_t add2(uint64_t a, uint64_t b) { uint64_t s = a + b; return s >= P2 ? s - P2 : s; }
inline uint64_t sub2(uint64_t a, uint64_t b) { return a >= b ? a - b : a + P2 - b; }
inline uint64_t mul2(uint64_t a, uint64_t b) {
    u128 t = (u128)a * b;
    uint64_t s = ((uint64_t)t & P2) + (uint64_t)(t >> 61);
    return s >= P2 ? s - P2 : s;
}

// GF(p^2) for either prime, i^2 = -1 (field.rs:131-222).
template <class E> struct Gf;
template <> struct Gf<F1> {
    static constexpr int order_log2 = 32;
    static constexpr uint64_t cofactor = (1ull << 30) - 1;
    static F1 make(uint64_t re, uint64_t im) { return F1{(uint32_t)re, (uint32_t)im}; }
    static F1 add(F1 a, F1 b) { return F1{add1(a.re, b.re), add1(a.im, b.im)}; }
    static F1 sub(F1 a, F1 b) { return F1{sub1(a.re, b.re), sub1(a.im, b.im)}; }
    static F1 mul(F1 a, F1 b) {
        return F1{sub1(mul1(a.re, b.re), mul1(a.im, b.im)), add1(mul1(a.re, b.im), mul1(a.im, b.re))};
    }
    static uint32_t bpow(uint32_t b, uint64_t e) { uint32_t r = 1; while (e) { if (e & 1) r = mul1(r, b); b = mul1(b, b); e >>= 1; } return r; }
    static F1 inv(F1 a) {
        uint32_t n = add1(mul1(a.re, a.re), mul1(a.im, a.im));
        uint32_t ni = bpow(n, P1 - 2);
        return F1{mul1(a.re, ni), mul1(sub1(0, a.im), ni)};
    }
    static F1 from(uint64_t v) { return F1{(uint32_t)(v % P1), 0}; }
};
template <> struct Gf<F2> {
    static constexpr int order_log2 = 62;
    static constexpr uint64_t cofactor = (1ull << 60) - 1;
    static F2 make(uint64_t re, uint64_t im) { return F2{re, im}; }
    static F2 add(F2 a, F2 b) { return F2{add2(a.re, b.re), add2(a.im, b.im)}; }
    static F2 sub(F2 a, F2 b) { return F2{sub2(a.re, b.re), sub2(a.im, b.im)}; }
    static F2 mul(F2 a, F2 b) {
        return F2{sub2(mul2(a.re, b.re), mul2(a.im, b.im)), add2(mul2(a.re, b.im), mul2(a.im, b.re))};
    }
    static uint64_t bpow(uint64_t b, uint64_t e) { uint64_t r = 1; while (e) { if (e & 1) r = mul2(r, b); b = mul2(b, b); e >>= 1; } return r; }
    static F2 inv(F2 a) {
        uint64_t n = add2(mul2(a.re, a.re), mul2(a.im, a.im));
        uint64_t ni = bpow(n, P2 - 2);
        return F2{mul2(a.re, ni), mul2(sub2(0, a.im), ni)};
    }
    static F2 from(uint64_t v) { return F2{v % P2, 0}; }
};

template <class E> inline bool eq(E a, E b) { return a.re == b.re && a.im == b.im; }
template <class E> inline E one() { return Gf<E>::make(1, 0); }
template <class E> inline E iunit() { return Gf<E>::make(0, 1); }
template <class E> inline E gpow(E b, uint64_t e) {
    E r = one<E>();
    while (e) { if (e & 1) r = Gf<E>::mul(r, b); b = Gf<E>::mul(b, b); e >>= 1; }
    return r;
}

// Generator of the 2-Sylow subgroup: the first a + i, a >= 1, whose cofactor power has order
// exactly 2^order_log2 (field.rs:111-120).
template <class E> inline E sylow2() {
    for (uint32_t a = 1;; ++a) {
        E g = gpow(Gf<E>::make(a, 1), Gf<E>::cofactor);
        if (!eq(gpow(g, 1ull << (Gf<E>::order_log2 - 1)), one<E>())) return g;
    }
}

// omega (primitive 2^m-th root) and zeta (zeta^(2^m) = i) of FieldTables::new(2^m) (field.rs:238-248).
template <class E> inline void roots(int m, E& omega, E& zeta) {
    E g = sylow2<E>();
    omega = gpow(g, 1ull << (Gf<E>::order_log2 - m));
    zeta = gpow(g, 1ull << (Gf<E>::order_log2 - m - 2));
    if (!eq(gpow(zeta, 1ull << m), iunit<E>())) zeta = Gf<E>::inv(zeta);
    if (!eq(gpow(zeta, 1ull << m), iunit<E>())) throw std::runtime_error("zeta^n != i");
}

inline int rev_bits(int v, int bits) {
    int r = 0;
    for (int b = 0; b < bits; ++b) r |= ((v >> b) & 1) << (bits - 1 - b);
    return r;
}

// Tables of one transform (length 2^m, weighted or not) into t[0 .. tab_size(m, weighted)).
template <class E> inline void gen_transform(int m, bool weighted, E* t) {
    E omega, zeta;
    roots<E>(m, omega, zeta);
    const int n = 1 << m, P = sched_passes(m);
    const E zi = Gf<E>::inv(zeta);
    for (int i = 0; i < P; ++i) {
        const int R = sched_radix(m, i), q = sched_q(m, i), lr = ilog2c(R);
        if (q <= 1) continue;
        const E W = gpow(omega, (uint64_t)(n / (R * q))), V = Gf<E>::inv(W);
        E* f = t + tab_fwd_off(m, i, weighted);
        E* b = t + tab_inv_off(m, i, weighted);
        const bool w0 = weighted && i == 0;
        for (int k = w0 ? 0 : 1; k < R; ++k) {
            const int row = w0 ? k : k - 1;
            const uint64_t rk = (uint64_t)rev_bits(k, lr);
            for (int j = 0; j < q; ++j) {
                E fw = gpow(W, rk * j), bw = gpow(V, rk * j);
                if (w0) { fw = Gf<E>::mul(fw, gpow(zeta, j)); bw = Gf<E>::mul(bw, gpow(zi, j)); }
                f[row * q + j] = fw;
                b[row * q + j] = bw;
            }
        }
    }
    if (weighted) {
        const int R0 = sched_radix(m, 0), q0 = sched_q(m, 0);
        const E ninv = Gf<E>::inv(Gf<E>::from((uint64_t)n));
        for (int k = 0; k < R0; ++k) {
            t[tab_in_const_off(m, true) + k] = gpow(zeta, (uint64_t)q0 * k);
            t[tab_out_const_off(m, true) + k] = Gf<E>::mul(gpow(zi, (uint64_t)q0 * k), ninv);
        }
    }
}

// All tables of transform length L = 2^(m+1) (layout lt_* of mm_common.h).
template <class E> inline std::vector<E> gen_length_tables(int m) {
    std::vector<E> t(lt_size(m), E{});
    gen_transform<E>(m, true, t.data() + lt_full_off(m));
    gen_transform<E>(m - 1, false, t.data() + lt_half_off(m));
    // Unpack roots over h = n/2 positions: w = primitive n-th root (= omega of length n).
    E omega, zeta;
    roots<E>(m, omega, zeta);
    const E wi = Gf<E>::inv(omega);
    const int h = 1 << (m - 1);
    for (int p = 0; p < h; ++p) {
        const int r = rev_bits(p, m - 1);
        t[lt_unpack_off(m) + p] = gpow(omega, (uint64_t)r);
        t[lt_unpack_off(m) + h + p] = gpow(wi, (uint64_t)r);
    }
    return t;
}

// The global passes of a length-2^m transform (weighted or not) into t[0 .. gl_tab_size).
// Same roots as gen_transform; powers are formed by repeated multiplication.
template <class E> inline void gen_global_transform(int m, bool weighted, E* t) {
    E omega, zeta;
    roots<E>(m, omega, zeta);
    const uint64_t n = 1ull << m;
    const E zi = Gf<E>::inv(zeta);
    for (int i = 0; i < gl_passes(m); ++i) {
        const int R = gl_radix(m, i), lr = ilog2c(R);
        const uint64_t q = 1ull << gl_lq(m, i);
        const E W = gpow(omega, n / (R * q)), V = Gf<E>::inv(W);
        E* f = t + gl_fwd_off(m, i, weighted);
        E* b = t + gl_inv_off(m, i, weighted);
        const bool w0 = weighted && i == 0;
        for (int k = w0 ? 0 : 1; k < R; ++k) {
            const int row = w0 ? k : k - 1;
            const uint64_t rk = (uint64_t)rev_bits(k, lr);
            const E fs = gpow(W, rk), bs = gpow(V, rk);
            E fw = one<E>(), bw = one<E>(), zf = one<E>(), zb = one<E>();
            for (uint64_t j = 0; j < q; ++j) {
                f[row * q + j] = w0 ? Gf<E>::mul(fw, zf) : fw;
                b[row * q + j] = w0 ? Gf<E>::mul(bw, zb) : bw;
                fw = Gf<E>::mul(fw, fs);
                bw = Gf<E>::mul(bw, bs);
                if (w0) { zf = Gf<E>::mul(zf, zeta); zb = Gf<E>::mul(zb, zi); }
            }
        }
    }
    if (weighted) {
        const int R0 = gl_radix(m, 0);
        const uint64_t q0 = 1ull << gl_lq(m, 0);
        const E ninv = Gf<E>::inv(Gf<E>::from(n));
        for (int k = 0; k < R0; ++k) {
            t[gl_in_const_off(m, true) + k] = gpow(zeta, q0 * k);
            t[gl_out_const_off(m, true) + k] = Gf<E>::mul(gpow(zi, q0 * k), ninv);
        }
    }
}

// All tables of global-mode length L = 2^(m+1) (layout glt_* of mm_common.h).
template <class E> inline std::vector<E> gen_global_length_tables(int m) {
    std::vector<E> t(glt_size(m), E{});
    gen_global_transform<E>(m, true, t.data());
    gen_transform<E>(kTileLog, false, t.data() + glt_tile_off(m));
    if (m - 1 > kTileLog) gen_global_transform<E>(m - 1, false, t.data() + glt_half_off(m));
    E omega, zeta;
    roots<E>(m, omega, zeta);
    const E wi = Gf<E>::inv(omega);
    const int h = 1 << (m - 1);
    std::vector<E> pw(h), pwi(h);   // omega^j and omega^-j, j < h
    E a = one<E>(), b = one<E>();
    for (int j = 0; j < h; ++j) { pw[j] = a; pwi[j] = b; a = Gf<E>::mul(a, omega); b = Gf<E>::mul(b, wi); }
    for (int p = 0; p < h; ++p) {
        const int r = rev_bits(p, m - 1);
        t[glt_unpack_off(m) + p] = pw[r];
        t[glt_unpack_off(m) + h + p] = pwi[r];
    }
    return t;
}

// M61 tables as the device's Karatsuba products read them: (re, im, re + im, im - re) mod p.
inline std::vector<F2K> karatsuba_form(const std::vector<F2>& t) {
    std::vector<F2K> out(t.size());
    for (size_t i = 0; i < t.size(); ++i)
        out[i] = F2K{t[i].re, t[i].im, add2(t[i].re, t[i].im), sub2(t[i].im, t[i].re)};
    return out;
}

// (8 h)^-1 with h = n/2 = 2^(m-1) (cpu.rs:243).
template <class E> inline E inv8h(int m) { return Gf<E>::inv(Gf<E>::from((uint64_t)8 << (m - 1))); }

// The device butterflies hard-code omega_8 = (1 + i) 2^s and omega_4 = i; they must be the
// reference's roots omega_n^(n/8) and omega_n^(n/4) for every length.
inline bool check_fixed_roots() {
    for (int m = 3; m <= 24; ++m) {
        F1 o1, z1; roots<F1>(m, o1, z1);
        F2 o2, z2; roots<F2>(m, o2, z2);
        const uint64_t n = 1ull << m;
        if (!eq(gpow(o1, n / 4), iunit<F1>()) || !eq(gpow(o2, n / 4), iunit<F2>())) return false;
        if (!eq(gpow(o1, n / 8), F1{1u << 15, 1u << 15})) return false;
        if (!eq(gpow(o2, n / 8), F2{1ull << 30, 1ull << 30})) return false;
    }
    return true;
}

}  // namespace host
}  // namespace mm
