/* TEST INFRASTRUCTURE ONLY — CPU oracle for the MontMul hot path (see oracle.h).
 *
 * Every function below restates one function of the reference's Rust crate and names it by
 * file:line (paths inside the reference project). The arithmetic is exact and integer-only, so
 * the oracle's raw Montgomery limbs are the reference `Cpu` backend's, bit for bit.
 */
#include "oracle.h"

#include <pthread.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

typedef unsigned __int128 u128;

/* ---- field.rs:7-42: M31 and M61 arithmetic ---- */
#define P1 0x7fffffffu
#define P2 0x1fffffffffffffffull

static inline uint32_t add1(uint32_t a, uint32_t b) { uint32_t s = a + b; return s >= P1 ? s - P1 : s; }
static inline uint32_t sub1(uint32_t a, uint32_t b) { return a >= b ? a - b : a + P1 - b; }
static inline uint32_t mul1(uint32_t a, uint32_t b) {
    uint64_t t = (uint64_t)a * b;
    uint32_t s = (uint32_t)((t & P1) + (t >> 31));
    return s >= P1 ? s - P1 : s;
}
static inline uint64_t add2(uint64_t a, uint64_t b) { uint64_t s = a + b; return s >= P2 ? s - P2 : s; }
static inline uint64_t sub2(uint64_t a, uint64_t b) { return a >= b ? a - b : a + P2 - b; }
static inline uint64_t mul2(uint64_t a, uint64_t b) {
    u128 t = (u128)a * b;
    uint64_t s = ((uint64_t)t & P2) + (uint64_t)(t >> 61);
    return s >= P2 ? s - P2 : s;
}

/* ---- field.rs:131-222: GF(p^2) with i^2 = -1 ---- */
typedef oc_f1 F1;
typedef oc_f2 F2;

static inline F1 f1_new(uint32_t re, uint32_t im) { F1 r = {re, im}; return r; }
static inline F2 f2_new(uint64_t re, uint64_t im) { F2 r = {re, im}; return r; }
static inline F1 f1_from(uint32_t v) { return f1_new(v >= P1 ? v - P1 : v, 0); }      /* field.rs:139-141 */
static inline F2 f2_from(uint32_t v) { return f2_new(v, 0); }                         /* field.rs:186-188 */
static inline F1 f1_add(F1 a, F1 b) { return f1_new(add1(a.re, b.re), add1(a.im, b.im)); }
static inline F1 f1_sub(F1 a, F1 b) { return f1_new(sub1(a.re, b.re), sub1(a.im, b.im)); }
static inline F1 f1_mul(F1 a, F1 b) {                                                 /* field.rs:151-156 */
    return f1_new(sub1(mul1(a.re, b.re), mul1(a.im, b.im)), add1(mul1(a.re, b.im), mul1(a.im, b.re)));
}
static inline F1 f1_scale(F1 a, uint32_t c) { c = c >= P1 ? c - P1 : c; return f1_new(mul1(a.re, c), mul1(a.im, c)); }
static inline F2 f2_add(F2 a, F2 b) { return f2_new(add2(a.re, b.re), add2(a.im, b.im)); }
static inline F2 f2_sub(F2 a, F2 b) { return f2_new(sub2(a.re, b.re), sub2(a.im, b.im)); }
static inline F2 f2_mul(F2 a, F2 b) {                                                 /* field.rs:198-203 */
    return f2_new(sub2(mul2(a.re, b.re), mul2(a.im, b.im)), add2(mul2(a.re, b.im), mul2(a.im, b.re)));
}
static inline F2 f2_scale(F2 a, uint32_t c) { return f2_new(mul2(a.re, c), mul2(a.im, c)); }
static inline int f1_eq(F1 a, F1 b) { return a.re == b.re && a.im == b.im; }
static inline int f2_eq(F2 a, F2 b) { return a.re == b.re && a.im == b.im; }

static uint32_t base_pow1(uint32_t b, uint64_t e) {                                   /* field.rs:88-98 */
    uint32_t r = 1;
    while (e) { if (e & 1) r = mul1(r, b); b = mul1(b, b); e >>= 1; }
    return r;
}
static uint64_t base_pow2(uint64_t b, uint64_t e) {                                   /* field.rs:99-109 */
    uint64_t r = 1;
    while (e) { if (e & 1) r = mul2(r, b); b = mul2(b, b); e >>= 1; }
    return r;
}
static F1 f1_pow(F1 b, uint64_t e) {                                                  /* field.rs:60-71 */
    F1 r = f1_new(1, 0);
    while (e) { if (e & 1) r = f1_mul(r, b); b = f1_mul(b, b); e >>= 1; }
    return r;
}
static F2 f2_pow(F2 b, uint64_t e) {
    F2 r = f2_new(1, 0);
    while (e) { if (e & 1) r = f2_mul(r, b); b = f2_mul(b, b); e >>= 1; }
    return r;
}
static F1 f1_inv(F1 a) {                                                              /* field.rs:162-166 */
    uint32_t n = add1(mul1(a.re, a.re), mul1(a.im, a.im));
    uint32_t ni = base_pow1(n, P1 - 2);
    return f1_new(mul1(a.re, ni), mul1(sub1(0, a.im), ni));
}
static F2 f2_inv(F2 a) {                                                              /* field.rs:208-212 */
    uint64_t n = add2(mul2(a.re, a.re), mul2(a.im, a.im));
    uint64_t ni = base_pow2(n, P2 - 2);
    return f2_new(mul2(a.re, ni), mul2(sub2(0, a.im), ni));
}
static inline F1 f1_i(void) { return f1_new(0, 1); }
static inline F2 f2_i(void) { return f2_new(0, 1); }
static inline F1 f1_conj(F1 a) { return f1_new(a.re, sub1(0, a.im)); }               /* cpu.rs:148-155 */
static inline F2 f2_conj(F2 a) { return f2_new(a.re, sub2(0, a.im)); }                /* cpu.rs:156-163 */

/* field.rs:111-129: smallest a + i, a >= 1, whose cofactor power has order exactly 2^e. */
static F1 f1_sylow2(void) {
    for (uint32_t a = 1;; a++) {
        F1 g = f1_pow(f1_add(f1_from(a), f1_scale(f1_i(), 1)), (1ull << 30) - 1);
        if (!f1_eq(f1_pow(g, 1ull << 31), f1_new(1, 0))) return g;
    }
}
static F2 f2_sylow2(void) {
    for (uint32_t a = 1;; a++) {
        F2 g = f2_pow(f2_add(f2_from(a), f2_scale(f2_i(), 1)), (1ull << 60) - 1);
        if (!f2_eq(f2_pow(g, 1ull << 61), f2_new(1, 0))) return g;
    }
}

void oc_sylow2_f1(uint32_t out[2]) { F1 g = f1_sylow2(); out[0] = g.re; out[1] = g.im; }
void oc_sylow2_f2(uint64_t out[2]) { F2 g = f2_sylow2(); out[0] = g.re; out[1] = g.im; }
void oc_pow_f1(const uint32_t a[2], uint64_t e, uint32_t out[2]) { F1 r = f1_pow(f1_new(a[0], a[1]), e); out[0] = r.re; out[1] = r.im; }
void oc_pow_f2(const uint64_t a[2], uint64_t e, uint64_t out[2]) { F2 r = f2_pow(f2_new(a[0], a[1]), e); out[0] = r.re; out[1] = r.im; }

/* field.rs:283-294 */
uint32_t oc_crt_inv(void) { return base_pow1((uint32_t)(P2 % P1), P1 - 2); }
static inline u128 crt(uint32_t c1, uint64_t c2, uint32_t inv) {
    uint32_t c2m = (uint32_t)(c2 % P1);
    uint32_t h = mul1(sub1(c1, c2m), inv);
    return (u128)c2 + (u128)P2 * h;
}
void oc_crt(uint32_t c1, uint64_t c2, uint64_t out[2]) {
    u128 v = crt(c1, c2, oc_crt_inv());
    out[0] = (uint64_t)v; out[1] = (uint64_t)(v >> 64);
}

/* ---- field.rs:224-281: tables for complex length n ---- */
typedef struct {
    size_t n;
    F1 *tw1, *itw1, *w1, *iw1;
    F2 *tw2, *itw2, *w2, *iw2;
} Tables;

static int log2z(size_t n) { int l = 0; while (((size_t)1 << l) < n) l++; return l; }

static Tables *tables_new(size_t n) {
    if (n < 2 || (n & (n - 1))) return NULL;
    int log = log2z(n);
    Tables *t = calloc(1, sizeof *t);
    t->n = n;
    t->tw1 = malloc(sizeof(F1) * (n / 2)); t->itw1 = malloc(sizeof(F1) * (n / 2));
    t->w1 = malloc(sizeof(F1) * n); t->iw1 = malloc(sizeof(F1) * n);
    t->tw2 = malloc(sizeof(F2) * (n / 2)); t->itw2 = malloc(sizeof(F2) * (n / 2));
    t->w2 = malloc(sizeof(F2) * n); t->iw2 = malloc(sizeof(F2) * n);
    {   /* GF(M31^2), ORDER_LOG2 = 32 */
        F1 g = f1_sylow2();
        F1 omega = f1_pow(g, 1ull << (32 - log));
        F1 zeta = f1_pow(g, 1ull << (32 - log - 2));
        if (!f1_eq(f1_pow(zeta, n), f1_i())) zeta = f1_inv(zeta);
        F1 ninv = f1_inv(f1_from((uint32_t)n));
        F1 x = f1_new(1, 0), oi = f1_inv(omega), zi = f1_inv(zeta);
        for (size_t j = 0; j < n / 2; j++) { t->tw1[j] = x; x = f1_mul(x, omega); }
        x = f1_new(1, 0);
        for (size_t j = 0; j < n / 2; j++) { t->itw1[j] = x; x = f1_mul(x, oi); }
        x = f1_new(1, 0);
        for (size_t j = 0; j < n; j++) { t->w1[j] = x; x = f1_mul(x, zeta); }
        x = f1_new(1, 0);
        for (size_t j = 0; j < n; j++) { t->iw1[j] = f1_mul(x, ninv); x = f1_mul(x, zi); }
    }
    {   /* GF(M61^2), ORDER_LOG2 = 62 */
        F2 g = f2_sylow2();
        F2 omega = f2_pow(g, 1ull << (62 - log));
        F2 zeta = f2_pow(g, 1ull << (62 - log - 2));
        if (!f2_eq(f2_pow(zeta, n), f2_i())) zeta = f2_inv(zeta);
        F2 ninv = f2_inv(f2_from((uint32_t)n));
        F2 x = f2_new(1, 0), oi = f2_inv(omega), zi = f2_inv(zeta);
        for (size_t j = 0; j < n / 2; j++) { t->tw2[j] = x; x = f2_mul(x, omega); }
        x = f2_new(1, 0);
        for (size_t j = 0; j < n / 2; j++) { t->itw2[j] = x; x = f2_mul(x, oi); }
        x = f2_new(1, 0);
        for (size_t j = 0; j < n; j++) { t->w2[j] = x; x = f2_mul(x, zeta); }
        x = f2_new(1, 0);
        for (size_t j = 0; j < n; j++) { t->iw2[j] = f2_mul(x, ninv); x = f2_mul(x, zi); }
    }
    return t;
}

static void tables_free(Tables *t) {
    if (!t) return;
    free(t->tw1); free(t->itw1); free(t->w1); free(t->iw1);
    free(t->tw2); free(t->itw2); free(t->w2); free(t->iw2);
    free(t);
}

/* A small cache of tables by n, shared by all states (cpu.rs:38-41). */
static pthread_mutex_t g_tab_lock = PTHREAD_MUTEX_INITIALIZER;
static Tables *g_tabs[40];

static Tables *tables(size_t n) {
    int l = log2z(n);
    if (l <= 0 || l >= 40 || ((size_t)1 << l) != n) return NULL;
    pthread_mutex_lock(&g_tab_lock);
    if (!g_tabs[l]) g_tabs[l] = tables_new(n);
    Tables *t = g_tabs[l];
    pthread_mutex_unlock(&g_tab_lock);
    return t;
}

int oc_tables(size_t n, F1 *tw1, F1 *itw1, F1 *w1, F1 *iw1, F2 *tw2, F2 *itw2, F2 *w2, F2 *iw2) {
    Tables *t = tables(n);
    if (!t) return -1;
    memcpy(tw1, t->tw1, sizeof(F1) * (n / 2)); memcpy(itw1, t->itw1, sizeof(F1) * (n / 2));
    memcpy(w1, t->w1, sizeof(F1) * n); memcpy(iw1, t->iw1, sizeof(F1) * n);
    memcpy(tw2, t->tw2, sizeof(F2) * (n / 2)); memcpy(itw2, t->itw2, sizeof(F2) * (n / 2));
    memcpy(w2, t->w2, sizeof(F2) * n); memcpy(iw2, t->iw2, sizeof(F2) * n);
    return 0;
}

/* ---- cpu.rs:49-83: radix-2 DIF (natural in, bit-reversed out) and DIT (reverse, unscaled) ---- */
static void dif1(F1 *a, size_t n, const F1 *tw) {
    size_t h = n / 2, s = 0;
    while (h >= 1) {
        for (size_t g = 0; g < n; g += 2 * h)
            for (size_t j = 0; j < h; j++) {
                F1 u = a[g + j], v = a[g + j + h];
                a[g + j] = f1_add(u, v);
                a[g + j + h] = f1_mul(f1_sub(u, v), tw[j << s]);
            }
        h /= 2; s++;
    }
}
static void dif2(F2 *a, size_t n, const F2 *tw) {
    size_t h = n / 2, s = 0;
    while (h >= 1) {
        for (size_t g = 0; g < n; g += 2 * h)
            for (size_t j = 0; j < h; j++) {
                F2 u = a[g + j], v = a[g + j + h];
                a[g + j] = f2_add(u, v);
                a[g + j + h] = f2_mul(f2_sub(u, v), tw[j << s]);
            }
        h /= 2; s++;
    }
}
static void dit1(F1 *a, size_t n, const F1 *itw) {
    size_t h = 1, s = (size_t)log2z(n);
    while (h < n) {
        s--;
        for (size_t g = 0; g < n; g += 2 * h)
            for (size_t j = 0; j < h; j++) {
                F1 u = a[g + j], v = f1_mul(a[g + j + h], itw[j << s]);
                a[g + j] = f1_add(u, v);
                a[g + j + h] = f1_sub(u, v);
            }
        h *= 2;
    }
}
static void dit2(F2 *a, size_t n, const F2 *itw) {
    size_t h = 1, s = (size_t)log2z(n);
    while (h < n) {
        s--;
        for (size_t g = 0; g < n; g += 2 * h)
            for (size_t j = 0; j < h; j++) {
                F2 u = a[g + j], v = f2_mul(a[g + j + h], itw[j << s]);
                a[g + j] = f2_add(u, v);
                a[g + j + h] = f2_sub(u, v);
            }
        h *= 2;
    }
}

/* cpu.rs:85-103 */
static void forward1(F1 *a1, F2 *a2, const Tables *t) {
    for (size_t j = 0; j < t->n; j++) { a1[j] = f1_mul(a1[j], t->w1[j]); a2[j] = f2_mul(a2[j], t->w2[j]); }
    dif1(a1, t->n, t->tw1);
    dif2(a2, t->n, t->tw2);
}
static void inverse1(F1 *a1, F2 *a2, const Tables *t) {
    dit1(a1, t->n, t->itw1);
    dit2(a2, t->n, t->itw2);
    for (size_t j = 0; j < t->n; j++) { a1[j] = f1_mul(a1[j], t->iw1[j]); a2[j] = f2_mul(a2[j], t->iw2[j]); }
}

/* cpu.rs:105-115: packs up to 2n real coefficients (c_j -> re, c_{j+n} -> im) and forward-transforms. */
static void forward_limbs(const uint32_t *c, size_t clen, F1 *a1, F2 *a2, const Tables *t) {
    size_t n = t->n;
    for (size_t j = 0; j < n; j++) {
        uint32_t re = j < clen ? c[j] : 0, im = j + n < clen ? c[j + n] : 0;
        a1[j] = f1_new(re % P1, im % P1);
        a2[j] = f2_new(re, im);
    }
    forward1(a1, a2, t);
}

/* cpu.rs:117-129: CRT and carry into 2n limbs; returns the carry out of the top. */
static u128 carry(const F1 *a1, const F2 *a2, size_t n, uint32_t *out, uint32_t inv) {
    u128 c = 0;
    for (size_t q = 0; q < 2 * n; q++) {
        size_t j = q % n;
        u128 v = q < n ? crt(a1[j].re, a2[j].re, inv) : crt(a1[j].im, a2[j].im, inv);
        c += v;
        out[q] = (uint32_t)c;
        c >>= 32;
    }
    return c;
}

/* cpu.rs:131-140 */
static void pointwise1(F1 *a1, F2 *a2, const F1 *b1, const F2 *b2, size_t n, uint32_t c) {
    for (size_t j = 0; j < n; j++) {
        a1[j] = f1_mul(a1[j], b1[j]);
        a2[j] = f2_mul(a2[j], b2[j]);
        if (c != 1) { a1[j] = f1_scale(a1[j], c); a2[j] = f2_scale(a2[j], c); }
    }
}

/* ---- cpu.rs:165-328: the wraparound ("half") path ---- */
typedef struct {
    Tables *tab;        /* tables at length h */
    size_t h;
    size_t *partner;    /* position of index (h - rev(p)) mod h */
    F1 *u1, *iu1;       /* Unpack: w^rev(p), w^-rev(p), w a primitive 2h-th root */
    F2 *u2, *iu2;
} Half;

static size_t rev_bits(size_t p, int bits) {
    size_t r = 0;
    for (int b = 0; b < bits; b++) r |= ((p >> b) & 1) << (bits - 1 - b);
    return r;
}

/* cpu.rs:172-202 */
static Half *half_new(Tables *tab) {
    Half *hf = calloc(1, sizeof *hf);
    size_t h = tab->n;
    int bits = log2z(h);
    hf->tab = tab; hf->h = h;
    hf->partner = malloc(sizeof(size_t) * h);
    for (size_t p = 0; p < h; p++) hf->partner[p] = rev_bits((h - rev_bits(p, bits)) % h, bits);
    int l2h = log2z(2 * h);
    F1 w1 = f1_pow(f1_sylow2(), 1ull << (32 - l2h)), wi1 = f1_inv(w1);
    F2 w2 = f2_pow(f2_sylow2(), 1ull << (62 - l2h)), wi2 = f2_inv(w2);
    hf->u1 = malloc(sizeof(F1) * h); hf->iu1 = malloc(sizeof(F1) * h);
    hf->u2 = malloc(sizeof(F2) * h); hf->iu2 = malloc(sizeof(F2) * h);
    for (size_t p = 0; p < h; p++) {
        size_t r = rev_bits(p, bits);
        hf->u1[p] = f1_pow(w1, r); hf->iu1[p] = f1_pow(wi1, r);
        hf->u2[p] = f2_pow(w2, r); hf->iu2[p] = f2_pow(wi2, r);
    }
    return hf;
}
static void half_free(Half *hf) {
    if (!hf) return;
    free(hf->partner); free(hf->u1); free(hf->iu1); free(hf->u2); free(hf->iu2); free(hf);
}

/* cpu.rs:212-219 */
static inline void half_spectrum1(F1 zk, F1 zj, F1 u, F1 *x, F1 *y) {
    F1 mi = f1_sub(f1_new(0, 0), f1_i());
    F1 e = f1_add(zk, f1_conj(zj));
    F1 wo = f1_mul(f1_mul(f1_sub(zk, f1_conj(zj)), mi), u);
    *x = f1_add(e, wo); *y = f1_sub(e, wo);
}
static inline void half_spectrum2(F2 zk, F2 zj, F2 u, F2 *x, F2 *y) {
    F2 mi = f2_sub(f2_new(0, 0), f2_i());
    F2 e = f2_add(zk, f2_conj(zj));
    F2 wo = f2_mul(f2_mul(f2_sub(zk, f2_conj(zj)), mi), u);
    *x = f2_add(e, wo); *y = f2_sub(e, wo);
}
/* cpu.rs:204-210 */
static inline F1 half_one1(F1 zk, F1 zj, F1 nx, F1 ny, F1 u, F1 iu) {
    F1 x, y; half_spectrum1(zk, zj, u, &x, &y);
    F1 px = f1_mul(x, nx), py = f1_mul(y, ny);
    return f1_add(f1_add(px, py), f1_mul(f1_mul(f1_sub(px, py), iu), f1_i()));
}
static inline F2 half_one2(F2 zk, F2 zj, F2 nx, F2 ny, F2 u, F2 iu) {
    F2 x, y; half_spectrum2(zk, zj, u, &x, &y);
    F2 px = f2_mul(x, nx), py = f2_mul(y, ny);
    return f2_add(f2_add(px, py), f2_mul(f2_mul(f2_sub(px, py), iu), f2_i()));
}
/* cpu.rs:221-237 */
static void half_pointwise1(F1 *z, const F1 *s, const Half *hf) {
    F1 x0 = f1_new(s[0].re, 0), y0 = f1_new(s[0].im, 0);
    for (size_t p = 0; p < hf->h; p++) {
        size_t q = hf->partner[p];
        if (q < p) continue;
        F1 zp = z[p], zq = z[q];
        F1 nx = p == 0 ? x0 : s[p], ny = p == 0 ? y0 : f1_conj(s[q]);
        z[p] = half_one1(zp, zq, nx, ny, hf->u1[p], hf->iu1[p]);
        if (q != p) z[q] = half_one1(zq, zp, s[q], f1_conj(s[p]), hf->u1[q], hf->iu1[q]);
    }
}
static void half_pointwise2(F2 *z, const F2 *s, const Half *hf) {
    F2 x0 = f2_new(s[0].re, 0), y0 = f2_new(s[0].im, 0);
    for (size_t p = 0; p < hf->h; p++) {
        size_t q = hf->partner[p];
        if (q < p) continue;
        F2 zp = z[p], zq = z[q];
        F2 nx = p == 0 ? x0 : s[p], ny = p == 0 ? y0 : f2_conj(s[q]);
        z[p] = half_one2(zp, zq, nx, ny, hf->u2[p], hf->iu2[p]);
        if (q != p) z[q] = half_one2(zq, zp, s[q], f2_conj(s[p]), hf->u2[q], hf->iu2[q]);
    }
}
/* cpu.rs:239-249 */
static void half_nhat1(F1 *z, const Half *hf) {
    size_t h = hf->h;
    F1 c = f1_inv(f1_from((uint32_t)(8 * h)));
    F1 *src = malloc(sizeof(F1) * h);
    memcpy(src, z, sizeof(F1) * h);
    for (size_t p = 0; p < h; p++) {
        F1 x, y; half_spectrum1(src[p], src[hf->partner[p]], hf->u1[p], &x, &y);
        z[p] = p == 0 ? f1_add(f1_mul(x, c), f1_mul(f1_mul(y, c), f1_i())) : f1_mul(x, c);
    }
    free(src);
}
static void half_nhat2(F2 *z, const Half *hf) {
    size_t h = hf->h;
    F2 c = f2_inv(f2_from((uint32_t)(8 * h)));
    F2 *src = malloc(sizeof(F2) * h);
    memcpy(src, z, sizeof(F2) * h);
    for (size_t p = 0; p < h; p++) {
        F2 x, y; half_spectrum2(src[p], src[hf->partner[p]], hf->u2[p], &x, &y);
        z[p] = p == 0 ? f2_add(f2_mul(x, c), f2_mul(f2_mul(y, c), f2_i())) : f2_mul(x, c);
    }
    free(src);
}
/* cpu.rs:286-295: packs k real coefficients as z_j = c_2j + i c_2j+1 and forward-transforms. */
static void half_forward(const uint32_t *c, F1 *a1, F2 *a2, const Half *hf) {
    for (size_t j = 0; j < hf->h; j++) {
        uint32_t re = c[2 * j], im = c[2 * j + 1];
        a1[j] = f1_new(re % P1, im % P1);
        a2[j] = f2_new(re, im);
    }
    dif1(a1, hf->h, hf->tab->tw1);
    dif2(a2, hf->h, hf->tab->tw2);
}
/* cpu.rs:251-259 */
static void half_nhat_of(const uint32_t *n, const Half *hf, F1 *a1, F2 *a2) {
    half_forward(n, a1, a2, hf);
    half_nhat1(a1, hf);
    half_nhat2(a2, hf);
}

/* cpu.rs:261-284: the device's form of the half pointwise step, A at p and B at h + p. */
int oc_half_factors(const uint32_t *n_limbs, size_t len, F1 *ab1, F2 *ab2) {
    size_t n = len / 2, h = n / 2;
    Tables *t = tables(h);
    if (!t || h < 2) return -1;
    Half *hf = half_new(t);
    F1 *s1 = malloc(sizeof(F1) * h);
    F2 *s2 = malloc(sizeof(F2) * h);
    half_nhat_of(n_limbs, hf, s1, s2);
    F1 i1 = f1_i(), one1 = f1_new(1, 0), mi1 = f1_sub(f1_new(0, 0), i1);
    F2 i2 = f2_i(), one2 = f2_new(1, 0), mi2 = f2_sub(f2_new(0, 0), i2);
    for (size_t p = 0; p < h; p++) {
        F1 nx1 = p == 0 ? f1_new(s1[0].re, 0) : s1[p], ny1 = p == 0 ? f1_new(s1[0].im, 0) : f1_conj(s1[hf->partner[p]]);
        F1 x1 = f1_mul(nx1, f1_add(one1, f1_mul(i1, hf->iu1[p])));
        F1 y1 = f1_mul(ny1, f1_sub(one1, f1_mul(i1, hf->iu1[p])));
        ab1[p] = f1_add(x1, y1);
        ab1[h + p] = f1_mul(f1_mul(f1_sub(x1, y1), mi1), hf->u1[p]);
        F2 nx2 = p == 0 ? f2_new(s2[0].re, 0) : s2[p], ny2 = p == 0 ? f2_new(s2[0].im, 0) : f2_conj(s2[hf->partner[p]]);
        F2 x2 = f2_mul(nx2, f2_add(one2, f2_mul(i2, hf->iu2[p])));
        F2 y2 = f2_mul(ny2, f2_sub(one2, f2_mul(i2, hf->iu2[p])));
        ab2[p] = f2_add(x2, y2);
        ab2[h + p] = f2_mul(f2_mul(f2_sub(x2, y2), mi2), hf->u2[p]);
    }
    free(s1); free(s2); half_free(hf);
    return 0;
}

/* cpu.rs:297-328: x = floor(T/R) + ((cyclic + T mod R) mod (R - 1)), end-around carry. */
static int wrap_combine(const F1 *a1, const F2 *a2, const uint32_t *t, uint32_t *x, size_t k, uint32_t inv) {
    u128 c = 0;
    for (size_t q = 0; q < k; q++) {
        F1 e1 = a1[q / 2]; F2 e2 = a2[q / 2];
        c += (q % 2 == 0) ? crt(e1.re, e2.re, inv) : crt(e1.im, e2.im, inv);
        c += t[q];
        x[q] = (uint32_t)c;
        c >>= 32;
    }
    while (c != 0) {
        for (size_t q = 0; q < k; q++) {
            c += x[q];
            x[q] = (uint32_t)c;
            c >>= 32;
            if (c == 0) break;
        }
    }
    for (size_t q = 0; q < k; q++) {
        c += (u128)x[q] + t[k + q];
        x[q] = (uint32_t)c;
        c >>= 32;
    }
    return c == 0 ? 0 : -1;
}

/* ---- cpu.rs:409-578: the Backend ---- */
typedef struct {
    F1 *nhat1, *nphat1;
    F2 *nhat2, *nphat2;
    uint32_t *two_n, *x, *exp;
    size_t nexp, nbits, pos;
    int err;
    /* Gmp backend fields (gmp.rs:29-41), as limb strings */
} Slot;

/* mpz_t with the documented GMP layout (gmp.h: __mpz_struct). */
typedef struct { int alloc; int size; void *d; } mpz_s;
typedef mpz_s mpz_t[1];
void __gmpz_init(mpz_s *);
void __gmpz_clear(mpz_s *);
void __gmpz_import(mpz_s *, size_t, int, size_t, int, size_t, const void *);
void *__gmpz_export(void *, size_t *, int, size_t, int, size_t, const mpz_s *);
void __gmpz_mul(mpz_s *, const mpz_s *, const mpz_s *);
void __gmpz_mul_ui(mpz_s *, const mpz_s *, unsigned long);
void __gmpz_add(mpz_s *, const mpz_s *, const mpz_s *);
void __gmpz_fdiv_r_2exp(mpz_s *, const mpz_s *, unsigned long);
void __gmpz_fdiv_q_2exp(mpz_s *, const mpz_s *, unsigned long);
void __gmpz_set(mpz_s *, const mpz_s *);
int __gmpz_cmp(const mpz_s *, const mpz_s *);
size_t __gmpz_sizeinbase(const mpz_s *, int);

typedef struct {
    mpz_t n, nprime, two_n, x, t, m;
} GSlot;

struct oc_state {
    int mode;       /* OC_PLAIN, OC_FULL_K, OC_WRAP, or 3 = Gmp */
    size_t k, slots;
    uint32_t base;
    Tables *tab;
    Half *half;
    Slot *s;
    GSlot *g;
};

typedef struct { F1 *a1; F2 *a2; uint32_t *t, *s, *m; } Scratch;

static void scratch_init(Scratch *sc, size_t n) {
    sc->a1 = malloc(sizeof(F1) * n); sc->a2 = malloc(sizeof(F2) * n);
    sc->t = calloc(2 * n, 4); sc->s = calloc(2 * n, 4); sc->m = calloc(2 * n, 4);
}
static void scratch_free(Scratch *sc) { free(sc->a1); free(sc->a2); free(sc->t); free(sc->s); free(sc->m); }

/* cpu.rs:452-484: from T in sc->t (2n limbs), x = T R^-1 (lazy, in [0, 2N)). */
static int redc(const oc_state *st, const Slot *s, Scratch *sc, uint32_t *x, uint32_t inv) {
    size_t k = st->k, n = st->tab->n;
    int flag = 0;
    for (size_t j = 0; j < k; j++) flag |= sc->t[j] != 0;
    forward_limbs(sc->t, k, sc->a1, sc->a2, st->tab);
    pointwise1(sc->a1, sc->a2, s->nphat1, s->nphat2, n, 1);
    inverse1(sc->a1, sc->a2, st->tab);
    carry(sc->a1, sc->a2, n, sc->s, inv);
    memcpy(sc->m, sc->s, 4 * k);
    if (st->half) {
        const Half *hf = st->half;
        half_forward(sc->m, sc->a1, sc->a2, hf);
        half_pointwise1(sc->a1, s->nhat1, hf);
        half_pointwise2(sc->a2, s->nhat2, hf);
        dit1(sc->a1, hf->h, hf->tab->itw1);
        dit2(sc->a2, hf->h, hf->tab->itw2);
        return wrap_combine(sc->a1, sc->a2, sc->t, x, k, inv);
    }
    forward_limbs(sc->m, k, sc->a1, sc->a2, st->tab);
    pointwise1(sc->a1, sc->a2, s->nhat1, s->nhat2, n, 1);
    inverse1(sc->a1, sc->a2, st->tab);
    u128 top = carry(sc->a1, sc->a2, n, sc->s, inv);
    uint64_t c = (uint64_t)flag;
    for (size_t j = 0; j < k; j++) {
        c += (uint64_t)sc->t[k + j] + sc->s[k + j];
        x[j] = (uint32_t)c;
        c >>= 32;
    }
    return (top == 0 && c == 0) ? 0 : -1;
}

/* cpu.rs:486-497 */
static int square_step(const oc_state *st, Slot *s, Scratch *sc, uint32_t c, uint32_t inv) {
    size_t n = st->tab->n;
    forward_limbs(s->x, st->k, sc->a1, sc->a2, st->tab);
    for (size_t j = 0; j < n; j++) {
        sc->a1[j] = f1_scale(f1_mul(sc->a1[j], sc->a1[j]), c);
        sc->a2[j] = f2_scale(f2_mul(sc->a2[j], sc->a2[j]), c);
    }
    inverse1(sc->a1, sc->a2, st->tab);
    u128 top = carry(sc->a1, sc->a2, n, sc->t, inv);
    return redc(st, s, sc, s->x, inv) | (top != 0 ? -1 : 0);
}

/* gmp.rs:43-60: m = (T mod R) N' mod R, x = (T + m N) / R. */
static void g_redc(GSlot *g, unsigned long rbits) {
    __gmpz_fdiv_r_2exp(g->m, g->t, rbits);
    __gmpz_mul(g->m, g->m, g->nprime);
    __gmpz_fdiv_r_2exp(g->m, g->m, rbits);
    __gmpz_mul(g->m, g->m, g->n);
    __gmpz_add(g->t, g->t, g->m);
    __gmpz_fdiv_q_2exp(g->t, g->t, rbits);
    __gmpz_set(g->x, g->t);
}
static void g_square_step(GSlot *g, uint32_t c, unsigned long rbits) {
    __gmpz_mul(g->t, g->x, g->x);
    __gmpz_mul_ui(g->t, g->t, c);
    g_redc(g, rbits);
}

static void limbs_to_mpz(mpz_s *z, const uint32_t *l, size_t k) { __gmpz_import(z, k, -1, 4, 0, 0, l); }
static void mpz_to_limbs(uint32_t *l, size_t k, const mpz_s *z) {
    memset(l, 0, 4 * k);
    size_t cnt = (__gmpz_sizeinbase(z, 2) + 31) / 32;
    if (z->size == 0) return;
    if (cnt > k) { memset(l, 0xff, 4 * k); return; }
    __gmpz_export(l, &cnt, -1, 4, 0, 0, z);
}

static oc_state *state_new(int mode, size_t k, size_t len, uint32_t base, size_t slots) {
    if (slots == 0 || len < 8 || (len & (len - 1)) || k == 0 || k > len / 2) return NULL;
    oc_state *st = calloc(1, sizeof *st);
    st->mode = mode; st->k = k; st->slots = slots; st->base = base;
    return st;
}

/* cpu.rs:502-533 */
oc_state *oc_create(int mode, size_t k, size_t len, uint32_t base, size_t slots, const uint32_t *n,
                    const uint32_t *nprime, const uint32_t *two_n) {
    oc_state *st = state_new(mode, k, len, base, slots);
    if (!st) return NULL;
    st->tab = tables(len / 2);
    size_t nn = st->tab->n;
    if (mode == OC_WRAP) {
        if (k != nn) { free(st); return NULL; }   /* "wraparound needs k = L/2" */
        st->half = half_new(tables(len / 4));
    }
    st->s = calloc(slots, sizeof(Slot));
    Scratch sc; scratch_init(&sc, nn);
    for (size_t i = 0; i < slots; i++) {
        Slot *s = &st->s[i];
        s->nhat1 = malloc(sizeof(F1) * nn); s->nhat2 = malloc(sizeof(F2) * nn);
        s->nphat1 = malloc(sizeof(F1) * nn); s->nphat2 = malloc(sizeof(F2) * nn);
        if (st->half) half_nhat_of(n + i * k, st->half, s->nhat1, s->nhat2);
        else forward_limbs(n + i * k, k, s->nhat1, s->nhat2, st->tab);
        forward_limbs(nprime + i * k, k, s->nphat1, s->nphat2, st->tab);
        s->two_n = malloc(4 * k); memcpy(s->two_n, two_n + i * k, 4 * k);
        s->x = calloc(k, 4);
    }
    scratch_free(&sc);
    return st;
}

/* gmp.rs:72-87 */
oc_state *og_create(size_t k, size_t len, uint32_t base, size_t slots, const uint32_t *n,
                    const uint32_t *nprime, const uint32_t *two_n) {
    oc_state *st = state_new(3, k, len, base, slots);
    if (!st) return NULL;
    st->s = calloc(slots, sizeof(Slot));
    st->g = calloc(slots, sizeof(GSlot));
    for (size_t i = 0; i < slots; i++) {
        GSlot *g = &st->g[i];
        __gmpz_init(g->n); __gmpz_init(g->nprime); __gmpz_init(g->two_n);
        __gmpz_init(g->x); __gmpz_init(g->t); __gmpz_init(g->m);
        limbs_to_mpz(g->n, n + i * k, k);
        limbs_to_mpz(g->nprime, nprime + i * k, k);
        limbs_to_mpz(g->two_n, two_n + i * k, k);
    }
    return st;
}

void oc_load(oc_state *st, size_t i, const uint32_t *limbs) {
    if (st->g) limbs_to_mpz(st->g[i].x, limbs, st->k);
    else memcpy(st->s[i].x, limbs, 4 * st->k);
}

void oc_set_exponent(oc_state *st, size_t i, const uint32_t *words, size_t nwords, size_t nbits) {
    Slot *s = &st->s[i];
    free(s->exp);
    s->exp = malloc(4 * (nwords ? nwords : 1));
    if (nwords) memcpy(s->exp, words, 4 * nwords);
    s->nexp = nwords; s->nbits = nbits; s->pos = 0;
}

typedef struct { oc_state *st; size_t bits, first, step; } RunArg;

/* cpu.rs:543-556 and gmp.rs:97-109: per slot, up to `bits` steps x <- x^2 c^bit R^-1. */
static void *run_worker(void *p) {
    RunArg *a = p;
    oc_state *st = a->st;
    uint32_t inv = oc_crt_inv();
    Scratch sc;
    int gm = st->g != NULL;
    if (!gm) scratch_init(&sc, st->tab->n);
    for (size_t i = a->first; i < st->slots; i += a->step) {
        Slot *s = &st->s[i];
        for (size_t b = 0; b < a->bits; b++) {
            if (s->pos >= s->nbits) break;
            uint32_t bit = (s->exp[s->pos / 32] >> (31 - s->pos % 32)) & 1;
            uint32_t c = bit ? st->base : 1;
            if (gm) g_square_step(&st->g[i], c, 32ul * st->k);
            else if (square_step(st, s, &sc, c, inv)) s->err = 1;
            s->pos++;
        }
    }
    if (!gm) scratch_free(&sc);
    return NULL;
}

void oc_run(oc_state *st, size_t bits, int threads) {
    if (threads <= 0) threads = (int)sysconf(_SC_NPROCESSORS_ONLN);
    if ((size_t)threads > st->slots) threads = (int)st->slots;
    if (threads < 1) threads = 1;
    pthread_t *th = malloc(sizeof(pthread_t) * threads);
    RunArg *args = malloc(sizeof(RunArg) * threads);
    for (int t = 0; t < threads; t++) {
        args[t].st = st; args[t].bits = bits; args[t].first = (size_t)t; args[t].step = (size_t)threads;
        if (threads == 1) run_worker(&args[t]);
        else pthread_create(&th[t], NULL, run_worker, &args[t]);
    }
    if (threads > 1) for (int t = 0; t < threads; t++) pthread_join(th[t], NULL);
    free(th); free(args);
}

/* cpu.rs:558-571 and gmp.rs:110-115 */
void oc_mul(oc_state *st, size_t out, size_t a, size_t b) {
    if (st->g) {
        GSlot *g = &st->g[out];
        mpz_t t; __gmpz_init(t);
        __gmpz_mul(t, st->g[a].x, st->g[b].x);
        __gmpz_set(g->t, t);
        __gmpz_clear(t);
        g_redc(g, 32ul * st->k);
        return;
    }
    size_t n = st->tab->n;
    uint32_t inv = oc_crt_inv();
    Scratch sc; scratch_init(&sc, n);
    F1 *b1 = malloc(sizeof(F1) * n); F2 *b2 = malloc(sizeof(F2) * n);
    forward_limbs(st->s[b].x, st->k, b1, b2, st->tab);
    forward_limbs(st->s[a].x, st->k, sc.a1, sc.a2, st->tab);
    pointwise1(sc.a1, sc.a2, b1, b2, n, 1);
    inverse1(sc.a1, sc.a2, st->tab);
    u128 top = carry(sc.a1, sc.a2, n, sc.t, inv);
    uint32_t *x = calloc(st->k, 4);
    if (redc(st, &st->s[out], &sc, x, inv) || top) st->s[out].err = 1;
    memcpy(st->s[out].x, x, 4 * st->k);
    free(x); free(b1); free(b2); scratch_free(&sc);
}

void oc_read(const oc_state *st, size_t i, uint32_t *limbs) {
    if (st->g) mpz_to_limbs(limbs, st->k, st->g[i].x);
    else memcpy(limbs, st->s[i].x, 4 * st->k);
}

size_t oc_remaining(const oc_state *st, size_t i) { return st->s[i].nbits - st->s[i].pos; }

void oc_destroy(oc_state *st) {
    if (!st) return;
    for (size_t i = 0; i < st->slots; i++) {
        Slot *s = &st->s[i];
        free(s->nhat1); free(s->nhat2); free(s->nphat1); free(s->nphat2);
        free(s->two_n); free(s->x); free(s->exp);
        if (st->g) {
            GSlot *g = &st->g[i];
            __gmpz_clear(g->n); __gmpz_clear(g->nprime); __gmpz_clear(g->two_n);
            __gmpz_clear(g->x); __gmpz_clear(g->t); __gmpz_clear(g->m);
        }
    }
    free(st->s); free(st->g);
    half_free(st->half);
    free(st);
}

/* ---- cpu.rs:349-407: the Transform trait on host arrays ---- */
void oc_upload(const uint32_t *coeffs, size_t len, size_t count, F1 *f1, F2 *f2) {
    size_t n = len / 2;
    for (size_t v = 0; v < count; v++)
        for (size_t j = 0; j < n; j++) {
            const uint32_t *c = coeffs + v * len;
            f1[v * n + j] = f1_new(c[j] % P1, c[j + n] % P1);
            f2[v * n + j] = f2_new(c[j], c[j + n]);
        }
}
void oc_download(const F1 *f1, const F2 *f2, size_t len, size_t count, uint64_t *out) {
    size_t n = len / 2;
    uint32_t inv = oc_crt_inv();
    for (size_t v = 0; v < count; v++)
        for (size_t j = 0; j < n; j++) {
            u128 a = crt(f1[v * n + j].re, f2[v * n + j].re, inv);
            u128 b = crt(f1[v * n + j].im, f2[v * n + j].im, inv);
            out[2 * (v * len + j)] = (uint64_t)a; out[2 * (v * len + j) + 1] = (uint64_t)(a >> 64);
            out[2 * (v * len + j + n)] = (uint64_t)b; out[2 * (v * len + j + n) + 1] = (uint64_t)(b >> 64);
        }
}
void oc_forward(F1 *f1, F2 *f2, size_t len, size_t count) {
    Tables *t = tables(len / 2);
    for (size_t v = 0; v < count; v++) forward1(f1 + v * t->n, f2 + v * t->n, t);
}
void oc_inverse(F1 *f1, F2 *f2, size_t len, size_t count) {
    Tables *t = tables(len / 2);
    for (size_t v = 0; v < count; v++) inverse1(f1 + v * t->n, f2 + v * t->n, t);
}
void oc_pointwise(F1 *o1, F2 *o2, const F1 *a1, const F2 *a2, const F1 *b1, const F2 *b2,
                  const uint32_t *scales, size_t len, size_t count) {
    size_t n = len / 2;
    for (size_t v = 0; v < count; v++) {
        memcpy(o1 + v * n, a1 + v * n, sizeof(F1) * n);
        memcpy(o2 + v * n, a2 + v * n, sizeof(F2) * n);
        pointwise1(o1 + v * n, o2 + v * n, b1 + v * n, b2 + v * n, n, scales ? scales[v] : 1);
    }
}
