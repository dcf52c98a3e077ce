/* TEST INFRASTRUCTURE ONLY — the CPU oracle for the MontMul hot path.
 *
 * A plain-C restatement of the reference's semantics authority, the `Cpu` backend
 * (montmul/src/cpu.rs) with its field arithmetic (montmul/src/field.rs), and of the `Gmp`
 * backend's REDC (montmul/src/gmp.rs:45-60) over libgmp's public API. Only the tests, the
 * smoke check and the bench's CPU-baseline leg may load this library; the product never does.
 *
 * Parity pin: the oracle is checked against the reference's own known answers (the
 * `exactness` coefficient formula, tests/common/mod.rs:46-51; the Sylow orders and CRT round
 * trip, field.rs:297-317; the tribonacci PRP verdicts of tests/common/mod.rs:284-288 and
 * tests/cpu.rs:61-63) and against GMP's mpz_powm and Python integers.
 */
#ifndef MONTMUL_ORACLE_H
#define MONTMUL_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Field elements with the reference's layouts (field.rs:74-86). */
typedef struct { uint32_t re, im; } oc_f1;
typedef struct { uint64_t re, im; } oc_f2;

/* Backend modes of `Cpu` (cpu.rs:16-36). */
enum { OC_PLAIN = 0, OC_FULL_K = 1, OC_WRAP = 2 };

typedef struct oc_state oc_state;

/* Field-level checks (field.rs:111-120, 283-294). */
void oc_sylow2_f1(uint32_t out[2]);
void oc_sylow2_f2(uint64_t out[2]);
void oc_pow_f1(const uint32_t a[2], uint64_t e, uint32_t out[2]);
void oc_pow_f2(const uint64_t a[2], uint64_t e, uint64_t out[2]);
uint32_t oc_crt_inv(void);
/* CRT value as two u64 halves (lo, hi). */
void oc_crt(uint32_t c1, uint64_t c2, uint64_t out[2]);

/* FieldTables::new(n) for both fields (field.rs:237-266): tw, itw (n/2 each), w, iw (n each). */
int oc_tables(size_t n, oc_f1 *tw1, oc_f1 *itw1, oc_f1 *w1, oc_f1 *iw1, oc_f2 *tw2, oc_f2 *itw2,
              oc_f2 *w2, oc_f2 *iw2);

/* Transform trait of `Cpu` (cpu.rs:349-407), `count` vectors of length `len` (n = len/2 elements). */
void oc_upload(const uint32_t *coeffs, size_t len, size_t count, oc_f1 *f1, oc_f2 *f2);
void oc_download(const oc_f1 *f1, const oc_f2 *f2, size_t len, size_t count, uint64_t *out /* 2 u64 per coeff */);
void oc_forward(oc_f1 *f1, oc_f2 *f2, size_t len, size_t count);
void oc_inverse(oc_f1 *f1, oc_f2 *f2, size_t len, size_t count);
void oc_pointwise(oc_f1 *o1, oc_f2 *o2, const oc_f1 *a1, const oc_f2 *a2, const oc_f1 *b1,
                  const oc_f2 *b2, const uint32_t *scales /* may be NULL */, size_t len, size_t count);

/* Wraparound-path factors A|B of one modulus (cpu.rs:265-284): n elements per field, from k = n
 * limbs of N. Used to pin the device's own set-up of the same factors. */
int oc_half_factors(const uint32_t *n_limbs, size_t len, oc_f1 *ab1, oc_f2 *ab2);

/* Backend trait (transform.rs:61-77) of `Cpu` (cpu.rs:499-578) and of `Gmp` (gmp.rs:69-122).
 * `n`, `nprime`, `two_n`: slots × k limbs, row-major. Returns NULL on a bad setup. */
oc_state *oc_create(int mode, size_t k, size_t len, uint32_t base, size_t slots,
                    const uint32_t *n, const uint32_t *nprime, const uint32_t *two_n);
oc_state *og_create(size_t k, size_t len, uint32_t base, size_t slots, const uint32_t *n,
                    const uint32_t *nprime, const uint32_t *two_n);
void oc_load(oc_state *st, size_t i, const uint32_t *limbs);
void oc_set_exponent(oc_state *st, size_t i, const uint32_t *words, size_t nwords, size_t nbits);
/* Runs up to `bits` steps on every slot over `threads` host threads (0 = one per core). */
void oc_run(oc_state *st, size_t bits, int threads);
void oc_mul(oc_state *st, size_t out, size_t a, size_t b);
void oc_read(const oc_state *st, size_t i, uint32_t *limbs);
size_t oc_remaining(const oc_state *st, size_t i);
void oc_destroy(oc_state *st);

#ifdef __cplusplus
}
#endif
#endif
