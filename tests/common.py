"""Backend-generic test cases, restating montmul/tests/common/mod.rs; every check is against GMP.

Each case takes a backend factory (`make()` returns a fresh backend object) and drives it
through `ModBatch`, exactly as the reference's generic cases drive any `Backend`.
"""
from __future__ import annotations

import numpy as np

from montmul_b200 import ModBatch, MontMulError, Params, fermat, to_limbs
from montmul_b200.gmp import RandState, invert, powm

# OEIS A092835 lists n - 1 for prime T(n) (A000073 indexing): 3, 5, 6, 10, 86, 97, 214, 801,
# 4201, 18698, 96878. T(4) = 2 is even, so these are the odd ones below 1000 bits
# (tests/common/mod.rs:284-288).
A092835_SMALL = [6, 7, 11, 87, 98, 215, 802]
A092835_LARGE = [4202, 18699, 96879]
COMPOSITE_NS = [8, 9, 10, 12, 13, 20, 86, 88, 803]   # tests/cpu.rs:61-63


def tribonacci(n: int) -> int:
    """T(n) with T(0) = T(1) = 0, T(2) = 1 (montmul/src/seq.rs:6-15)."""
    a, b, c = 0, 0, 1
    for _ in range(n):
        a, b, c = b, c, a + b + c
    return a


def rand_odd(rng: RandState, bits: int) -> int:
    """tests/common/mod.rs:10-15"""
    n = rng.random_bits(bits)
    return n | (1 << (bits - 1)) | 1


def expected(x: int, c: int, n: int, k: int) -> int:
    """x^2 c R^-1 mod N (tests/common/mod.rs:17-21)."""
    rinv = invert(1 << (32 * k), n)
    return x * x * c * rinv % n


def random_modmul(make, bits, cases, seed, base):
    """tests/common/mod.rs:93-120"""
    rng = RandState(seed)
    moduli = [rand_odd(rng, bits) for _ in range(cases)]
    batch = ModBatch(make(), moduli, base)
    k = batch.params.k
    xs = [rng.random_below(2 * n) for n in moduli]
    for i, x in enumerate(xs):
        batch.load_raw(i, x)
        batch.set_exponent(i, 2)
    prev = list(xs)
    for c in (base, 1):
        batch.run(1)
        for i in range(cases):
            n = moduli[i]
            raw = batch.read_raw(i)
            assert raw < 2 * n, f"lazy range, bits {bits} slot {i}"
            assert raw % n == expected(prev[i], c, n, k), f"bits {bits} slot {i} c {c}"
            prev[i] = raw


def edge_sizes(max_log_len: int):
    sizes = [28, 60, 124, 252, 1020, 4092, 32764]
    for m in range(3, max_log_len + 1):
        kmax = (1 << m) // 2
        sizes.append(32 * kmax - 4)
        sizes.append(32 * (kmax // 2) - 3)
    return sizes


def edges(make, base, max_log_len=16):
    """x = 0, N, 2N - 1 and N = 2^b - 1 at the top and bottom of each length's bucket
    (tests/common/mod.rs:122-159)."""
    rng = RandState()
    lengths = make().supported_lengths()
    for bits in edge_sizes(max_log_len):
        if Params.for_bits(bits, [1 << e for e in range(3, 25)]).len > max(lengths):
            continue
        moduli = [rand_odd(rng, bits), (1 << bits) - 1]
        batch = ModBatch(make(), moduli, base)
        k = batch.params.k
        for which in range(3):
            vals = [0 if which == 0 else (n if which == 1 else 2 * n - 1) for n in moduli]
            for i, x in enumerate(vals):
                batch.load_raw(i, x)
                batch.set_exponent(i, 1)
            batch.run(1)
            for i, n in enumerate(moduli):
                raw = batch.read_raw(i)
                assert raw < 2 * n, f"lazy range bits {bits}"
                assert raw % n == expected(vals[i], base, n, k), f"bits {bits} case {which}"


def batch_independence(make, bits, sizes):
    """tests/common/mod.rs:161-188"""
    rng = RandState()
    target = rand_odd(rng, bits)
    e = rng.random_bits(64) | 1
    reference = None
    for size in sizes:
        moduli = [rand_odd(rng, bits) for _ in range(size)]
        pos = min(size * 5 // 7, size - 1)
        for p in (0, pos, size - 1):
            moduli[p] = target
        batch = ModBatch(make(), moduli, 3)
        batch.load_all([1] * size)
        batch.set_exponents([e] * size)
        batch.run(1000)
        for p in (0, pos, size - 1):
            raw = to_limbs(batch.read_raw(p), batch.params.k)
            if reference is None:
                reference = raw
            else:
                assert np.array_equal(raw, reference), f"size {size} slot {p}"
            assert batch.read(p) == powm(3, e, target)


def powmod_and_mul(make, bits, count):
    """tests/common/mod.rs:190-220"""
    rng = RandState()
    moduli = [rand_odd(rng, bits) for _ in range(count)]
    batch = ModBatch(make(), moduli, 3)
    exps = []
    for i in range(count):
        e = rng.random_bits(32 + i * 7) | 1
        batch.load(i, 1)
        batch.set_exponent(i, e)
        exps.append(e)
    while any(batch.remaining(i) > 0 for i in range(count)):
        batch.run(37)
    for i, n in enumerate(moduli):
        assert batch.read(i) == powm(3, exps[i], n), f"slot {i}"
    n = rand_odd(rng, bits)
    batch = ModBatch(make(), [n, n, n], 3)
    a = rng.random_below(n)
    b = rng.random_below(n)
    batch.load(0, a)
    batch.load(1, b)
    batch.mul(2, 0, 1)
    assert batch.read(2) == a * b % n
    batch.mul(0, 0, 0)
    assert batch.read(0) == a * a % n


def rand_exponent(rng, bits):
    return rng.random_bits(bits) | (1 << (bits - 1))


def same_raw(make_a, make_b, bits, slots, steps):
    """Two backends on the same moduli end with equal raw limbs (tests/common/mod.rs:229-247)."""
    rng = RandState()
    moduli = [rand_odd(rng, bits) for _ in range(slots)]
    exps = [rand_exponent(rng, steps) for _ in range(slots)]
    x = ModBatch(make_a(), moduli, 3)
    y = ModBatch(make_b(), moduli, 3)
    for b in (x, y):
        b.load_all([1] * slots)
        b.set_exponents(exps)
        b.run(steps)
    for i in range(slots):
        assert x.read_raw(i) == y.read_raw(i), f"bits {bits} slot {i}"
    return x, y


def long_run(make, bits, slots, ebits):
    """tests/common/mod.rs:249-264"""
    rng = RandState()
    moduli = [rand_odd(rng, bits) for _ in range(slots)]
    exps = [rand_exponent(rng, ebits) for _ in range(slots)]
    batch = ModBatch(make(), moduli, 3)
    batch.load_all([1] * slots)
    batch.set_exponents(exps)
    batch.run(ebits)
    for i, n in enumerate(moduli):
        assert batch.remaining(i) == 0, f"slot {i}"
        assert batch.read(i) == powm(3, exps[i], n), f"bits {bits} slot {i}"


def end_to_end(make, ns, chunk=500):
    """Fermat base 3 on T(n) against pow_mod, grouped by length (tests/common/mod.rs:266-282)."""
    moduli = [t for t in (tribonacci(n) for n in ns) if t % 2 == 1 and t > 3]
    lengths = make().supported_lengths()
    groups = {}
    for m in moduli:
        groups.setdefault(Params.for_bits(m.bit_length(), lengths).len, []).append(m)
    for ms in groups.values():
        got = fermat(make(), ms, 3, chunk)
        for m, g in zip(ms, got):
            assert g == (powm(3, m - 1, m) == 1), f"T with {m.bit_length()} bits"


def known_prps(make, prime_ns, composite_ns):
    """tests/common/mod.rs:290-300"""
    for n, want in [(n, True) for n in prime_ns] + [(n, False) for n in composite_ns]:
        t = tribonacci(n)
        if t % 2 == 0:
            continue
        got = fermat(make(), [t], 3, 1 << 20)
        assert got[0] == want, f"T({n})"


def api_contract(make):
    """Rejections, parameter rules, tiny moduli, chunked runs, frozen slots, re-arming
    (tests/common/mod.rs:302-374)."""
    import pytest
    lengths = make().supported_lengths()
    assert all(l & (l - 1) == 0 for l in lengths)
    for moduli, base, what in [([], 3, "empty"), ([10], 3, "even"), ([1], 3, "one"), ([-7], 3, "negative"),
                               ([11], 5, "base"), ([11], 0, "base 0"), ([101, (1 << 5000) + 1], 3, "mixed")]:
        with pytest.raises(MontMulError):
            ModBatch(make(), moduli, base)
    for bits in (2, 28, 29, 60, 61, 1000, 87_914):
        p = Params.for_bits(bits, lengths)
        assert p.k * 32 >= bits + 4 and (p.k - 1) * 32 < bits + 4
        assert p.len >= 2 * p.k and (p.len == lengths[0] or p.len // 2 < 2 * p.k)
    if make().coefficient_bound() < (1 << 128) - 1:
        with pytest.raises(MontMulError):
            Params(1 << 30, 1 << 31).check_exact(4, make().coefficient_bound())
    rng = RandState()
    for n in (3, 5, 7, 9, 15, 101, 65_537, 4_294_967_291, 0xFFFFFFFF):
        b = ModBatch(make(), [n], 3)
        for x in (0, 1, n, n * 5 + 2, -4):
            b.load(0, x)
            assert b.read(0) == x % n, f"read after load, n {n}"
            assert b.is_one(0) == (x % n == 1), f"is_one, n {n}"
            e = rng.random_bits(40) + 1
            b.load(0, x)
            b.set_exponent(0, e)
            b.run(1 << 20)
            assert b.remaining(0) == 0
            sq = 1 << e.bit_length()
            want = powm(x % n, sq, n) * powm(3, e, n) % n
            assert b.read(0) == want, f"pow, n {n}"
    moduli = [rand_odd(rng, 777) for _ in range(5)]
    exps = [rng.random_bits(10 + 60 * i) | 1 for i in range(5)]
    a = ModBatch(make(), moduli, 3)
    b = ModBatch(make(), moduli, 3)
    for i in range(5):
        for m in (a, b):
            m.load(i, 1)
            m.set_exponent(i, exps[i])
    a.run(0)
    assert a.remaining(4) == exps[4].bit_length()
    a.run(1000)
    for chunk in (1, 2, 3, 5, 8, 13, 21, 34, 55, 89, 144, 1000):
        b.run(chunk)
    for i in range(5):
        assert a.read(i) == powm(3, exps[i], moduli[i])
        assert a.read_raw(i) == b.read_raw(i), f"chunked run slot {i}"
    a.run(100)
    assert a.read(0) == powm(3, exps[0], moduli[0]), "frozen after finish"
    a.load(0, 2)
    a.set_exponent(0, 5)
    a.run(10)
    assert a.read(0) == 256 * 243 % moduli[0]


def carry_stress(make, max_len):
    """x = 2N - 1 with N = 2^b - 1 and N = 2^b - 2^(b/2) + 1, 32 steps, every length
    (tests/common/mod.rs:376-398)."""
    for length in [l for l in make().supported_lengths() if 8 <= l <= max_len]:
        bits = 32 * (length // 2) - 4
        n1 = (1 << bits) - 1
        n2 = (1 << bits) - (1 << (bits // 2)) + 1
        b = ModBatch(make(), [n1, n2], 3)
        e = 0xFFFFFFFF
        for i, m in enumerate((n1, n2)):
            b.load_raw(i, 2 * m - 1)
            b.set_exponent(i, e)
        b.run(32)
        k = b.params.k
        for i, m in enumerate((n1, n2)):
            rinv = invert(1 << (32 * k), m)
            x = (m - rinv) % m
            want = powm(x, 1 << 32, m) * powm(3, e, m) % m
            assert b.read(i) == want, f"len {length} slot {i}"
