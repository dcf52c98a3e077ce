"""Pins the CPU oracle (a C restatement of the reference's Cpu and Gmp backends) against the
reference's own known answers and against GMP / Python integers. CPU only."""
import numpy as np
import pytest

import common
from montmul_b200 import ModBatch, MontMulError, fermat
from montmul_b200.gmp import RandState, powm


@pytest.fixture(scope="module")
def o(oracle):
    return oracle


# ---- field.rs:296-317 ----

def test_sylow_orders(o):
    g1 = o.sylow2_f1()
    assert o.pow_f1(g1, 1 << 32) == (1, 0)
    assert o.pow_f1(g1, 1 << 31) != (1, 0)
    g2 = o.sylow2_f2()
    assert o.pow_f2(g2, 1 << 62) == (1, 0)
    assert o.pow_f2(g2, 1 << 61) != (1, 0)


def test_crt_roundtrip(o):
    for c in (0, 1, o.Q - 1, o.Q // 3, 123456789012345678901234567 % o.Q):
        assert o.crt(c % o.P1, c % o.P2) == c


def test_fixed_roots(o):
    """The device butterflies assume omega_n^(n/4) = i and omega_n^(n/8) = (1 + i) 2^s."""
    for n in (8, 64, 4096, 1 << 16):
        t = o.tables(n)
        assert tuple(t["tw1"][n // 4]) == (0, 1) and tuple(t["tw2"][n // 4]) == (0, 1)
        if n >= 16:
            assert tuple(t["tw1"][n // 8]) == (1 << 15, 1 << 15)
            assert tuple(t["tw2"][n // 8]) == (1 << 30, 1 << 30)


# ---- tests/common/mod.rs:23-53: exactness of the transform at the coefficient bound ----

@pytest.mark.parametrize("length", [1 << e for e in range(3, 13)])
def test_exactness(o, length):
    k, c = length // 2, 4
    coeffs = np.zeros(length, np.uint32)
    coeffs[:k] = 0xFFFFFFFF
    x = o.upload(coeffs, length, 1)
    o.forward(*x, length, 1)
    out = o.pointwise(x, x, [c], length, 1)
    o.inverse(*out, length, 1)
    got = o.download(*out, length, 1)
    a = (1 << (32 * k)) - 1
    assert sum(v << (32 * q) for q, v in enumerate(got)) == a * a * c
    sq = (1 << 32) - 1
    for q in range(length):
        cnt = q + 1 if q < k else (2 * k - 1 - q if q < 2 * k - 1 else 0)
        assert got[q] == c * sq * sq * cnt, f"len {length} coeff {q}"


def test_transform_batched(o):
    """tests/common/mod.rs:55-91: three vectors, scales [1, 3, 4] then none."""
    rng = RandState()
    for length in [1 << e for e in range(3, 11)]:
        k, count = length // 2, 3
        coeffs = [np.zeros(length * count, np.uint32) for _ in range(2)]
        for c in coeffs:
            for v in range(count):
                for q in range(k):
                    c[v * length + q] = rng.random_bits(32)
        for scales in ([1, 3, 4], None):
            x = o.upload(coeffs[0], length, count)
            o.forward(*x, length, count)
            y = o.upload(coeffs[1], length, count)
            o.forward(*y, length, count)
            out = o.pointwise(x, y, scales, length, count)
            o.inverse(*out, length, count)
            got = o.download(*out, length, count)
            for v in range(count):
                val = sum(cv << (32 * q) for q, cv in enumerate(got[v * length:(v + 1) * length]))
                a = int.from_bytes(coeffs[0][v * length:(v + 1) * length].tobytes(), "little")
                b = int.from_bytes(coeffs[1][v * length:(v + 1) * length].tobytes(), "little")
                assert val == a * b * (scales[v] if scales else 1)


# ---- the Backend cases of tests/cpu.rs and tests/gmp.rs, at CPU-friendly sizes ----

MAKERS = {
    "cpu": lambda o: (lambda: o.OracleBackend.plain()),
    "wrap": lambda o: (lambda: o.OracleBackend.wraparound()),
    "gmp": lambda o: (lambda: o.OracleBackend.gmp_backend()),
}


@pytest.mark.parametrize("kind", ["cpu", "wrap", "gmp"])
def test_random_modmul(o, kind):
    make = MAKERS[kind](o)
    for bits, cases in [(64, 60), (100, 60), (1000, 30), (10_000, 6), (100_000, 2)]:
        for base in (3, 4):
            common.random_modmul(make, bits, cases, bits, base)


@pytest.mark.parametrize("kind", ["cpu", "wrap", "gmp"])
def test_edges(o, kind):
    make = MAKERS[kind](o)
    for base in (3, 4):
        common.edges(make, base, max_log_len=12)


@pytest.mark.parametrize("kind", ["cpu", "wrap", "gmp"])
def test_independence(o, kind):
    common.batch_independence(MAKERS[kind](o), 3000, [1, 7, 16])


@pytest.mark.parametrize("kind", ["cpu", "wrap", "gmp"])
def test_powmod_mul(o, kind):
    common.powmod_and_mul(MAKERS[kind](o), 2000, 9)


@pytest.mark.parametrize("kind", ["cpu", "wrap"])
def test_fermat_tribonacci(o, kind):
    common.end_to_end(MAKERS[kind](o), common.A092835_SMALL + [100, 200, 1001, 2000])


@pytest.mark.parametrize("kind", ["wrap", "gmp"])
def test_tribonacci_prps(o, kind):
    """A092835 primes report PRP, the listed composites do not (tests/cpu.rs:60-63)."""
    common.known_prps(MAKERS[kind](o), common.A092835_SMALL, common.COMPOSITE_NS)


def test_t802_is_prp(o):
    """tests/cli.rs:10-14: T(802) is a PRP."""
    assert fermat(o.OracleBackend.wraparound(), [common.tribonacci(802)], 3, 1 << 16) == [True]


@pytest.mark.parametrize("kind", ["cpu", "wrap", "gmp"])
def test_api(o, kind):
    common.api_contract(MAKERS[kind](o))


@pytest.mark.parametrize("kind", ["cpu", "wrap", "gmp"])
def test_carries(o, kind):
    common.carry_stress(MAKERS[kind](o), 1 << 11)


def test_long_run(o):
    common.long_run(MAKERS["wrap"](o), 3000, 4, 500)


def test_is_one_upper_lazy_representative(o):
    """tests/cpu.rs:83-95"""
    rng = RandState()
    n = common.rand_odd(rng, 1000)
    b = ModBatch(o.OracleBackend.plain(), [n], 3)
    r = (1 << (32 * b.params.k)) % n
    b.load_raw(0, r + n)
    assert b.is_one(0)
    b.load_raw(0, r)
    assert b.is_one(0)
    b.load_raw(0, r + 1)
    assert not b.is_one(0)


def test_load_raw_rejects_out_of_range(o):
    """tests/cpu.rs:97-103"""
    n = 1_000_003
    b = ModBatch(o.OracleBackend.plain(), [n], 3)
    with pytest.raises(MontMulError, match=r"raw value outside \[0, 2N\)"):
        b.load_raw(0, 2 * n)


def test_fermat_chunk_zero_is_error(o):
    with pytest.raises(MontMulError):
        fermat(o.OracleBackend.plain(), [1_000_003], 3, 0)


def test_wraparound_matches_full_product(o):
    """tests/cpu.rs:111-121: same k = L/2 on both sides, so the raw limbs agree exactly."""
    for bits in (64, 1000, 87_914):
        common.same_raw(lambda: o.OracleBackend.with_full_k(), lambda: o.OracleBackend.wraparound(), bits, 4, 20)


def test_gmp_same_raw_as_cpu(o):
    """tests/gmp.rs:63-66 (smaller step count)."""
    common.same_raw(lambda: o.OracleBackend.gmp_backend(), lambda: o.OracleBackend.plain(), 87_914, 2, 10)


def test_half_factors_layout(o):
    """The wraparound factors exist for every supported length."""
    rng = RandState()
    for e in range(3, 12):
        length = 1 << e
        n = common.rand_odd(rng, 16 * length - 4)
        limbs = np.frombuffer(n.to_bytes(2 * length, "little"), "<u4").astype(np.uint32)
        ab1, ab2 = o.half_factors(limbs, length)
        assert ab1.shape == (length // 2, 2) and int(ab2.max()) < o.P2


def test_score_workload_rng_is_gmp_default(o):
    """score.rs:45-61: N = urandomb(bits) with top and bottom bits set, seed 2026; the stream is
    GMP's default generator, so the first modulus is a fixed value (pinned by its low word)."""
    from montmul_b200.score import ScoreConfig, workload
    moduli, exps = workload(ScoreConfig(bits=1000, slots=3, ebits=100, repeats=1, seed=2026))
    assert all(m.bit_length() == 1000 and m % 2 == 1 for m in moduli)
    assert all(e == (m - 1) >> 900 for m, e in zip(moduli, exps))
    rng = RandState(2026)
    first = rng.random_bits(1000) | (1 << 999) | 1
    assert moduli[0] == first
    assert powm(3, exps[0], moduli[0]) == powm(3, (moduli[0] - 1) >> 900, moduli[0])
