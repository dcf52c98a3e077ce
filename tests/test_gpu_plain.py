"""The path without the wraparound correction (GpuOptions::wraparound = false, gpu/mod.rs:36-44):
k = k0 limbs and the plain REDC, bit-identical to the reference Cpu::default (the oracle's
plain backend). Restates montmul/tests/gpu.rs:333-345."""
import pytest

import common
from montmul_b200 import ModBatch
from montmul_b200.gmp import RandState

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def nowrap():
    from montmul_b200 import B200
    dev = B200(wraparound=False)
    return lambda: dev


@pytest.fixture(scope="module")
def nowrap_global():
    from montmul_b200 import B200
    dev = B200(wraparound=False, force_global=True)
    return lambda: dev


@pytest.fixture(scope="module")
def plain(oracle):
    return lambda: oracle.OracleBackend.plain()


def test_limits(nowrap):
    assert nowrap().full_k() is False
    b = ModBatch(nowrap(), [(1 << 99_999) | 1], 3)
    assert b.params.k == 3126 and b.params.len == 8192


@pytest.mark.parametrize("bits,slots,steps", [(100_000, 8, 100), (1000, 7, 100), (64, 5, 100), (5000, 4, 60)])
def test_same_raw_as_cpu_default(nowrap, plain, bits, slots, steps):
    common.same_raw(nowrap, plain, bits, slots, steps)


def test_same_raw_forced_global(nowrap_global, plain):
    common.same_raw(nowrap_global, plain, 87_914, 8, 50)


def test_same_raw_global_length(nowrap, plain):
    """Naturally global: 400,000 bits, L = 32768."""
    common.same_raw(nowrap, plain, 400_000, 2, 20)


@pytest.mark.parametrize("length", [1 << e for e in range(3, 16)])
def test_every_length_top_of_bucket(nowrap, plain, length):
    """k = k0 at the top of each bucket (k = L/2) and just above the bucket below (k < L/2)."""
    common.same_raw(nowrap, plain, 16 * length - 36, 2, 12)
    common.same_raw(nowrap, plain, 8 * length + 1, 2, 12)


def test_powmod_mul_and_modmul(nowrap):
    common.powmod_and_mul(nowrap, 2000, 9)
    common.random_modmul(nowrap, 1000, 100, 1000, 3)
    common.random_modmul(nowrap, 100_000, 8, 100_000, 4)


def test_edges(nowrap):
    for base in (3, 4):
        common.edges(nowrap, base, max_log_len=16)


def test_carries(nowrap):
    common.carry_stress(nowrap, 1 << 16)


def test_mixed_plan_with_plain_batches(nowrap):
    """A mixed launch over batches without the wraparound path (shared and global lengths)."""
    from montmul_b200.backend import Plan
    from montmul_b200.gmp import powm
    rng = RandState(12)
    spec = []
    for bits in (3000, 90_000, 300_000):
        moduli = [common.rand_odd(rng, bits) for _ in range(3)]
        exps = [common.rand_exponent(rng, 30) for _ in range(3)]
        spec.append((moduli, exps))
    bs = []
    for moduli, exps in spec:
        b = ModBatch(nowrap(), moduli, 3)
        b.load_all([1] * 3)
        b.set_exponents(exps)
        bs.append(b)
    plan = Plan(bs, 8)
    plan.run(30)
    for (moduli, exps), b in zip(spec, bs):
        for i in range(3):
            assert b.read(i) == powm(3, exps[i], moduli[i])


def test_noalloc_rejects_plain(nowrap):
    """The allocation-free product runs the wraparound REDC only; the check precedes any use of
    the (here dummy, never dereferenced) device pointers."""
    from montmul_b200.backend import lib
    b = ModBatch(nowrap(), [(1 << 999) | 1], 3)
    rc = lib().mm_b200_mul_noalloc(b.state.ptr, 0, 16, 16, 16, None, None)
    assert rc != 0 and b"wraparound" in lib().mm_b200_last_error()
