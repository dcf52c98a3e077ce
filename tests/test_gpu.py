"""Parity of the B200 backend with the oracle (the reference Cpu backend with wraparound, raw
Montgomery limbs bit for bit) and with GMP, through the C ABI. Restates montmul/tests/gpu.rs."""
import pytest

import common
from montmul_b200 import ModBatch, MontMulError
from montmul_b200.gmp import RandState

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu():
    from montmul_b200 import B200
    dev = B200()
    return lambda: dev


@pytest.fixture(scope="module")
def wrap(oracle):
    return lambda: oracle.OracleBackend.wraparound()


@pytest.mark.parametrize("length", [1 << e for e in range(3, 15)])
def test_same_raw_every_length(gpu, wrap, length):
    """Every shared-memory length against Cpu::with_wraparound, top of the bucket."""
    bits = 16 * length - 4
    common.same_raw(gpu, wrap, bits, 3, 12)


@pytest.mark.parametrize("bits", [64, 200, 400, 1000, 5000, 87_914, 100_000])
def test_wraparound_matches_cpu_wraparound(gpu, wrap, bits):
    """tests/gpu.rs:315-330 (8 slots, 100 steps at the smaller sizes)."""
    steps = 100 if bits < 50_000 else 30
    common.same_raw(gpu, wrap, bits, 8, steps)


def test_random_modmul_sizes(gpu):
    for bits, cases in [(64, 100), (1000, 60), (10_000, 20), (100_000, 8), (200_000, 2)]:
        for base in (3, 4):
            common.random_modmul(gpu, bits, cases, bits, base)


def test_edges(gpu):
    for base in (3, 4):
        common.edges(gpu, base, max_log_len=14)


def test_independence(gpu):
    common.batch_independence(gpu, 3000, [1, 7, 64, 1024])


def test_powmod_mul(gpu):
    common.powmod_and_mul(gpu, 2000, 9)
    common.powmod_and_mul(gpu, 87_914, 2)


def test_api(gpu):
    common.api_contract(gpu)


def test_carries(gpu):
    common.carry_stress(gpu, 1 << 14)


def test_fermat_tribonacci(gpu):
    common.end_to_end(gpu, [6, 7, 11, 87, 98, 215, 802, 1001, 2000, 4000])


def test_tribonacci_prps(gpu):
    common.known_prps(gpu, [4202], [4203])


def test_long_run_split_into_launches(gpu):
    """tests/gpu.rs:179-184 at 8 slots and 3,000 exponent bits (several launches of 512 steps)."""
    common.long_run(gpu, 87_914, 8, 3000)


def _carry_overflow(make, bits):
    rng = RandState()
    moduli = [common.rand_odd(rng, bits), common.rand_odd(rng, bits)]
    b = ModBatch(make(), moduli, 4)
    k = b.params.k
    for i in range(2):
        b.load(i, 1)
        b.set_exponent(i, 1)
    import numpy as np
    be, st = b.backend_and_state()
    be.load(st, 1, np.full(k, 0xFFFFFFFF, np.uint32))
    b.run(1)


@pytest.mark.parametrize("bits", [1000, 87_914])
def test_carry_overflow_names_the_slot(gpu, bits):
    """x = R - 1 is outside [0, 2N): the product carries out and the error names slot 1
    (tests/gpu.rs:269-305). Only an error word is set on the device; nothing faults."""
    with pytest.raises(MontMulError, match="slot 1"):
        _carry_overflow(gpu, bits)


def test_oversized_batch_is_error(gpu):
    """tests/gpu.rs:186-196: create fails with a message naming the bytes. The check runs before
    the setup arrays are read, so one row of limbs stands in for the oversized batch."""
    import ctypes as C
    import numpy as np
    from montmul_b200.backend import lib
    dev = gpu()
    k, length = 8192, 16384
    per_slot = lib().mm_b200_batch_bytes(2, length, 1) - lib().mm_b200_batch_bytes(1, length, 1)
    slots = dev.free_memory() // per_slot * 11 // 10 + 1
    assert lib().mm_b200_batch_bytes(slots, length, 1) > dev.free_memory()
    row = np.zeros((1, k), np.uint32)
    ptr = C.c_void_p()
    rc = lib().mm_b200_create(dev._dev, k, length, 3, slots, row, row, row, C.byref(ptr))
    assert rc == 2 and b"bytes" in lib().mm_b200_last_error()


def test_two_batches_interleaved(gpu):
    """tests/gpu.rs:227-258: two live batches of different L, run alternately."""
    from montmul_b200.gmp import powm
    rng = RandState()
    batches = []
    for bits in (3000, 50_000):
        moduli = [common.rand_odd(rng, bits) for _ in range(4)]
        exps = [rng.random_bits(300) | 1 for _ in range(4)]
        b = ModBatch(gpu(), moduli, 3)
        b.load_all([1] * 4)
        b.set_exponents(exps)
        batches.append((b, moduli, exps))
    assert batches[0][0].params.len != batches[1][0].params.len
    while any(b.remaining(i) > 0 for b, _, _ in batches for i in range(4)):
        for b, _, _ in batches:
            b.run(7)
    for b, moduli, exps in batches:
        for i in range(4):
            assert b.read(i) == powm(3, exps[i], moduli[i])


@pytest.mark.parametrize("length,alt", [(4096, 256), (8192, 256), (16384, 1024)])
def test_alternative_block_shape_same_raw(gpu, wrap, length, alt):
    """The alternative block shape a schedule may select (threads per block, mm_abi.h
    alt_threads_for) runs the same steps: raw limbs equal the oracle's, and switching shapes in
    the middle of a run changes nothing."""
    dev = gpu()

    class Alt:
        def __getattr__(self, name):
            return getattr(dev, name)

        def create(self, *a):
            st = dev.create(*a)
            dev.set_schedule(st, 0, 5, 0.0, alt)
            assert dev.get_schedule(st)["threads"] == alt
            return st

    common.same_raw(lambda: Alt(), wrap, 16 * length - 4, 3, 12)
    rng = RandState(length)
    moduli = [common.rand_odd(rng, 16 * length - 4) for _ in range(4)]
    exps = [common.rand_exponent(rng, 20) for _ in range(4)]
    a, b = ModBatch(dev, moduli, 3), ModBatch(dev, moduli, 3)
    for x in (a, b):
        x.load_all([1] * 4)
        x.set_exponents(exps)
    be, st = a.backend_and_state()
    be.set_schedule(st, 0, 0, 0.0, alt)
    a.run(7)
    be.set_schedule(st, 0, 0, 0.0, 0)
    a.run(20)
    b.run(20)
    assert [a.read_raw(i) for i in range(4)] == [b.read_raw(i) for i in range(4)]
    with pytest.raises(MontMulError, match="threads per block"):
        be.set_schedule(st, 0, 0, 0.0, 96)
