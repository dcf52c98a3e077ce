"""Global mode (L >= 32768: the vector in device memory, 2,048-element tiles streamed through
shared memory) against the oracle and GMP, through the C ABI. The reference runs these lengths
with its global-memory kernels (montmul/src/gpu/mod.rs:455-511) and tests them in
montmul/tests/gpu.rs (force_global cases, lengths up to 2^17)."""
import pytest

import common
from montmul_b200 import ModBatch, MontMulError
from montmul_b200.gmp import RandState, powm

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu():
    from montmul_b200 import B200
    dev = B200()
    return lambda: dev


@pytest.fixture(scope="module")
def gpu_forced():
    from montmul_b200 import B200
    dev = B200(force_global=True)
    return lambda: dev


@pytest.fixture(scope="module")
def wrap(oracle):
    return lambda: oracle.OracleBackend.wraparound()


@pytest.mark.parametrize("length,steps", [(1 << 15, 12), (1 << 16, 8), (1 << 17, 5), (1 << 18, 3)])
def test_global_same_raw_as_oracle(gpu, wrap, length, steps):
    """Global lengths against Cpu::with_wraparound at the top of the bucket, raw limbs."""
    common.same_raw(gpu, wrap, 16 * length - 4, 3, steps)


@pytest.mark.parametrize("bits", [131_068, 262_140])
def test_forced_global_same_raw_as_shared(gpu, gpu_forced, bits):
    """force_global at L = 8192 and 16384 (gpu/mod.rs:36-44) gives the shared-memory kernels'
    raw limbs exactly: the same transform split into global passes and tiles."""
    common.same_raw(gpu, gpu_forced, bits, 6, 40)


def test_forced_global_random_modmul(gpu_forced):
    common.random_modmul(gpu_forced, 100_000, 6, 100_000, 3)


@pytest.mark.parametrize("bits", [300_000, 600_000, 1_500_000])
def test_global_random_modmul(gpu, bits):
    """Every step's raw result is x^2 c R^-1 mod N in [0, 2N), checked with GMP."""
    common.random_modmul(gpu, bits, 4, bits, 3)


def test_global_edges(gpu):
    """x = 0, N, 2N - 1 and N = 2^b - 1 at the top and bottom of the global buckets."""
    for base in (3, 4):
        common.edges(gpu, base, max_log_len=17)


def test_global_powmod_and_mul(gpu):
    common.powmod_and_mul(gpu, 400_000, 3)


def test_global_long_run(gpu):
    """Several launches (max_launch_steps = 16) on one batch equal pow_mod."""
    from montmul_b200 import B200
    dev = B200(max_launch_steps=16)
    common.long_run(lambda: dev, 500_000, 3, 40)


def test_global_carry_overflow_names_the_slot(gpu):
    rng = RandState()
    bits = 500_000
    moduli = [common.rand_odd(rng, bits), common.rand_odd(rng, bits)]
    b = ModBatch(gpu(), moduli, 4)
    k = b.params.k
    for i in range(2):
        b.load(i, 1)
        b.set_exponent(i, 1)
    import numpy as np
    be, st = b.backend_and_state()
    be.load(st, 1, np.full(k, 0xFFFFFFFF, np.uint32))
    with pytest.raises(MontMulError, match="slot 1"):
        b.run(1)


def test_global_pow_prefix(gpu):
    """3^e mod N for the top 64 bits e of N - 1, random odd 700,000-bit N (global length 2^16),
    against GMP."""
    rng = RandState()
    moduli = [common.rand_odd(rng, 700_000) for _ in range(2)]
    exps = [n - 1 for n in moduli]
    b = ModBatch(gpu(), moduli, 3)
    assert b.params.len >= 1 << 16
    b.load_all([1] * 2)
    b.set_exponents([e >> (e.bit_length() - 64) for e in exps])   # the top 64 bits: a prefix run
    b.run(64)
    for i, n in enumerate(moduli):
        assert b.read(i) == powm(3, exps[i] >> (exps[i].bit_length() - 64), n)


@pytest.mark.parametrize("bits", [300_000, 100_000])
def test_bounded_wait_runs_out_and_context_stays_usable(gpu, wrap, bits):
    """The failure path of the bounded waits on bulk copies (the error word of gpu/mod.rs:179-184,
    extended with code 2): a wait on an mbarrier armed for a copy that is never issued runs out
    after 1 ms and the call reports the time-out naming the slot, with nothing left in flight.
    The same batch then runs normally and stays bit-exact with the oracle."""
    rng = RandState(bits + 5)
    moduli = [common.rand_odd(rng, bits) for _ in range(3)]
    exps = [common.rand_exponent(rng, 24) for _ in range(3)]
    b = ModBatch(gpu(), moduli, 3)
    be, st = b.backend_and_state()
    with pytest.raises(MontMulError, match="slot 0 did not complete within its time limit"):
        be.wait_check(st, 1_000_000)
    ref = ModBatch(wrap(), moduli, 3)
    for batch in (b, ref):
        batch.load_all([5, 6, 7])
        batch.set_exponents(exps)
        batch.run(24)
    assert [b.read_raw(i) for i in range(3)] == [ref.read_raw(i) for i in range(3)]
    for i, (n, e) in enumerate(zip(moduli, exps)):
        assert b.read(i) == powm(5 + i, 1 << e.bit_length(), n) * powm(3, e, n) % n


@pytest.mark.parametrize("length,steps,per_sm", [(1 << 15, 10, 512), (1 << 15, 10, 1024), (1 << 16, 6, 512)])
def test_cluster_mode_same_raw_as_oracle(gpu, wrap, length, steps, per_sm):
    """Cluster mode (one thread-block cluster per slot, the vector in the cluster's shared memory:
    blocks of 8,192 elements, one per SM, or at L = 32768 blocks of 4,096 elements, two per SM)
    at the top of the bucket: raw limbs equal Cpu::with_wraparound."""
    dev = gpu()

    class Cluster:
        def __getattr__(self, name):
            return getattr(dev, name)

        def create(self, *a):
            st = dev.create(*a)
            dev.set_schedule(st, 2, 0, threads=per_sm)
            sc = dev.get_schedule(st)
            assert sc["mode"] == "cluster" and sc["threads"] == per_sm
            return st

    common.same_raw(lambda: Cluster(), wrap, 16 * length - 4, 3, steps)


@pytest.mark.parametrize("bits", [300_000, 1_000_000])
def test_cluster_mode_equals_global_mode_and_pow_mod(gpu, bits):
    """The same batch stepped in cluster mode, then switched to global mode and on, ends with the
    raw limbs of a global-mode run and the value pow_mod gives; a bare step leaves x alone."""
    rng = RandState(bits + 11)
    moduli = [common.rand_odd(rng, bits) for _ in range(5)]
    exps = [common.rand_exponent(rng, 30) for _ in range(5)]
    runs = []
    # (mode, threads per SM) before and after the switch; at L = 32768 also the two-blocks-per-SM
    # cluster shape, switched to and from mid-run
    plans = [((1, 0), (1, 0)), ((2, 0), (1, 0)), ((2, 0), (2, 0))]
    if bits == 300_000:
        plans += [((2, 1024), (2, 0)), ((2, 0), (2, 1024)), ((1, 0), (2, 1024))]
    for first, then in plans:
        b = ModBatch(gpu(), moduli, 3)
        be, st = b.backend_and_state()
        b.load_all([2, 3, 4, 5, 6])
        b.set_exponents(exps)
        be.set_schedule(st, first[0], 7, threads=first[1])
        b.run(13)
        be.set_schedule(st, then[0], 7, threads=then[1])
        b.run(30)
        runs.append([b.read_raw(i) for i in range(5)])
        for i, (n, e) in enumerate(zip(moduli, exps)):
            assert b.read(i) == powm(2 + i, 1 << e.bit_length(), n) * powm(3, e, n) % n
    assert all(r == runs[0] for r in runs)
    b = ModBatch(gpu(), moduli[:2], 3)
    be, st = b.backend_and_state()
    be.set_schedule(st, 2, 0)
    b.load_all([7, 8])
    b.set_exponents(exps[:2])
    before = [b.read_raw(i) for i in range(2)]
    be.run_bare(st, 5)
    assert [b.read_raw(i) for i in range(2)] == before and b.remaining(0) == exps[0].bit_length() - 5


def test_cluster_mode_rejects_other_lengths(gpu):
    b = ModBatch(gpu(), [common.rand_odd(RandState(3), 100_000)], 3)
    be, st = b.backend_and_state()
    with pytest.raises(MontMulError, match="cluster mode runs L = 32768 and 65536 only"):
        be.set_schedule(st, 2, 0)
    b = ModBatch(gpu(), [common.rand_odd(RandState(4), 1_000_000)], 3)
    be, st = b.backend_and_state()
    with pytest.raises(MontMulError, match="cluster mode runs 512 threads per SM"):
        be.set_schedule(st, 2, 0, threads=1024)
