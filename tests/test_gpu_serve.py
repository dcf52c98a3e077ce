"""The continuous-batching serve loop: requests of several sizes admitted while others run, slots
refilled in place. Each Fermat result must be the same raw Montgomery value as the same request
run alone in its own batch, each verdict equal to pow_mod's, each mul equal to a b mod N."""
import pytest

from montmul_b200 import ModBatch, fermat
from montmul_b200.gmp import powm

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dev():
    from montmul_b200 import B200
    return B200()


def _alone_raw(dev, n):
    b = ModBatch(dev, [n], 3)
    b.load_all([1])
    b.set_exponents([n - 1])
    while b.remaining(0):
        b.run(1 << 16)
    return b.read_raw(0)


@pytest.mark.parametrize("launch", ["stream", "items", "plan"])
def test_served_stream_same_as_alone(dev, launch):
    """Every launch mode: segments that launch, read and refill on their own streams; ticks of
    per-segment uniform launches over slot lists; ticks of one mixed-length persistent plan."""
    from montmul_b200 import serve
    # Seeded next_prime primes up to 6,000 bits (a quick search), Mersenne primes above.
    reqs = serve.stream(40, 400.0, 2000, 40_000, prime_frac=0.2, mul_frac=0.1, seed=20, prime_limit=6000)
    assert {r.prime for r in reqs if r.prime} == {"next_prime", "mersenne"}
    # Small segments force several segments per lane and waiting requests; every verdict is
    # checked while the stream runs.
    checker = serve.VerdictChecker(threads=4)
    srv = serve.Server(dev, quantum=64, segment_slots=6, tuned=False, checker=checker, launch=launch, slice_ms=2.0)
    srv.serve(reqs)
    srv.close()
    assert all(r.done is not None for r in reqs)
    assert len(srv.ticks) > 3 and max(b for _, b, _ in srv.ticks) > 1
    assert len(srv.lanes) >= 3
    for r in reqs:
        if r.kind == "mul":
            assert r.value == r.a * r.b % r.n
            continue
        assert r.verdict == (powm(3, r.n - 1, r.n) == 1)
        if r.prime:
            assert r.verdict
        assert r.raw == _alone_raw(dev, r.n), f"request {r.rid} ({r.n.bit_length()} bits)"
    c = serve.check(dev, reqs, checker.finish(), sample=5)
    ferm = [r for r in reqs if r.kind == "fermat"]
    assert c["mul"] == len(reqs) - len(ferm)
    assert c["primes"] == sum(1 for r in ferm if r.prime)
    assert c["verdicts"] == len(ferm) == c["mersenne_prime"] + c["small_factor"] + c["gmp_powm"]
    assert c["mersenne_prime"] == sum(1 for r in ferm if r.prime == "mersenne")
    assert c["alone"] == 5


def test_run_items_steps_listed_slots_only(dev):
    """mm_b200_run_items_async: listed slots advance by their own budgets (capped at what they have
    left), unlisted ones stay; the results are those of plain run()."""
    from montmul_b200.gmp import RandState
    rng = RandState(9)
    moduli = [rng.random_bits(30_000) | (1 << 29_999) | 1 for _ in range(6)]
    exps = [rng.random_bits(40) | (1 << 39) for _ in range(6)]
    a, b = ModBatch(dev, moduli, 3), ModBatch(dev, moduli, 3)
    for x in (a, b):
        x.load_all([1] * 6)
        x.set_exponents(exps)
    be, st = a.backend_and_state()
    be.run_items_async(st, [4, 1, 2], [10, 3, 100])
    be.sync(st)
    assert [a.remaining(i) for i in range(6)] == [40, 37, 0, 40, 30, 40]
    be.run_items_async(st, [0, 1, 3, 4, 5], [40, 37, 40, 30, 40])
    be.sync(st)
    b.run(40)
    assert [a.read_raw(i) for i in range(6)] == [b.read_raw(i) for i in range(6)]
    for i in range(6):
        assert a.read(i) == powm(3, exps[i], moduli[i])


def test_fermat_driver_on_mersenne_primes(dev):
    """fermat() (batch.rs:187-198) on known primes of two lengths and a composite neighbour."""
    assert fermat(dev, [(1 << 4423) - 1], 3) == [True]
    assert fermat(dev, [(1 << 9689) - 1, (1 << 9689) + 1], 3) == [True, False]
