"""Mixed-length persistent launches, schedule switches and in-place refill (no counterpart in the
reference: its launches each cover one batch of one length). Every result must be bit-identical
to the same slots run alone in uniform batches, and equal to GMP's pow_mod."""
import pytest

import common
from montmul_b200 import ModBatch, MontMulError
from montmul_b200.gmp import RandState, powm

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dev():
    from montmul_b200 import B200
    return B200()


def _batches(dev, sizes, slots, ebits, seed):
    rng = RandState(seed)
    out = []
    for j, bits in enumerate(sizes):
        moduli = [common.rand_odd(rng, bits) for _ in range(slots)]
        exps = [common.rand_exponent(rng, ebits) for _ in range(slots)]
        base = 2 + j % 3
        out.append((moduli, exps, base))
    return out


def _arm(dev, spec):
    bs = []
    for moduli, exps, base in spec:
        b = ModBatch(dev, moduli, base)
        b.load_all([1] * len(moduli))
        b.set_exponents(exps)
        bs.append(b)
    return bs


@pytest.mark.parametrize("quantum", [7, 1 << 16])
def test_mixed_plan_same_as_alone(dev, quantum):
    """Batches of L = 256 .. 32768 (shared and global mode in one launch) end with the raw limbs
    they reach alone, and with pow_mod."""
    from montmul_b200.backend import Plan
    spec = _batches(dev, [3000, 30_000, 100_000, 200_000, 400_000], 5, 40, 11)
    mixed = _arm(dev, spec)
    assert sorted({b.params.len for b in mixed}) == [256, 2048, 8192, 16384, 32768]
    plan = Plan(mixed, quantum)
    plan.run(40)
    assert plan.launches() == -(-40 // quantum)
    assert plan.graph_launches() == 40 // quantum
    alone = _arm(dev, spec)
    for b in alone:
        b.run(40)
    for (moduli, exps, base), bm, ba in zip(spec, mixed, alone):
        for i in range(len(moduli)):
            assert bm.remaining(i) == 0
            assert bm.read_raw(i) == ba.read_raw(i), f"L {bm.params.len} slot {i}"
        for i in (0, len(moduli) - 1):
            assert bm.read(i) == powm(base, exps[i], moduli[i])
    plan.close()


@pytest.mark.parametrize("quantum", [9, 1 << 16])
def test_mixed_plan_cluster_items(dev, quantum):
    """L = 32768 batches in cluster mode run as cluster items of the mixed launch (a block pair on
    one slot), beside an L = 32768 batch in global mode on the workers and shorter lengths; every
    slot ends as it does alone, and with pow_mod."""
    from montmul_b200.backend import Plan
    spec = _batches(dev, [300_000, 400_000, 500_000, 100_000, 250_000], 4, 33, 23)
    mixed = _arm(dev, spec)
    modes = [2, 1, 2, 1, 0]
    for b, mode in zip(mixed, modes):
        be, st = b.backend_and_state()
        be.set_schedule(st, mode, 0)
    assert [b.params.len for b in mixed] == [32768, 32768, 32768, 8192, 16384]
    plan = Plan(mixed, quantum)
    plan.run(33)
    alone = _arm(dev, spec)
    for b in alone:
        b.run(33)
    for (moduli, exps, base), bm, ba in zip(spec, mixed, alone):
        for i in range(len(moduli)):
            assert bm.remaining(i) == 0
            assert bm.read_raw(i) == ba.read_raw(i), f"L {bm.params.len} slot {i}"
        assert bm.read(0) == powm(base, exps[0], moduli[0])
    plan.close()


def test_mixed_plan_partial_runs(dev):
    """plan.run(bits) advances every slot by at most `bits`; uneven exponent lengths finish at
    their own step."""
    from montmul_b200.backend import Plan
    rng = RandState(5)
    spec = []
    for bits in (10_000, 120_000):
        moduli = [common.rand_odd(rng, bits) for _ in range(4)]
        exps = [common.rand_exponent(rng, 10 + 9 * i) for i in range(4)]
        spec.append((moduli, exps, 3))
    bs = _arm(dev, spec)
    plan = Plan(bs, 4)
    for _ in range(3):
        plan.run(10)
    for (moduli, exps, _), b in zip(spec, bs):
        for i, e in enumerate(exps):
            assert b.remaining(i) == max(0, e.bit_length() - 30)
    plan.run(100)
    for (moduli, exps, _), b in zip(spec, bs):
        for i, e in enumerate(exps):
            assert b.read(i) == powm(3, e, moduli[i])


@pytest.mark.parametrize("bits", [100_000, 200_000])
def test_schedule_switch_mid_run(dev, bits):
    """Shared and global mode compute the same constants and steps: switching between them
    mid-run leaves the raw limbs of a shared-only run."""
    rng = RandState(21)
    moduli = [common.rand_odd(rng, bits) for _ in range(4)]
    exps = [common.rand_exponent(rng, 60) for _ in range(4)]
    a = ModBatch(dev, moduli, 3)
    b = ModBatch(dev, moduli, 3)
    for x in (a, b):
        x.load_all([1] * 4)
        x.set_exponents(exps)
    a.run(60)
    be, st = b.backend_and_state()
    for mode in (False, True, False):
        be.set_schedule(st, mode, launch_steps=7)
        assert be.get_schedule(st)["global"] == mode
        b.run(20)
    for i in range(4):
        assert a.read_raw(i) == b.read_raw(i)


def test_schedule_rejects_shared_above_16384(dev):
    rng = RandState(2)
    b = ModBatch(dev, [common.rand_odd(rng, 400_000)], 3)
    be, st = b.backend_and_state()
    with pytest.raises(MontMulError, match="global mode only"):
        be.set_schedule(st, False)


@pytest.mark.parametrize("bits", [50_000, 400_000])
def test_refill_in_place(dev, bits):
    """Two slots get new moduli, values and exponents mid-run; the others keep going."""
    rng = RandState(8)
    moduli = [common.rand_odd(rng, bits) for _ in range(6)]
    exps = [common.rand_exponent(rng, 50) for _ in range(6)]
    b = ModBatch(dev, moduli, 3)
    b.load_all([1] * 6)
    b.set_exponents(exps)
    b.run(20)
    new_n = [common.rand_odd(rng, bits - 7), common.rand_odd(rng, bits)]
    new_x = [5, 12345]
    new_e = [common.rand_exponent(rng, 33), common.rand_exponent(rng, 70)]
    b.refill([1, 4], new_n, new_x, new_e)
    assert b.remaining(1) == 33 and b.remaining(4) == 70 and b.remaining(0) == 30
    b.run(100)
    for i in range(6):
        if i == 1:
            want = _pow_from(5, new_e[0], 3, new_n[0])
        elif i == 4:
            want = _pow_from(12345, new_e[1], 3, new_n[1])
        else:
            want = powm(3, exps[i], moduli[i])
        assert b.read(i) == want, f"slot {i}"
    raws = b.read_raw_slots([5, 1, 4])
    assert raws == [b.read_raw(5), b.read_raw(1), b.read_raw(4)]


def _pow_from(x0, e, c, n):
    """The step's semantics from x0: x <- x^2 c^bit for the bits of e, MSB first."""
    x = x0 % n
    for bit in bin(e)[2:]:
        x = x * x % n
        if bit == "1":
            x = x * c % n
    return x


def test_refill_between_plan_runs(dev):
    """A refill on one batch between two mixed launches is ordered with them."""
    from montmul_b200.backend import Plan
    rng = RandState(9)
    spec = _batches(dev, [20_000, 300_000], 4, 30, 13)
    bs = _arm(dev, spec)
    plan = Plan(bs, 8)
    plan.run(12)
    n2 = common.rand_odd(rng, 20_000)
    e2 = common.rand_exponent(rng, 25)
    bs[0].refill([2], [n2], [7], [e2])
    plan.run(64)
    assert bs[0].read(2) == _pow_from(7, e2, spec[0][2], n2)
    for j, (moduli, exps, base) in enumerate(spec):
        for i in range(4):
            if j == 0 and i == 2:
                continue
            assert bs[j].read(i) == powm(base, exps[i], moduli[i])


def test_plan_run_each_budgets(dev):
    """plan.run_each: per-batch step budgets in one launch, 0 leaving a batch untouched."""
    from montmul_b200.backend import Plan
    spec = _batches(dev, [5000, 60_000, 250_000], 3, 50, 23)
    bs = _arm(dev, spec)
    plan = Plan(bs, 16)
    plan.run_each([40, 0, 7])
    assert [bs[0].remaining(i) for i in range(3)] == [10] * 3
    assert [bs[1].remaining(i) for i in range(3)] == [50] * 3
    assert [bs[2].remaining(i) for i in range(3)] == [43] * 3
    plan.run_each([40, 50, 43])
    plan.run(1)   # nothing left: no launch
    for (moduli, exps, base), b in zip(spec, bs):
        for i in range(3):
            assert b.remaining(i) == 0 and b.read(i) == powm(base, exps[i], moduli[i])
    assert plan.graph_launches() == 2


def test_plan_run_items_lists(dev):
    """plan.run_items: an explicit work list (any order, per-slot budgets, unlisted slots idle);
    the same slot twice in one list is rejected."""
    from montmul_b200.backend import Plan
    spec = _batches(dev, [4000, 150_000], 3, 40, 29)
    bs = _arm(dev, spec)
    plan = Plan(bs, 8)
    assert plan.blocks() >= 148 and plan.blocks() == 2 * plan.wide_blocks()
    assert plan.batch_wide(1) and not plan.batch_wide(0)   # L = 16384 in shared mode
    plan.run_items([1, 0, 0], [2, 0, 1], [30, 5, 40])
    assert [bs[0].remaining(i) for i in range(3)] == [35, 0, 40]
    assert [bs[1].remaining(i) for i in range(3)] == [40, 40, 10]
    with pytest.raises(MontMulError, match="twice"):
        plan.run_items([0, 0], [2, 2], [1, 1])
    plan.run_items([0, 0, 1, 1, 1], [0, 2, 0, 1, 2], [35, 40, 40, 40, 10])
    for (moduli, exps, base), b in zip(spec, bs):
        for i in range(3):
            assert b.remaining(i) == 0 and b.read(i) == powm(base, exps[i], moduli[i])


def test_wide_and_global_16384_in_one_plan(dev):
    """L = 16384 runs as wide items (a whole block, the vector in shared memory) or, for a batch
    tuned to global mode, on a worker in global mode; beside L = 512 items both end with the raw
    limbs of the batches run alone, and with pow_mod."""
    from montmul_b200.backend import Plan
    spec = _batches(dev, [200_000, 190_000, 4000], 4, 30, 41)
    bs = _arm(dev, spec)
    be, st = bs[1].backend_and_state()
    be.set_schedule(st, True, launch_steps=7)
    plan = Plan(bs, 16)
    assert [plan.batch_wide(i) for i in range(3)] == [True, False, False]
    plan.run_items([2, 0, 1, 0, 2], [0, 1, 2, 3, 3], [30, 11, 30, 30, 5])
    plan.run(30)
    alone = _arm(dev, spec)
    for b in alone:
        b.run(30)
    for (moduli, exps, base), bm, ba in zip(spec, bs, alone):
        for i in range(4):
            assert bm.remaining(i) == 0
            assert bm.read_raw(i) == ba.read_raw(i), f"L {bm.params.len} slot {i}"
            assert bm.read(i) == powm(base, exps[i], moduli[i])
    plan.close()


def test_plan_run_after_a_schedule_switch(dev):
    """plan.run keeps the item kinds of the plan's creation: an L = 16384 batch tuned to global
    mode (a worker item) and one in shared mode (a wide item) both switch mode after the plan
    exists, and both end with the raw limbs of the batches run alone, and with pow_mod."""
    from montmul_b200.backend import Plan
    spec = _batches(dev, [190_000, 200_000], 3, 24, 43)
    bs = _arm(dev, spec)
    be0, st0 = bs[0].backend_and_state()
    be0.set_schedule(st0, True, launch_steps=7)
    plan = Plan(bs, 16)
    assert [plan.batch_wide(i) for i in range(2)] == [False, True]
    be0.set_schedule(st0, False, launch_steps=7)
    be1, st1 = bs[1].backend_and_state()
    be1.set_schedule(st1, True, launch_steps=7)
    plan.run(24)
    alone = _arm(dev, spec)
    for b in alone:
        b.run(24)
    for (moduli, exps, base), bm, ba in zip(spec, bs, alone):
        for i in range(3):
            assert bm.remaining(i) == 0
            assert bm.read_raw(i) == ba.read_raw(i), f"L {bm.params.len} slot {i}"
            assert bm.read(i) == powm(base, exps[i], moduli[i])
    plan.close()
