"""Size sweep: uniform batches from 1,024 to 1,000,000 bits (shared mode up to L = 16,384, global
mode above), the reference's sweep (scripts/sweep_bits.sh over `montmul bench`) with device
throughput per size.

For each size: random odd moduli (top and bottom bits set, GMP stream seeded 2026), base 3,
exponent = the top `ebits` bits of N - 1, slots filling 80% of free device memory (at most
`max_slots`), the tuned schedule of the length, one warm-up run, one timed run. Slot 0, the last
slot and two seeded slots are checked against GMP's pow_mod, and `mul` is checked on two slot
pairs that share a modulus.

    python -m montmul_b200 sweep [--bits 1024 8192 ...] [--slots S] [--ebits 256]
"""
from __future__ import annotations

import time

from . import gmp, tune
from .batch import ModBatch, MontMulError, Params


def butterfly_pairs(n: int) -> int:
    """Butterfly pairs per modular squaring at complex length n (4 length-n and 2 length-n/2
    transforms, 4n weight products, n square, n F(N') and n wraparound pointwise products)."""
    lg = n.bit_length() - 1
    return 2 * n * lg + (n // 2) * (lg - 1) + 7 * n


def one_size(dev, bits: int, slots: int, ebits: int, seed: int = 2026) -> dict:
    from .backend import lib
    length = Params.for_bits(bits, dev.supported_lengths()).len
    if not slots:
        per = lib().mm_b200_batch_bytes(2, length, 1) - lib().mm_b200_batch_bytes(1, length, 1)
        slots = max(1, int(0.8 * dev.free_memory()) // per)
    rng = gmp.RandState(seed)
    # Two extra slots repeat the moduli of slots 0 and 1, for the mul check.
    moduli = [rng.random_bits(bits) | (1 << (bits - 1)) | 1 for _ in range(slots)]
    if slots >= 4:
        moduli[-2], moduli[-1] = moduli[0], moduli[1]
    e_bits = min(ebits, bits)
    exps = [(n - 1) >> (bits - e_bits) for n in moduli]
    b = ModBatch(dev, moduli, 3)
    tuned = tune.apply(b)
    b.load_all([1] * slots)
    b.set_exponents(exps)
    b.run(16)
    b.load_all([1] * slots)
    b.set_exponents(exps)
    be, st = b.backend_and_state()
    from .clocks import ClockSampler
    # The timed run repeats (re-armed each time) until about a second has been timed, so that
    # short sizes get a clock record too; the median run counts.
    runs = []
    with ClockSampler(dev.device) as clk:
        while True:
            b.load_all([1] * slots)
            b.set_exponents(exps)
            be.push(st)
            t = time.perf_counter()
            b.run(e_bits)
            runs.append(time.perf_counter() - t)
            if sum(runs) >= 1.0 or len(runs) >= 64:
                break
    secs = sorted(runs)[len(runs) // 2]
    srng = gmp.RandState(seed + 1)
    for i in [0, slots - 1] + [srng.random_below(slots) for _ in range(2)]:
        if b.read(i) != gmp.powm(3, exps[i], moduli[i]):
            raise MontMulError(f"{bits} bits: slot {i} disagrees with pow_mod")
    muls = 0
    if slots >= 4:
        for out, a_, c_ in ((0, 0, slots - 2), (1, slots - 1, 1)):
            x, y = b.read(a_), b.read(c_)
            b.mul(out, a_, c_)
            if b.read(out) != x * y % moduli[out]:
                raise MontMulError(f"{bits} bits: mul disagrees")
            muls += 1
    sched = be.get_schedule(st)
    n = length // 2
    rate = slots * e_bits / secs
    return {"bits": bits, "L": length, "slots": slots, "ebits": e_bits, "seconds": secs, "modsq_per_s": rate,
            "bitsteps_per_s": rate * bits, "gbfly_per_s": rate * butterfly_pairs(n) / 1e9,
            "mode": sched["mode"], "tuned": tuned, "mul_checked": muls, "timed_runs": len(runs),
            "clocks": clk.summary()}


def main(args) -> dict:
    from .backend import B200
    dev = B200(device=args.device)
    cap = args.max_slots or 16 * dev.sm_count()
    rows = []
    for bits in args.bits:
        slots = args.slots or 0
        if not slots:
            from .backend import lib
            length = Params.for_bits(bits, dev.supported_lengths()).len
            per = lib().mm_b200_batch_bytes(2, length, 1) - lib().mm_b200_batch_bytes(1, length, 1)
            slots = min(cap, max(1, int(0.8 * dev.free_memory()) // per))
        rows.append(one_size(dev, bits, slots, args.ebits))
    return {"workload": "uniform batches, base 3, top ebits of N-1, GMP seed 2026", "sizes": rows}
