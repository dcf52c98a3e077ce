"""Uneven-size persistent batch: slots of many sizes in one launch, against the same slots run as
separate uniform batches on the same GPU (no counterpart in the reference, which runs one
uniform batch per launch).

The workload: `slots` random odd moduli whose bit sizes are drawn log-uniform in [lo, hi] (GMP
stream, seed 7), a base c in {2, 3, 4} per slot, exponent = the top `ebits` bits of N - 1. Slots
are grouped by (transform length, c) into uniform batches; the mixed run covers all groups with
one plan (persistent launches over a device work queue, longest items first, replayed from a
CUDA graph), the separate run calls run() on each group in turn. Every slot's result is checked
against GMP's pow_mod.

    python -m montmul_b200 mixed [--slots 2000] [--lo 8192] [--hi 300000] [--ebits 1000]
"""
from __future__ import annotations

import math
import time
from concurrent.futures import ThreadPoolExecutor

from . import gmp
from .batch import ModBatch, MontMulError, Params

MAX_DRAW = 1 << 30


def workload(slots: int = 2000, lo: int = 8192, hi: int = 300_000, ebits: int = 1000, seed: int = 7):
    """(bits, N, c, e) per slot: bits log-uniform in [lo, hi], N with its top and bottom bits set,
    c uniform in {2, 3, 4}, e = (N - 1) >> (bits - ebits)."""
    if not 2 <= lo <= hi or ebits > lo:
        raise MontMulError("need 2 <= lo <= hi and ebits <= lo")
    rng = gmp.RandState(seed)
    out = []
    for _ in range(slots):
        u = rng.random_below(MAX_DRAW) / MAX_DRAW
        bits = int(round(math.exp(math.log(lo) + u * (math.log(hi) - math.log(lo)))))
        n = rng.random_bits(bits) | (1 << (bits - 1)) | 1
        c = 2 + rng.random_below(3)
        out.append((bits, n, c, (n - 1) >> (bits - ebits)))
    return out


def group(dev, work):
    """Uniform batches by (L, c): list of (ModBatch, [slot indices into work], exps)."""
    lengths = dev.supported_lengths()
    groups = {}
    for idx, (bits, n, c, e) in enumerate(work):
        key = (Params.for_bits(bits, lengths).len, c)
        groups.setdefault(key, []).append(idx)
    out = []
    for (length, c), idxs in sorted(groups.items()):
        b = ModBatch(dev, [work[i][1] for i in idxs], c)
        out.append((b, idxs, [work[i][3] for i in idxs]))
    return out


def arm(groups) -> None:
    for b, _, exps in groups:
        b.load_all([1] * len(exps))
        b.set_exponents(exps)


def verify(groups, work, threads: int = 32) -> int:
    """Every slot against pow_mod(c, e, N); returns the number checked."""
    # Reads stay on this thread (a batch serves one host thread at a time); pow_mod runs threaded.
    jobs = []
    for b, idxs, _ in groups:
        for j, i in enumerate(idxs):
            if b.remaining(j) != 0:
                raise MontMulError(f"slot {j} of the L={b.params.len} c={b.base} batch has bits left")
            jobs.append((b.params.len, b.base, j, b.read(j), work[i]))

    def one(job):
        length, base, j, got, (_, n, c, e) = job
        if got != gmp.powm(c, e, n):
            raise MontMulError(f"slot {j} of the L={length} c={base} batch disagrees with pow_mod")
        return 1

    with ThreadPoolExecutor(threads) as ex:
        return sum(ex.map(one, jobs))


def run_mixed(groups, ebits: int, quantum: int, tuned: bool = True):
    """One plan over every group; returns (seconds, launches, graph launches)."""
    from .backend import Plan
    from . import tune
    if tuned:
        table = tune.load_table()
        for b, _, _ in groups:
            tune.apply(b, table)
    plan = Plan([b for b, _, _ in groups], quantum)
    arm(groups)
    for b, _, _ in groups:
        b.backend.push(b.state)
    t = time.perf_counter()
    plan.run(ebits)
    dt = time.perf_counter() - t
    out = (dt, plan.launches(), plan.graph_launches())
    plan.close()
    return out


def run_separate(groups, ebits: int):
    arm(groups)
    for b, _, _ in groups:
        b.backend.push(b.state)
    t = time.perf_counter()
    for b, _, _ in groups:
        b.run(ebits)
    return time.perf_counter() - t


def main(args) -> dict:
    from .backend import B200
    dev = B200(device=args.device)
    work = workload(args.slots, args.lo, args.hi, args.ebits, args.seed)
    groups = group(dev, work)
    total = len(work) * args.ebits
    # Warm-up of both paths (tables, graph capture, clocks).
    run_mixed(groups, min(args.ebits, 32), args.quantum)
    run_separate(groups, min(args.ebits, 32))
    from .clocks import ClockSampler
    with ClockSampler(args.device) as c_sep:
        t_sep = run_separate(groups, args.ebits)
    checked_sep = verify(groups, work)
    with ClockSampler(args.device) as c_mix:
        t_mix, launches, graph = run_mixed(groups, args.ebits, args.quantum)
    checked_mix = verify(groups, work)
    return {
        "workload": f"{len(work)} slots, bits log-uniform in [{args.lo}, {args.hi}] (seed {args.seed}), "
                    f"c in {{2,3,4}}, top {args.ebits} bits of N-1",
        "groups": [{"L": b.params.len, "c": b.base, "slots": len(idxs)} for b, idxs, _ in groups],
        "mixed_modsq_per_s": total / t_mix, "separate_modsq_per_s": total / t_sep,
        "mixed_over_separate": t_sep / t_mix, "mixed_seconds": t_mix, "separate_seconds": t_sep,
        "mixed_launches": launches, "mixed_graph_launches": graph, "quantum": args.quantum,
        "checked": f"all {checked_mix} slots equal GMP pow_mod after each run ({checked_sep} separate)",
        "clocks": c_mix.summary(), "clocks_separate": c_sep.summary(),
    }
