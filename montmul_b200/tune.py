"""Autotuner and cached per-length schedule table (no counterpart in the reference, whose planner
fixes the schedule: montmul/src/gpu/plan.rs:26-60).

For each transform length L the tuner times every schedule the library can switch at run time on
the device and keeps the fastest:

  - the mode: shared memory, global mode or cluster mode. L <= 4096 run in shared memory only;
    L = 8192 and 16384 in shared memory or global mode (16384 in shared memory holds one block per
    SM, in global mode two); L = 32768 and 65536 in global mode or cluster mode (a thread-block
    cluster of L / 16384 blocks per slot with the vector in the cluster's shared memory); longer
    lengths in global mode only;
  - steps per launch (launch_steps): a longer launch saves launch gaps, a shorter one bounds how
    long a batch holds the GPU.

It records the winner's time per slot-step (step_ns), and the length's time per slot-step inside
the mixed-length persistent launch (mixed_ns), which orders that launch's work items and sizes a
serving tick's budgets. The fixed parts of a schedule are reported beside it: threads per block,
the radix schedule of the length-n transform, the tile length of global mode and the blocks per
SM. The table is JSON keyed by device name, cached at $MONTMUL_B200_SCHEDULES or
~/.cache/montmul_b200/schedules.json; without a cache the table shipped in the package
(montmul_b200/schedules.json, measured on a B200 with this command) applies. B200 batches take
their length's row at creation.

    python -m montmul_b200.tune [--lengths 8192 16384 ...] [--force]
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

TILE = 2048           # global mode's tile length (elements of n)
MAX_SHARED_N = 8192   # n <= 8192 fits the shared-memory kernels
MIN_GLOBAL_N = 4096   # global mode from n = 4096 (L = 8192)
LAUNCH_STEPS = (64, 512)
MAX_MIXED_L = 65536     # lengths whose cost inside the mixed launch is measured too


# The table measured on a B200 and shipped with the package; used when no cache exists.
PACKAGED = os.path.join(os.path.dirname(os.path.abspath(__file__)), "schedules.json")


def cache_path() -> str:
    p = os.environ.get("MONTMUL_B200_SCHEDULES")
    if p:
        return p
    return os.path.join(os.path.expanduser("~"), ".cache", "montmul_b200", "schedules.json")


def radix_schedule(m: int):
    """Radix of every pass of a length-2^m transform (the device schedule, mm_common.h)."""
    if m <= 3:
        return [{1: 2, 2: 4, 3: 8}[m]] if m >= 1 else []
    if m % 3 == 0:
        return [8] * (m // 3)
    if m % 3 == 1:
        return [4, 4] + [8] * (m // 3 - 1)
    return [4] + [8] * (m // 3)


def threads_for(m: int) -> int:
    """Threads per block of the shared-memory kernels (mm_abi.h threads_for)."""
    if m >= 12:
        return 512
    return 32 if m - 3 <= 5 else (256 if m - 3 >= 8 else 1 << (m - 3))


SHARED, GLOBAL, CLUSTER = 0, 1, 2
MIN_CLUSTER_N, MAX_CLUSTER_N = 16384, 32768   # L = 32768 and 65536
CLUSTER_CHUNK = 8192                          # elements per block of a cluster


def mode_name(mode) -> str:
    return ("shared", "global", "cluster")[int(mode)]


def fixed_parts(length: int, global_mode, block_threads: int = 0):
    n = length // 2
    m = n.bit_length() - 1
    if int(global_mode) == CLUSTER:
        # 1024 threads per SM: two 512-thread blocks of half the default chunk on each SM
        chunk = CLUSTER_CHUNK // 2 if block_threads == 1024 else CLUSTER_CHUNK
        return {"threads": 512, "blocks_per_sm": CLUSTER_CHUNK // chunk, "cluster": n // chunk, "tile": None,
                "radix": radix_schedule(m)}
    if global_mode:
        g = m - TILE.bit_length() + 1
        return {"threads": 256, "blocks_per_sm": 2, "tile": TILE,
                "radix": {"global": radix_schedule(g), "tile": radix_schedule(TILE.bit_length() - 1)}}
    per_sm = 2 if m <= 12 else 1
    return {"threads": threads_for(m), "blocks_per_sm": per_sm, "tile": None, "radix": radix_schedule(m)}


def alt_threads(length: int, mode: int = SHARED) -> int:
    """The alternative shape at this length, 0 when none is built: in shared mode the step
    kernel's other block size (mm_abi.h alt_threads_for); in cluster mode at L = 32768, 1024
    threads per SM (two blocks of 4,096 elements per SM instead of one of 8,192)."""
    m = (length // 2).bit_length() - 1
    if int(mode) == CLUSTER:
        return 1024 if m == 14 else 0
    if int(mode) == GLOBAL:
        return 0
    return {11: 256, 12: 256, 13: 1024}.get(m, 0)


def candidates(length: int):
    n = length // 2
    modes = []
    if n <= MAX_SHARED_N:
        modes.append(SHARED)
    if n >= MIN_GLOBAL_N:
        modes.append(GLOBAL)
    if MIN_CLUSTER_N <= n <= MAX_CLUSTER_N:
        modes.append(CLUSTER)
    out = []
    for g in modes:
        shapes = [0] + ([alt_threads(length, g)] if alt_threads(length, g) else [])
        out += [(g, s, th) for th in shapes for s in LAUNCH_STEPS]
    return out


def bits_for(length: int) -> int:
    """Top of the bucket: the largest modulus size with this length (k = L/2 limbs, batch.rs:20)."""
    return 16 * length - 4


def measure(dev, length: int, global_mode, launch_steps: int, slots: int, steps: int, seed: int = 2026,
            threads: int = 0):
    """Seconds per slot-step of one schedule on a synthetic batch (random odd moduli at the top of
    the bucket, random exponents), after a warm-up launch."""
    from .batch import ModBatch
    from .gmp import RandState
    rng = RandState(seed)
    bits = bits_for(length)
    moduli = [rng.random_bits(bits) | (1 << (bits - 1)) | 1 for _ in range(slots)]
    exps = [rng.random_bits(steps + 8) | (1 << (steps + 7)) for _ in range(slots)]
    b = ModBatch(dev, moduli, 3)
    be, st = b.backend_and_state()
    be.set_schedule(st, global_mode, launch_steps, 0.0, threads)
    b.load_all([1] * slots)
    b.set_exponents(exps)
    b.run(8)
    t = time.perf_counter()
    b.run(steps)
    dt = time.perf_counter() - t
    return dt / (slots * steps)


def measure_mixed(dev, length: int, slots: int, steps: int, seed: int = 2026):
    """Seconds per slot-step of one length inside the mixed-length persistent launch (one
    512-thread block per SM: L = 16384 as wide items on whole blocks, shorter lengths on its two
    256-thread workers, longer ones in global mode), at full occupancy: the cost that orders a
    mixed launch's items and sizes a serving tick's budgets."""
    from .backend import Plan
    from .batch import ModBatch
    from .gmp import RandState
    rng = RandState(seed)
    bits = bits_for(length)
    moduli = [rng.random_bits(bits) | (1 << (bits - 1)) | 1 for _ in range(slots)]
    exps = [rng.random_bits(steps + 8) | (1 << (steps + 7)) for _ in range(slots)]
    b = ModBatch(dev, moduli, 3)
    b.load_all([1] * slots)
    b.set_exponents(exps)
    plan = Plan([b], steps + 8)
    plan.run(8)
    t = time.perf_counter()
    plan.run(steps)
    dt = time.perf_counter() - t
    plan.close()
    return dt / (slots * steps)


def tune_length(dev, length: int, budget_s: float = 4.0):
    """The fastest schedule of one length, with every candidate's time."""
    sms = dev.sm_count()
    n = length // 2
    # Enough slots for several waves of resident blocks, and enough steps for ~budget_s / candidates.
    slots = sms * (8 if n <= 8192 else 4)
    probe = measure(dev, length, candidates(length)[0][0], 512, slots, 4)
    cands = candidates(length)
    steps = max(8, min(2000, int(budget_s / len(cands) / (probe * slots))))
    results = []
    for g, s, th in cands:
        sec = measure(dev, length, g, s, slots, steps, threads=th)
        results.append({"global": g, "launch_steps": s, "block_threads": th, "step_ns": sec * 1e9})
    ranked = sorted(results, key=lambda r: r["step_ns"])
    best = ranked[0]
    out = dict(best)
    if len(ranked) > 1:
        out["runner_up"] = dict(ranked[1])
    out.update(fixed_parts(length, best["global"], best.get("block_threads", 0)))
    if best.get("block_threads") and int(best["global"]) == SHARED:
        out["threads"] = best["block_threads"]
    out["slots"] = slots
    out["steps"] = steps
    out["candidates"] = results
    if length <= MAX_MIXED_L:
        out["mixed_ns"] = measure_mixed(dev, length, slots, max(8, min(steps, 1000))) * 1e9
    return out


def load_table():
    """The cached table, or the packaged one when there is no cache."""
    for p in (cache_path(), PACKAGED):
        try:
            with open(p) as f:
                return json.load(f)
        except (OSError, ValueError):
            continue
    return {}


def save_table(table) -> None:
    p = cache_path()
    os.makedirs(os.path.dirname(p), exist_ok=True)
    tmp = p + ".tmp"
    with open(tmp, "w") as f:
        json.dump(table, f, indent=1, sort_keys=True)
    os.replace(tmp, p)


def schedule_for(device_name: str, length: int, table=None, cluster_ok: bool = True):
    """The cached schedule of one length on one device, or None. Without `cluster_ok` (a batch
    on the plain REDC path, which cluster mode does not run) a cluster-mode row gives way to its
    fastest measured candidate in another mode."""
    table = load_table() if table is None else table
    row = table.get(device_name, {}).get(str(length))
    if row and not cluster_ok and int(row["global"]) == CLUSTER:
        others = [c for c in row.get("candidates", []) if int(c["global"]) != CLUSTER]
        if not others:
            return None
        best = min(others, key=lambda c: c["step_ns"])
        row = dict(row, **best)
        row.pop("mixed_ns", None)
    return row


def apply(batch, table=None) -> bool:
    """Sets the cached schedule of the batch's length on its backend; False when none is cached."""
    be, st = batch.backend_and_state()
    sc = schedule_for(be.device_name(), batch.params.len, table, getattr(be, "wraparound", True))
    if not sc:
        return False
    be.set_schedule(st, sc["global"], sc["launch_steps"], sc.get("mixed_ns", sc["step_ns"]), sc.get("block_threads", 0))
    return True


def tune(dev, lengths, force: bool = False, log=print, mixed_only: bool = False):
    """Measures the schedule of every length not in the table (all with `force`), and each
    length's cost inside the mixed launch where the table lacks it (all with `mixed_only`, which
    keeps the schedules)."""
    table = load_table()
    name = dev.device_name()
    per = table.setdefault(name, {})
    for length in lengths:
        row = per.get(str(length))
        if row and mixed_only:
            row.pop("mixed_ns", None)
        if row and (mixed_only or not force):
            if "mixed_ns" not in row and length <= MAX_MIXED_L:
                steps = max(8, min(int(row.get("steps", 64)), 1000))
                row["mixed_ns"] = measure_mixed(dev, length, int(row.get("slots", 8 * dev.sm_count())), steps) * 1e9
                log(f"L={length}: {row['mixed_ns'] / 1e3:.2f} us/slot-step in the mixed launch")
                save_table(table)
            continue
        r = tune_length(dev, length)
        per[str(length)] = r
        log(f"L={length}: {mode_name(r['global'])} launch_steps={r['launch_steps']} "
            f"{r['step_ns'] / 1e3:.2f} us/slot-step")
        save_table(table)
    return per


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--lengths", type=int, nargs="*", default=[1 << e for e in range(8, 18)])
    ap.add_argument("--force", action="store_true", help="re-measure lengths already in the table")
    ap.add_argument("--mixed-only", action="store_true",
                    help="keep the schedules and re-measure only each length's cost inside the mixed launch")
    ap.add_argument("--device", type=int, default=0)
    a = ap.parse_args(argv)
    from .backend import B200
    dev = B200(device=a.device)
    per = tune(dev, a.lengths, a.force, mixed_only=a.mixed_only)
    print(json.dumps({str(k): {kk: v for kk, v in per[str(k)].items() if kk != "candidates"} for k in a.lengths}))
    return 0


if __name__ == "__main__":
    sys.exit(main())
