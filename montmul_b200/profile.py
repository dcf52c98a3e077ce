"""A profiling target: one batch of the score workload (100,000-bit moduli, L = 8,192) and a
given number of fused-step launches, for `ncu -k regex:step_kernel`.

    python -m montmul_b200.profile --slots 1184 --steps 16 --launches 2

The first launch warms up; every launch runs `--steps` steps on all slots. The batch runs in its
length's tuned mode (shared, global or cluster) unless `--mode` names one.
"""
from __future__ import annotations

import argparse
import sys
import time


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--slots", type=int, default=1184)
    ap.add_argument("--steps", type=int, default=16)
    ap.add_argument("--launches", type=int, default=2)
    ap.add_argument("--bits", type=int, default=100_000)
    ap.add_argument("--mode", choices=["tuned", "shared", "global", "cluster"], default="tuned")
    a = ap.parse_args(argv)
    from . import B200, ModBatch, tune
    from .score import ScoreConfig, arm, workload
    moduli, exps = workload(ScoreConfig(bits=a.bits, slots=a.slots, ebits=min(2000, a.bits), repeats=1, seed=2026))
    dev = B200(max_launch_steps=a.steps)
    b = ModBatch(dev, moduli, 3)
    be, st = b.backend_and_state()
    shape = 0
    if a.mode == "tuned":
        row = tune.schedule_for(dev.device_name(), b.params.len)
        mode = int(row["global"]) if row else None
        shape = int(row.get("block_threads", 0)) if row else 0
    else:
        mode = {"shared": tune.SHARED, "global": tune.GLOBAL, "cluster": tune.CLUSTER}[a.mode]
    if mode is not None:
        be.set_schedule(st, mode, a.steps, 0.0, shape)
    sc = be.get_schedule(st)
    print(f"L = {b.params.len}, mode {sc['mode']}, {sc['threads']} threads, {a.steps} steps per launch")
    arm(b, exps)
    for i in range(a.launches):
        t = time.perf_counter()
        b.run(a.steps)
        dt = time.perf_counter() - t
        print(f"launch {i}: {a.slots} slots x {a.steps} steps in {dt * 1e3:.1f} ms "
              f"({a.slots * a.steps / dt:.0f} modsq/s)")
    return 0


if __name__ == "__main__":
    sys.exit(main())
