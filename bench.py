#!/usr/bin/env python3
"""Benchmark of the B200 MontMul backend on the reference's score workload.

One step = one timed repeat of the score (montmul/src/score.rs:91-123): every slot loaded with 1
and the top 2,000 bits of N - 1 as exponent, then run(2000) over 100,000-bit moduli (L = 8,192,
k = 4,096), base 3. `value` is slot-steps (modular squarings) per second measured with CUDA
events on the batch's stream with the inputs already in HBM; `e2e` is the same metric through
the public API (ModBatch -> C ABI) with host buffers, so every step's host->device upload of x
and the exponents and the device->host read of x are inside the timed region.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

With N > 1 (torchrun, one process per GPU) every rank runs its own slots: the slots are
independent, so the work shards with no data-path collective (weak scaling); the step time is
the maximum over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "squarings/s @100k-bit"
UNIT = "modsq/s"
BITS, EBITS, SEED = 100_000, 2_000, 2026


def g_of_n(n: int) -> int:
    """Butterfly pairs per modular squaring (4 length-n and 2 length-n/2 transforms, 4n weight
    products, n square, n F(N') and n wraparound pointwise products)."""
    lg = n.bit_length() - 1
    return 2 * n * lg + (n // 2) * (lg - 1) + 7 * n


# dram__bytes_read.sum + dram__bytes_write.sum of one step_kernel launch at L = 8,192 (1,184
# slots x 16 steps): 360.3 MB + 95.6 MB, per slot-step.
DRAM_BYTES_PER_SLOT_STEP = (360.3e6 + 95.6e6) / (1184 * 16)


def hbm_bytes_per_slot_step(n: int) -> int:
    """Per-slot constants that stream per step: F(N') and the A|B factors, 2n elements of 24 B."""
    return 48 * n


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except OSError:
        return {}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def __enter__(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.out = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.out, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.out.close()

    def summary(self):
        if self.proc is None or not self.path:
            return None
        rows = []
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return None
        def num(v):
            try:
                return float(v)
            except ValueError:
                return None
        sm = [num(r[1]) for r in rows if num(r[1]) is not None]
        mx = [num(r[2]) for r in rows if num(r[2]) is not None]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for name, v in zip(names, r[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(rows)}


def dist_backend() -> str:
    """NCCL between GPUs; gloo where there is no GPU (the multi-rank path's CPU tests);
    $MONTMUL_DIST_BACKEND overrides."""
    b = os.environ.get("MONTMUL_DIST_BACKEND")
    if b:
        return b
    import torch
    return "nccl" if torch.cuda.is_available() else "gloo"


def dist_init(timeout_s: float = 600.0):
    """One process per GPU (torchrun): world size, rank and local rank from the environment."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        backend = dist_backend()
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return world, rank, local


def allmax(v: float, world: int) -> float:
    """The maximum of v over the ranks (every rank calls it at the same point)."""
    if world == 1:
        return v
    import torch
    import torch.distributed as dist
    device = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([v], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def shard(slots: int, world: int, rank: int):
    """Rank r runs slots [r * slots, (r + 1) * slots) of one seeded stream: independent moduli per
    rank, no data exchanged (weak scaling)."""
    return rank * slots, (rank + 1) * slots


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def cpu_baseline(seconds: float = 12.0, threads: int = 0):
    """The reference's Cpu backend (wraparound on), restated in C, on every host core, on a
    bounded sample of the score workload: one slot per thread, as many steps as fit ~`seconds`."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    from montmul_b200 import ModBatch
    from montmul_b200.score import ScoreConfig, arm, workload
    oracle.build()
    cores = threads or os.cpu_count() or 1
    moduli, exps = workload(ScoreConfig(bits=BITS, slots=cores, ebits=EBITS, repeats=1, seed=SEED))
    b = ModBatch(oracle.OracleBackend.wraparound(threads=cores), moduli, 3)
    arm(b, exps)
    t = time.perf_counter()
    b.run(2)
    probe = time.perf_counter() - t
    steps = max(2, min(EBITS, int(seconds / max(probe / 2, 1e-6))))
    arm(b, exps)
    t = time.perf_counter()
    b.run(steps)
    dt = time.perf_counter() - t
    return {"value": cores * steps / dt, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{cores} slots x {steps} steps of the 100,000-bit score workload (L=8192), "
                      f"{dt:.1f} s, oracle = reference Cpu backend with wraparound restated in C"}


def run_reference(args, world, rank):
    """--impl reference: the reference's CPU implementation of the path (its Rust crate cannot be
    built here, so the C restatement of its Cpu backend) on all host cores, same metric."""
    if rank != 0:
        return 0
    cores = os.cpu_count() or 1
    steps = []
    base = None
    for i in range(args.warmup + args.steps):
        r = cpu_baseline(seconds=args.ref_seconds, threads=cores)
        if i >= args.warmup:
            steps.append(r["value"])
        base = r
    value = statistics.median(steps)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * args.ref_seconds,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
            "data": "synthetic (GMP-seeded random odd moduli, seed 2026)",
            "config": {"workload": "score: 100,000-bit odd moduli, L=8192, k=4096, base 3, top 2,000 bits of N-1",
                       "bits": BITS, "ebits": EBITS, "L": 8192},
            "cpu_baseline": {**base, "value": value},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--slots", type=int, default=0, help="slots per GPU (0: best of 148 x {1,2,4,8,16})")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--ref-seconds", type=float, default=10.0)
    args = ap.parse_args(argv)
    if args.warmup < 3:
        ap.error("at least 3 warm-up steps")
    if args.impl == "reference":
        # The CPU reference arm needs no process group: rank 0 alone runs it.
        return run_reference(args, int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")))
    world, rank, local = dist_init()

    import ctypes as C

    from montmul_b200 import B200, ModBatch
    from montmul_b200 import backend as bk
    from montmul_b200.batch import exponent_words
    from montmul_b200.gmp import powm
    from montmul_b200.score import ScoreConfig, arm, checked_slots, workload

    dev = B200(device=local)
    sms = dev.sm_count()
    lib = bk.lib()

    # Workload of the largest candidate; smaller batches use its first slots (same GMP stream).
    # With several ranks each takes its own slice of the stream.
    cands = [sms * f for f in (1, 2, 4, 8, 16)]
    cands = [s for s in cands if lib.mm_b200_batch_bytes(s, 8192, 63) * 1.2 < dev.free_memory()]
    per_rank = max(cands + [args.slots])
    moduli_w, exps_w = workload(ScoreConfig(bits=BITS, slots=per_rank * world, ebits=EBITS, repeats=1, seed=SEED))
    lo, hi = shard(per_rank, world, rank)
    moduli_all, exps_all = moduli_w[lo:hi], exps_w[lo:hi]

    def make_batch(slots):
        return ModBatch(dev, moduli_all[:slots], 3)

    def device_time(batch, bits):
        be, st = batch.backend_and_state()
        stream = be.stream(st)
        import torch
        s = torch.cuda.ExternalStream(stream)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        be.push(st)   # the armed inputs reach HBM before the timed region
        e0.record(s)
        be.run_async(st, bits)
        e1.record(s)
        be.sync(st)
        return e0.elapsed_time(e1) * 1e-3

    import torch
    torch.cuda.set_device(local)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{local}")

    # Slot count: the reference's best_slots rule (score.rs:125-136) on device time.
    if args.slots:
        slots = args.slots
    else:
        best = (cands[0], 0.0)
        for s in cands:
            b = make_batch(s)
            arm(b, exps_all[:s])
            b.run(16)
            arm(b, exps_all[:s])
            rate = s * 200 / device_time(b, 200)
            if rate > best[1]:
                best = (s, rate)
            del b
        slots = best[0]
    slots = int(allmax(float(slots), world))   # every rank runs the same slot count

    batch = make_batch(slots)
    exps = exps_all[:slots]
    be, st = batch.backend_and_state()
    stream = torch.cuda.ExternalStream(be.stream(st))
    arm(batch, exps)
    batch.run(64)
    for _ in range(args.warmup):
        arm(batch, exps)
        device_time(batch, EBITS)

    # Timed steps: inputs resident (armed and pushed before each step), L2 flushed between steps.
    times = []
    launches0 = be.launches(st)
    barrier(world)
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            arm(batch, exps)
            flush.zero_()
            torch.cuda.synchronize()
            times.append(device_time(batch, EBITS))
    torch.cuda.synchronize()
    barrier(world)
    launches = be.launches(st) - launches0
    clocks = clk.summary()
    for i in checked_slots(ScoreConfig(bits=BITS, slots=slots, ebits=EBITS, repeats=1, seed=SEED)):
        want = powm(3, exps[i], moduli_all[i])
        if batch.remaining(i) != 0 or batch.read(i) != want:
            raise SystemExit(f"slot {i} disagrees with pow_mod")
    total = sum(times)
    total_max = allmax(total, world)
    value = world * slots * EBITS * args.steps / total_max
    ms_per_step = 1e3 * total_max / args.steps

    # End to end through the public API: pinned-host upload of x and exponents, run, read back.
    e2e_times = []
    k = batch.params.k
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        t = time.perf_counter()
        arm(batch, exps)
        batch.run(EBITS)
        be.read_all(st)
        e2e_times.append(time.perf_counter() - t)
    ew = max(len(exponent_words(e)[0]) for e in exps)
    e2e_t = allmax(statistics.median(e2e_times), world)
    e2e = {"value": world * slots * EBITS / e2e_t, "unit": UNIT,
           "h2d_bytes_per_step": slots * (4 * k + 4 * ew + 8), "d2h_bytes_per_step": slots * (4 * k + 4)}

    # Rooflines of the step kernel (it is every launch in the timed region).
    n = 4096
    per_step_s = total / args.steps
    peak_pairs, _ = bk.bfly_peak(local)
    achieved_pairs = slots * EBITS * g_of_n(n) / per_step_s
    peaks = measured_peaks()
    hbm = peaks.get("hbm_gbs")
    achieved_gbs = slots * EBITS * hbm_bytes_per_slot_step(n) / per_step_s / 1e9
    # DRAM traffic of one step-kernel launch: bytes per slot-step from the committed ncu capture
    # of this kernel on this workload, times the slot-steps of one launch here.
    steps_per_launch = EBITS * args.steps / max(1, launches)
    traffic = DRAM_BYTES_PER_SLOT_STEP * slots * steps_per_launch
    roofline = {"bound": "int", "achieved": achieved_pairs / 1e9, "peak": peak_pairs / 1e9, "unit": "Gbfly/s",
                "frac": achieved_pairs / peak_pairs, "traffic": traffic,
                "traffic_note": "bytes per launch: %.0f B per slot-step (dram__bytes_read+write of one ncu capture, "
                                "profiles/step_kernel_score_L8192.md) x %d slots x %.0f steps per launch"
                                % (DRAM_BYTES_PER_SLOT_STEP, slots, steps_per_launch),
                "note": "butterfly pairs (GF(p^2) product + add + sub in both fields), G(n)=%d per modsq at "
                        "L=8192; peak = the kernels' own arithmetic in register-resident chains on all SMs, "
                        "measured in this run" % g_of_n(n)}
    roofline_hbm = {"bound": "hbm", "achieved": achieved_gbs, "peak": hbm, "unit": "GB/s",
                    "frac": (achieved_gbs / hbm) if hbm else None,
                    "note": "48n B of per-slot constants per slot-step; peak of measured (MEASURED_PEAKS.json)"}

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u64", "data": "synthetic (GMP-seeded random odd moduli, seed 2026)",
            "config": {"workload": "score: 100,000-bit odd moduli, L=8192, k=4096, base 3, top 2,000 bits of N-1",
                       "slots_per_gpu": slots, "bits": BITS, "ebits": EBITS, "L": 8192,
                       "parallelism": f"slots sharded over {world} GPU(s)", "l2": "flushed between steps"},
            "fermat_tests_per_hour": value * 3600.0 / BITS, "e2e": e2e, "roofline": roofline,
            "roofline_hbm": roofline_hbm, "gpu_launches": launches, "clocks": clocks,
            "checked": "slot 0, last and 2 seeded slots equal GMP pow_mod"}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline()
    if rank == 0:
        print(json.dumps(line))
    del batch, st
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
