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
import sys
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


# dram__bytes_read.sum + dram__bytes_write.sum of one step_kernel launch of this workload, from
# one ncu capture of `python -m montmul_b200.profile --slots SLOTS --steps STEPS --launches 2`
# (second launch): the slots and steps per launch it ran, and its DRAM bytes.
TRAFFIC_CAPTURE = {"slots": 2368, "steps_per_launch": 64, "dram_bytes": 13403741696 + 8097713920}

# The step kernel against the hardware, from one ncu capture of step_kernel<12, 512> on this
# workload (296 slots x 16 steps, second launch): issue slots used, ALU pipe (integer add, logic,
# shift, min: 2 cycles per warp instruction on a B200) and FMA-heavy pipe (IMAD, IMAD.WIDE)
# cycles active. The integer pipes of a B200 SM (measured with single-instruction chains: 64
# ALU-pipe and 64 IMAD lanes per clock) are the ceiling the butterfly peak below runs against.
HW_CAPTURE = {"issue_active": 0.540, "alu_pipe": 0.556, "fmaheavy_pipe": 0.555, "warps_per_scheduler": 6.78,
              "capture": "ncu of step_kernel<12, 512>, 296 slots x 16 steps"}

# The uneven-size persistent batch: 2,000 slots, bits log-uniform in [8,192, 300,000] (seed 7),
# c in {2, 3, 4}, the top 1,000 bits of N - 1; the plan replays its launch from a CUDA graph
# every MIXED_QUANTUM steps.
MIXED_SLOTS, MIXED_LO, MIXED_HI, MIXED_EBITS, MIXED_SEED, MIXED_QUANTUM = 2000, 8192, 300_000, 1000, 7, 128


def hbm_bytes_per_slot_step(n: int) -> int:
    """Per-slot constants that stream per step: F(N') and the A|B factors, 2n elements of 24 B."""
    return 48 * n


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except OSError:
        return {}


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


class CpuScore:
    """The reference's score protocol (montmul/src/score.rs:91-136, main.rs:201-216) on one of its
    CPU backends, restated by the oracle: `cpu` = Cpu with the wraparound path (the semantics
    authority), `gmp` = the Gmp backend's REDC over libgmp. The slot count is the best of
    cores x {1, 2} at 200 exponent bits (best_slots), one worker thread per core; each repeat
    then loads 1 and the top 2,000 bits of N - 1 into every slot and runs all 2,000 steps."""

    def __init__(self, kind: str, cores: int = 0):
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle
        from montmul_b200 import ModBatch
        from montmul_b200.score import ScoreConfig, arm, workload
        oracle.build()
        self.kind = kind
        self.cores = cores or os.cpu_count() or 1
        make = oracle.OracleBackend.wraparound if kind == "cpu" else oracle.OracleBackend.gmp_backend
        self._arm = arm
        best = None
        for slots in (self.cores, 2 * self.cores):
            moduli, exps = workload(ScoreConfig(bits=BITS, slots=slots, ebits=EBITS, repeats=1, seed=SEED))
            probe = [(n - 1) >> (BITS - 200) for n in moduli]
            b = ModBatch(make(threads=self.cores), moduli, 3)
            arm(b, probe)
            t = time.perf_counter()
            b.run(200)
            rate = slots * 200 / (time.perf_counter() - t)
            if best is None or rate > best[0]:
                best = (rate, slots, b, moduli, exps)
        _, self.slots, self.batch, self.moduli, self.exps = best

    def repeat(self):
        """One timed repeat: (modsq/s, seconds)."""
        self._arm(self.batch, self.exps)
        t = time.perf_counter()
        self.batch.run(EBITS)
        dt = time.perf_counter() - t
        return self.slots * EBITS / dt, dt

    def check(self):
        """Slot 0 and the last slot against GMP's pow_mod (the reference's score gate)."""
        from montmul_b200.gmp import powm
        for i in (0, self.slots - 1):
            if self.batch.read(i) != powm(3, self.exps[i], self.moduli[i]):
                raise SystemExit(f"{self.kind} baseline: slot {i} disagrees with pow_mod")

    def describe(self, value, seconds, repeats):
        name = ("reference Cpu backend (wraparound on) restated in C" if self.kind == "cpu"
                else "reference Gmp backend (textbook REDC, k = k0) restated in C over libgmp")
        return {"value": value, "unit": UNIT, "cores": self.cores, "kind": "port",
                "sample": f"{self.slots} slots (best of {self.cores} x {{1,2}} host threads' slot rule) x "
                          f"{EBITS} steps of the 100,000-bit score workload per repeat, {seconds:.1f} s per repeat, "
                          f"median of {repeats}; {name}"}


def cpu_baselines():
    """Both CPU backends of the reference on this host's cores, one full repeat each."""
    out = {}
    for kind in ("cpu", "gmp"):
        s = CpuScore(kind)
        value, dt = s.repeat()
        s.check()
        out[kind] = s.describe(value, dt, 1)
    return out


def run_reference(args, world, rank):
    """--impl reference: the reference's own CPU implementation of the path on all host cores,
    same workload and metric. Its Rust crate cannot be built here, so its two CPU backends run as
    the oracle's C restatements (Cpu, and Gmp over libgmp); the faster one on this host is the
    reference arm. One step = one repeat of the score (2,000 steps on every slot)."""
    if rank != 0:
        return 0
    arms = {kind: CpuScore(kind) for kind in ("cpu", "gmp")}
    probe = {kind: s.repeat() for kind, s in arms.items()}
    kind = max(probe, key=lambda k: probe[k][0])
    s = arms[kind]
    rates, secs = [], []
    for i in range(args.warmup + args.steps):
        r, dt = s.repeat()
        if i >= args.warmup:
            rates.append(r)
            secs.append(dt)
    s.check()
    value = statistics.median(rates)
    other = "gmp" if kind == "cpu" else "cpu"
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * statistics.median(secs),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
            "data": "synthetic (GMP-seeded random odd moduli, seed 2026)",
            "config": {"workload": "score: 100,000-bit odd moduli, L=8192, k=4096, base 3, top 2,000 bits of N-1",
                       "bits": BITS, "ebits": EBITS, "L": 8192, "slots": s.slots, "backend": kind},
            "cpu_baseline": s.describe(value, statistics.median(secs), args.steps),
            "cpu_baseline_other": arms[other].describe(probe[other][0], probe[other][1], 1) | {"backend": other},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def mixed_leg(device: int) -> dict:
    """The uneven-size persistent batch (one plan over every slot, its launch replayed from a CUDA
    graph) against the same slots run as separate uniform batches one after another, on the same
    GPU; each timed with the host clock around the synchronous call, clocks sampled meanwhile,
    and every slot checked against GMP's pow_mod after each run."""
    from montmul_b200 import mixed as mx
    from montmul_b200.backend import B200
    from montmul_b200.clocks import ClockSampler
    dev = B200(device=device)
    work = mx.workload(MIXED_SLOTS, MIXED_LO, MIXED_HI, MIXED_EBITS, MIXED_SEED)
    groups = mx.group(dev, work)
    total = len(work) * MIXED_EBITS
    mx.run_mixed(groups, 32, MIXED_QUANTUM)
    mx.run_separate(groups, 32)
    with ClockSampler(device) as c1:
        t_sep = mx.run_separate(groups, MIXED_EBITS)
    checked_sep = mx.verify(groups, work)
    with ClockSampler(device) as c2:
        t_mix, launches, graph = mx.run_mixed(groups, MIXED_EBITS, MIXED_QUANTUM)
    checked_mix = mx.verify(groups, work)
    return {"workload": f"{len(work)} slots, bits log-uniform in [{MIXED_LO}, {MIXED_HI}] (seed {MIXED_SEED}), "
                        f"c in {{2,3,4}}, top {MIXED_EBITS} bits of N-1",
            "groups": len(groups), "value": total / t_mix, "unit": UNIT,
            "separate_value": total / t_sep, "mixed_over_separate": t_sep / t_mix,
            "mixed_seconds": t_mix, "separate_seconds": t_sep, "launches": launches, "graph_launches": graph,
            "quantum": MIXED_QUANTUM, "timing": "host clock around synchronous calls",
            "clocks": c2.summary(), "clocks_separate": c1.summary(),
            "checked": f"all {checked_mix} slots equal GMP pow_mod after the mixed run, {checked_sep} after the separate run"}


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--slots", type=int, default=0, help="slots per GPU (0: best of 148 x {1,2,4,8,16})")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-mixed", action="store_true", help="skip the uneven-size persistent batch leg")
    args = ap.parse_args(argv)
    if args.warmup < 3:
        ap.error("at least 3 warm-up steps")
    if args.impl == "reference":
        # The CPU reference arm needs no process group: rank 0 alone runs it.
        return run_reference(args, int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")))
    world, rank, local = dist_init()

    from montmul_b200 import B200, ModBatch
    from montmul_b200 import backend as bk
    from montmul_b200.batch import exponent_words
    from montmul_b200.clocks import ClockSampler
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
    # DRAM traffic of one step-kernel launch, from the committed ncu capture of this kernel on this
    # workload; scaled by the slot-steps per launch when this run's launches differ from the
    # captured one (the per-slot constants are re-read from L2 less often in longer launches, so
    # the scaled figure is an estimate and says so).
    steps_per_launch = EBITS * args.steps / max(1, launches)
    cap = TRAFFIC_CAPTURE
    same = cap["slots"] == slots and abs(cap["steps_per_launch"] - steps_per_launch) < 0.5
    traffic = cap["dram_bytes"] * (1.0 if same else slots * steps_per_launch / (cap["slots"] * cap["steps_per_launch"]))
    roofline = {"bound": "int", "achieved": achieved_pairs / 1e9, "peak": peak_pairs / 1e9, "unit": "Gbfly/s",
                "frac": achieved_pairs / peak_pairs, "traffic": traffic,
                "traffic_note": ("dram__bytes_read+write per launch, measured by ncu on a launch of this size"
                                 if same else
                                 "dram__bytes_read+write of an ncu capture of %d slots x %d steps per launch, "
                                 "scaled to this run's %d slots x %.0f steps per launch (estimate)"
                                 % (cap["slots"], cap["steps_per_launch"], slots, steps_per_launch)),
                "note": "butterfly pairs (GF(p^2) product + add + sub in both fields), G(n)=%d per modsq at "
                        "L=8192; peak = the kernels' own arithmetic in register-resident chains on all SMs, "
                        "measured in this run" % g_of_n(n)}
    roofline_hw = dict(HW_CAPTURE, note="fractions of the SM's issue slots and integer pipes the step kernel used "
                                         "in an ncu capture; the butterfly roofline above counts the same arithmetic "
                                         "against a register-resident chain of it")
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
            "roofline_hbm": roofline_hbm, "roofline_hw": roofline_hw, "gpu_launches": launches, "clocks": clocks,
            "checked": "slot 0, last and 2 seeded slots equal GMP pow_mod"}
    del batch, st
    if world == 1 and not args.no_mixed:
        line["mixed"] = mixed_leg(local)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        base = cpu_baselines()
        line["cpu_baseline"] = base["cpu"]
        line["cpu_baseline_gmp"] = base["gmp"]
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
