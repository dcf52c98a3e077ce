"""Command-line front end (the reference's montmul/src/main.rs with --backend b200):

    python -m montmul_b200 bench --backend b200 --bits B --slots S --steps K [--csv PATH]
    python -m montmul_b200 prp   --backend b200 --index N
    python -m montmul_b200 fermat --backend b200 [--slots 64] [--bits 4096] [--primes 4] [--seed 2026]
    python -m montmul_b200 score --backend b200 [--slots S] [--label TEXT] [--csv PATH] [--ncu]
    python -m montmul_b200 sweep [--bits 1024 8192 ...] [--slots S] [--ebits 256]
    python -m montmul_b200 mixed [--slots 2000] [--lo 8192] [--hi 300000] [--ebits 1000]
    python -m montmul_b200 serve [--load 0.7 0.95] [--duration 40] [--lo 10000] [--hi 200000]
    python -m montmul_b200 tune  [--lengths ...] [--force] [--mixed-only]

bench, prp and score print `key=value` fields as the reference does (and append a CSV row with
--csv); sweep, mixed and serve print one JSON object. Only the b200 backend is part of this
package: the reference's Cpu and Gmp backends exist here only as the test suite's oracles.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time


def _backend(name: str, device: int = 0):
    if name != "b200":
        raise SystemExit(f"unknown or unavailable backend {name} (this package provides b200)")
    from .backend import B200
    return B200(device=device)


def _device_name(dev) -> str:
    return "_".join(dev.device_name().split()).replace(",", "")


def _emit(fields, csv_path=None) -> None:
    print(" ".join(f"{k}={v}" for k, v in fields))
    if csv_path:
        d = os.path.dirname(csv_path)
        if d:
            os.makedirs(d, exist_ok=True)
        fresh = not os.path.exists(csv_path) or os.path.getsize(csv_path) == 0
        with open(csv_path, "a") as f:
            if fresh:
                f.write(",".join(k for k, _ in fields) + "\n")
            f.write(",".join(str(v) for _, v in fields) + "\n")


def cmd_bench(a) -> int:
    """Random odd moduli and `steps`-bit exponents, one warm-up run(16), one timed run(steps)
    (main.rs:134-180)."""
    from .batch import ModBatch
    from .gmp import RandState
    if a.bits < 2 or a.slots <= 0 or a.steps <= 0:
        raise SystemExit("bits >= 2, slots > 0 and steps > 0 required")
    dev = _backend(a.backend, a.device)
    rng = RandState()
    moduli = [rng.random_bits(a.bits) | (1 << (a.bits - 1)) | 1 for _ in range(a.slots)]
    exps = [rng.random_bits(a.steps) | (1 << (a.steps - 1)) for _ in range(a.slots)]
    b = ModBatch(dev, moduli, 3)
    from . import tune
    tune.apply(b)
    b.load_all([1] * a.slots)
    b.set_exponents(exps)
    b.run(16)
    b.load_all([1] * a.slots)
    b.set_exponents(exps)
    t = time.perf_counter()
    b.run(a.steps)
    secs = time.perf_counter() - t
    _emit([("backend", a.backend), ("device", _device_name(dev)), ("bits", a.bits), ("L", b.params.len),
           ("slots", a.slots), ("steps", a.steps), ("bare", "false"),
           ("us_per_step_slot", f"{secs * 1e6 / (a.steps * a.slots):.3f}"),
           ("bitsteps_per_s", f"{a.bits * a.slots * a.steps / secs:.4e}")], a.csv)
    return 0


def cmd_prp(a) -> int:
    """Fermat base 3 on the tribonacci number T(index) (main.rs:183-189)."""
    from .batch import fermat
    t0 = time.perf_counter()
    t = tribonacci(a.index)
    dev = _backend(a.backend, a.device)
    got = fermat(dev, [t], 3, 1 << 16)
    print(f"T({a.index}) bits={t.bit_length()} prp={str(got[0]).lower()} seconds={time.perf_counter() - t0:.3f}")
    return 0


def cmd_fermat(a) -> int:
    """The CPU-sized Fermat batch (`score.fermat_workload`: random odd moduli with seeded
    next_prime primes among them) through the Fermat driver, every slot's value and verdict
    checked against GMP's pow_mod."""
    from .score import fermat_checked, fermat_workload
    from .batch import Params
    dev = _backend(a.backend, a.device)
    moduli, primes = fermat_workload(a.slots, a.bits, a.primes, a.seed)
    verdicts, _, secs = fermat_checked(dev, moduli, 3)
    prp = [i for i, v in enumerate(verdicts) if v]
    if prp != primes:
        raise SystemExit(f"PRP slots {prp} differ from the planted primes {primes}")
    steps = sum(n.bit_length() for n in moduli)   # N - 1 has as many bits as N (N odd, > 1)
    _emit([("backend", a.backend), ("device", _device_name(dev)), ("bits", a.bits),
           ("L", Params.for_bits(a.bits, dev.supported_lengths()).len), ("slots", a.slots),
           ("prp", len(prp)), ("prp_slots", ";".join(map(str, prp))), ("seconds", f"{secs:.4f}"),
           ("modsq_per_s", f"{steps / secs:.2f}"), ("fermat_tests_per_hour", f"{3600.0 * a.slots / secs:.2f}"),
           ("checked", "every_slot_pow_mod_and_verdict")], a.csv)
    return 0


def tribonacci(n: int) -> int:
    """T(0) = T(1) = 0, T(2) = 1, T(n) = T(n-1) + T(n-2) + T(n-3) (montmul/src/seq.rs:6-15)."""
    a, b, c = 0, 0, 1
    for _ in range(n):
        a, b, c = b, c, a + b + c
    return a


NCU_SM = "sm__throughput.avg.pct_of_peak_sustained_elapsed"
NCU_MEM = "gpu__compute_memory_throughput.avg.pct_of_peak_sustained_elapsed"
NCU_MAX_SLOTS_PER_SM = 2


def parse_ncu_csv(text: str):
    """(SM throughput %, memory throughput %) of the last profiled launch in ncu's --csv output
    (main.rs:221-245): rows are quoted, the header names "Metric Name" and "Metric Value"."""
    import csv
    import io
    rows = [r for r in csv.reader(io.StringIO("\n".join(l for l in text.splitlines() if l.startswith('"'))))]
    if not rows:
        raise ValueError("no ncu output")
    head = rows[0]
    try:
        name, value = head.index("Metric Name"), head.index("Metric Value")
    except ValueError as e:
        raise ValueError(f"ncu column missing: {e}") from None

    def last(metric):
        for r in reversed(rows[1:]):
            if len(r) > max(name, value) and r[name] == metric:
                return float(r[value].replace(",", ""))
        raise ValueError(f"ncu metric {metric} missing")

    return last(NCU_SM), last(NCU_MEM)


def ncu_metrics(slots: int, device: int):
    """One 16-step launch of the score workload under Nsight Compute (clocks left alone), after
    the same command has run once without it; returns (SM %, memory %) of that launch."""
    import shutil
    import subprocess
    cmd = [sys.executable, "-m", "montmul_b200", "ncu-launch", "--slots", str(slots), "--device", str(device)]
    plain = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    if plain.returncode != 0:
        raise RuntimeError(f"ncu-launch failed without ncu: {plain.stderr.strip()[-400:]}")
    ncu = shutil.which("ncu") or "/usr/local/cuda/bin/ncu"
    r = subprocess.run([ncu, "--csv", "--clock-control", "none", "--kernel-name", "regex:step_kernel", "-c", "1",
                        "--metrics", f"{NCU_SM},{NCU_MEM}", *cmd], capture_output=True, text=True, timeout=900)
    if r.returncode != 0:
        raise RuntimeError(f"ncu failed: {r.stderr.strip()[-400:]}")
    return parse_ncu_csv(r.stdout)


def cmd_ncu_launch(a) -> int:
    """The profiled launch of score --ncu (main.rs:333-342): the score workload at --slots slots,
    armed, then one launch of 16 steps."""
    from .backend import B200
    from .batch import ModBatch
    from .score import ScoreConfig, arm, workload
    moduli, exps = workload(ScoreConfig.standard(a.slots))
    b = ModBatch(B200(device=a.device, max_launch_steps=16), moduli, 3)
    arm(b, exps)
    b.run(16)
    return 0


def cmd_score(a) -> int:
    """The standard score at --slots, or at the best of SMs x {1, 2, 4, 8, 16} (main.rs:192-299)."""
    from .score import GMP_M5_SECONDS_PER_MODSQ_100K, ScoreConfig, best_slots, gpu_overhead, score
    dev = _backend(a.backend, a.device)
    make = lambda: dev  # noqa: E731
    if a.slots:
        slots = a.slots
    else:
        from .backend import lib
        cands = [dev.sm_count() * f for f in (1, 2, 4, 8, 16)]
        cands = [s for s in cands if lib().mm_b200_batch_bytes(s, 8192, 63) * 1.2 < dev.free_memory()]
        slots = best_slots(make, 100_000, cands)
    s = score(make, ScoreConfig.standard(slots))
    s.overhead = gpu_overhead(make, ScoreConfig.standard(slots))
    sm_pct = mem_pct = ""
    if a.ncu:
        # One launch on at most two slots per SM: a profile of a few milliseconds.
        per = min(slots, NCU_MAX_SLOTS_PER_SM * dev.sm_count())
        try:
            sm, mem = ncu_metrics(per, a.device)
            sm_pct, mem_pct = f"{sm:.4f}", f"{mem:.4f}"
        except (RuntimeError, ValueError, OSError) as e:
            print(f"warning: ncu profile failed, sm_pct and mem_pct left empty: {e}", file=sys.stderr)
    _emit([("timestamp", int(time.time())), ("label", '"' + a.label.replace('"', '""') + '"'),
           ("device", _device_name(dev)), ("backend", a.backend), ("slots", s.slots),
           ("modsq_per_s", f"{s.modsq_per_s:.2f}"), ("mad", f"{s.mad:.2f}"),
           ("fermat_tests_per_hour", f"{s.fermat_tests_per_hour:.4f}"), ("overhead", f"{s.overhead:.4f}"), ("sm_pct", sm_pct),
           ("mem_pct", mem_pct), ("gmp_core_equiv", f"{s.modsq_per_s * GMP_M5_SECONDS_PER_MODSQ_100K:.4f}")], a.csv)
    return 0


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(prog="python -m montmul_b200", description=__doc__, allow_abbrev=False,
                                 formatter_class=argparse.RawDescriptionHelpFormatter)
    sub = ap.add_subparsers(dest="cmd", required=True)
    p = sub.add_parser("bench", allow_abbrev=False)
    p.add_argument("--backend", required=True)
    p.add_argument("--bits", type=int, required=True)
    p.add_argument("--slots", type=int, required=True)
    p.add_argument("--steps", type=int, required=True)
    p.add_argument("--csv")
    p = sub.add_parser("prp", allow_abbrev=False)
    p.add_argument("--backend", required=True)
    p.add_argument("--index", type=int, required=True)
    p = sub.add_parser("fermat", allow_abbrev=False)
    p.add_argument("--backend", required=True)
    p.add_argument("--slots", type=int, default=64)
    p.add_argument("--bits", type=int, default=4096)
    p.add_argument("--primes", type=int, default=4)
    p.add_argument("--seed", type=int, default=2026)
    p.add_argument("--csv")
    p = sub.add_parser("score", allow_abbrev=False)
    p.add_argument("--backend", required=True)
    p.add_argument("--slots", type=int, default=0)
    p.add_argument("--label", default="")
    p.add_argument("--csv")
    p.add_argument("--ncu", action="store_true", help="profile one step launch with Nsight Compute")
    p = sub.add_parser("ncu-launch", allow_abbrev=False, help=argparse.SUPPRESS)
    p.add_argument("--slots", type=int, required=True)
    p = sub.add_parser("sweep", allow_abbrev=False)
    p.add_argument("--bits", type=int, nargs="*", default=[1024, 8192, 32768, 100_000, 300_000, 1_000_000])
    p.add_argument("--slots", type=int, default=0, help="slots per size (0: 80%% of free memory, at most --max-slots)")
    p.add_argument("--max-slots", type=int, default=0, help="cap (0: 16 x SMs)")
    p.add_argument("--ebits", type=int, default=256)
    p = sub.add_parser("mixed", allow_abbrev=False)
    p.add_argument("--slots", type=int, default=2000)
    p.add_argument("--lo", type=int, default=8192)
    p.add_argument("--hi", type=int, default=300_000)
    p.add_argument("--ebits", type=int, default=1000)
    p.add_argument("--seed", type=int, default=7)
    p.add_argument("--quantum", type=int, default=128, help="steps per graph-replayed launch")
    p = sub.add_parser("serve", allow_abbrev=False)
    p.add_argument("--load", type=float, nargs="*", default=[0.7, 0.95])
    p.add_argument("--duration", type=float, default=40.0, help="seconds of arrivals")
    p.add_argument("--lo", type=int, default=10_000)
    p.add_argument("--hi", type=int, default=200_000)
    p.add_argument("--quantum", type=int, default=128)
    p.add_argument("--seed", type=int, default=2026)
    p.add_argument("--no-check", action="store_true")
    p.add_argument("--launch", choices=["stream", "items", "plan"], default="stream",
                   help="stream: every segment launches, reads and refills on its own; items: ticks of "
                        "per-segment launches; plan: ticks of one mixed-length launch")
    p.add_argument("--slice-ms", type=float, default=120.0, help="stream: device time budgeted per launch")
    p = sub.add_parser("tune", allow_abbrev=False)
    p.add_argument("--lengths", type=int, nargs="*", default=[1 << e for e in range(8, 18)])
    p.add_argument("--force", action="store_true")
    p.add_argument("--mixed-only", action="store_true")
    for p in sub.choices.values():
        p.add_argument("--device", type=int, default=0)
    args = sys.argv[1:] if argv is None else list(argv)
    seen = set()
    for t in args:   # a repeated option is an error, as in the reference's parser (main.rs:46)
        if t.startswith("--"):
            key = t.split("=", 1)[0]
            if key in seen:
                ap.error(f"{key} given twice")
            seen.add(key)
    a = ap.parse_args(args)
    if a.cmd == "bench":
        return cmd_bench(a)
    if a.cmd == "prp":
        return cmd_prp(a)
    if a.cmd == "score":
        return cmd_score(a)
    if a.cmd == "fermat":
        return cmd_fermat(a)
    if a.cmd == "ncu-launch":
        return cmd_ncu_launch(a)
    if a.cmd == "sweep":
        from . import sweep
        print(json.dumps(sweep.main(a)))
        return 0
    if a.cmd == "mixed":
        from . import mixed
        print(json.dumps(mixed.main(a)))
        return 0
    if a.cmd == "serve":
        from . import serve
        print(json.dumps(serve.main(a)))
        return 0
    if a.cmd == "tune":
        from . import tune
        return tune.main(["--lengths", *map(str, a.lengths), "--device", str(a.device)] + (["--force"] if a.force else [])
                         + (["--mixed-only"] if a.mixed_only else []))
    return 2


if __name__ == "__main__":
    sys.exit(main())
