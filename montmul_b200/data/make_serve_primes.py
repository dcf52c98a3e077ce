"""Writes serve_primes.json: the seeded next_prime primes of the default served stream.

The served stream (montmul_b200.serve.stream, GMP's generator seeded 2026, sizes log-uniform in
[10,000, 200,000] bits, 10% primes, 5% mul) draws for each prime request a random start of its
size with the top bit set; up to serve.PRIME_LIMIT_BITS its modulus is next_prime(start). Finding
those primes takes seconds to minutes each, so this script finds them once, with GMP's
mpz_nextprime on every host core, for the first `--requests` requests, and stores each as the
offset next_prime(start) - start keyed by request id: the stream re-draws the start and adds
the offset.

    python -m montmul_b200.data.make_serve_primes [--requests 4000] [--jobs N]
"""
from __future__ import annotations

import argparse
import json
import multiprocessing as mp
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))


def _next_prime(job):
    rid, bits, start = job
    from montmul_b200 import gmp
    t = time.perf_counter()
    p = gmp.next_prime(start)
    return rid, bits, p - start, time.perf_counter() - t


def main(argv=None) -> int:
    from montmul_b200 import serve
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--requests", type=int, default=4000)
    ap.add_argument("--seed", type=int, default=2026)
    ap.add_argument("--lo", type=int, default=10_000)
    ap.add_argument("--hi", type=int, default=200_000)
    ap.add_argument("--jobs", type=int, default=os.cpu_count() or 1)
    ap.add_argument("--out", default=os.path.join(HERE, "serve_primes.json"))
    a = ap.parse_args(argv)
    jobs = []

    def collect(rid, bits, start):
        jobs.append((rid, bits, start))
        return start   # placeholder; the stream drawn here is discarded

    # The stream must be drawn without the fixture, so every prime request reaches the hook.
    saved = serve.PRIMES_FIXTURE
    serve.PRIMES_FIXTURE = os.path.join(HERE, "does-not-exist.json")
    try:
        serve.stream(a.requests, 1.0, a.lo, a.hi, seed=a.seed, prime_source=collect)
    finally:
        serve.PRIMES_FIXTURE = saved
    print(f"{len(jobs)} prime requests of at most {serve.PRIME_LIMIT_BITS} bits among {a.requests}", flush=True)
    offsets = {}
    t0 = time.perf_counter()
    with mp.get_context("spawn").Pool(a.jobs) as pool:
        for rid, bits, off, dt in pool.imap_unordered(_next_prime, sorted(jobs, key=lambda j: -j[1])):
            offsets[str(rid)] = off
            print(f"  request {rid}: {bits} bits, offset {off}, {dt:.1f} s", flush=True)
    fx = {"seed": a.seed, "lo": a.lo, "hi": a.hi, "prime_frac": 0.1, "mul_frac": 0.05,
          "limit_bits": serve.PRIME_LIMIT_BITS, "requests": a.requests,
          "generator": "GMP mpz_nextprime of the stream's seeded start (python -m montmul_b200.data.make_serve_primes)",
          "offsets": dict(sorted(offsets.items(), key=lambda kv: int(kv[0])))}
    with open(a.out, "w") as f:
        json.dump(fx, f, indent=0)
        f.write("\n")
    print(f"wrote {a.out}: {len(offsets)} primes in {time.perf_counter() - t0:.0f} s")
    return 0


if __name__ == "__main__":
    sys.exit(main())
