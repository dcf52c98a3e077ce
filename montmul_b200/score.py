"""Efficiency score: sustained modular squarings per second on one fixed workload, reported only
after the results match GMP (restating montmul/src/score.rs).

The standard workload is 100,000-bit random odd moduli (L = 8,192, k = 4,096), seed 2026,
base 3, exponent = the top 2,000 bits of N - 1, a 64-step warm-up and the median of 5 timed
repeats; slot 0, the last slot and two seeded random slots are checked against pow_mod.
"""
from __future__ import annotations

import time
from dataclasses import dataclass
from typing import Callable, Optional

from . import gmp
from .batch import ModBatch, MontMulError

# Median seconds per modular squaring of `Gmp` with one slot on one Apple M5 performance core at
# 100,000 bits, as the reference publishes it (score.rs:9-13).
GMP_M5_SECONDS_PER_MODSQ_100K = 2.709e-4


@dataclass(frozen=True)
class ScoreConfig:
    bits: int
    slots: int
    ebits: int
    repeats: int
    seed: int

    @staticmethod
    def standard(slots: int) -> "ScoreConfig":
        """The score workload (score.rs:24-29)."""
        return ScoreConfig(bits=100_000, slots=slots, ebits=2_000, repeats=5, seed=2026)


@dataclass
class Score:
    slots: int
    modsq_per_s: float
    mad: float
    fermat_tests_per_hour: float
    overhead: Optional[float] = None


def workload(cfg: ScoreConfig):
    """Random odd moduli with the top bit set and the top `ebits` bits of N - 1 (score.rs:44-61)."""
    if cfg.slots <= 0 or cfg.repeats <= 0:
        raise MontMulError("slots and repeats must be positive")
    if not 0 < cfg.ebits <= cfg.bits:
        raise MontMulError("ebits must be in 1..=bits")
    rng = gmp.RandState(cfg.seed)
    moduli = []
    for _ in range(cfg.slots):
        n = rng.random_bits(cfg.bits)
        moduli.append(n | (1 << (cfg.bits - 1)) | 1)
    shift = cfg.bits - cfg.ebits
    return moduli, [(n - 1) >> shift for n in moduli]


def fermat_workload(slots: int = 64, bits: int = 4096, primes: int = 4, seed: int = 2026):
    """The CPU-sized Fermat batch: `slots` random odd `bits`-bit moduli (top and bottom bits set,
    GMP's default generator seeded `seed`, as score.rs:45-61 draws its moduli), then `primes`
    distinct slot positions drawn from the same stream, each replaced by next_prime of a random
    `bits`-bit start with the top bit set, so both verdicts occur. Returns (moduli, positions of
    the primes, sorted)."""
    if slots <= 0 or not 0 <= primes <= slots or bits < 3:
        raise MontMulError("need slots > 0, 0 <= primes <= slots and bits >= 3")
    rng = gmp.RandState(seed)
    moduli = [rng.random_bits(bits) | (1 << (bits - 1)) | 1 for _ in range(slots)]
    pos = []
    while len(pos) < primes:
        p = rng.random_below(slots)
        if p not in pos:
            pos.append(p)
    for p in pos:
        while True:
            q = gmp.next_prime(rng.random_bits(bits) | (1 << (bits - 1)))
            if q.bit_length() == bits:
                break
        moduli[p] = q
    return moduli, sorted(pos)


def fermat_checked(backend, moduli, base: int = 3, chunk: int = 1 << 16):
    """The Fermat driver (batch.rs:187-198) with every slot checked: the value left in slot i must
    equal pow_mod(base, N_i - 1, N_i) and its verdict must be (that value == 1). Returns
    (verdicts, raw Montgomery values, seconds spent in run)."""
    b = ModBatch(backend, moduli, base)
    b.load_all([1] * b.slots())
    b.set_exponents([m.n - 1 for m in b.moduli])
    secs = 0.0
    while any(b.remaining(i) > 0 for i in range(b.slots())):
        t = time.perf_counter()
        b.run(chunk)
        secs += time.perf_counter() - t
    verdicts, raws = [], []
    for i, m in enumerate(b.moduli):
        want = gmp.powm(base, m.n - 1, m.n)
        if b.read(i) != want:
            raise MontMulError(f"slot {i} disagrees with pow_mod")
        v = b.is_one(i)
        if v != (want == 1):
            raise MontMulError(f"slot {i}: verdict disagrees with pow_mod")
        verdicts.append(v)
        raws.append(b.read_raw(i))
    return verdicts, raws, secs


def arm(batch: ModBatch, exps) -> None:
    """Loads 1 and the exponent into every slot (score.rs:63-69)."""
    batch.load_all([1] * len(exps))
    batch.set_exponents(exps)


def median(v) -> float:
    s = sorted(v)
    m = len(s) // 2
    return s[m] if len(s) % 2 else (s[m - 1] + s[m]) / 2


def mad(v) -> float:
    """Median absolute deviation from the median (score.rs:78-82)."""
    m = median(v)
    return median([abs(x - m) for x in v])


def accept(old: Score, new: Score) -> bool:
    """Hill-climb acceptance: >= 2 % faster and by more than twice the larger MAD (score.rs:84-89)."""
    gain = new.modsq_per_s - old.modsq_per_s
    return gain >= 0.02 * old.modsq_per_s and gain > 2.0 * max(old.mad, new.mad)


def checked_slots(cfg: ScoreConfig):
    """Slot 0, the last slot and two slots drawn from GMP seeded with seed + 1 (score.rs:105-110)."""
    rng = gmp.RandState(cfg.seed + 1)
    return [0, cfg.slots - 1] + [rng.random_below(cfg.slots) for _ in range(2)]


def verify(batch: ModBatch, cfg: ScoreConfig, moduli, exps) -> None:
    for i in checked_slots(cfg):
        want = gmp.powm(3, exps[i], moduli[i])
        if batch.remaining(i) != 0 or batch.read(i) != want:
            raise MontMulError(f"slot {i} disagrees with pow_mod")


def score(make: Callable, cfg: ScoreConfig, timer: Optional[Callable] = None) -> Score:
    """One warm-up run(64), then `repeats` timed run(ebits) on freshly loaded slots
    (score.rs:91-123). `timer(batch, bits)` may replace the wall clock with device timing; it
    returns seconds."""
    moduli, exps = workload(cfg)
    batch = ModBatch(make(), moduli, 3)
    arm(batch, exps)
    batch.run(64)
    rates = []
    for _ in range(cfg.repeats):
        arm(batch, exps)
        if timer is None:
            t = time.perf_counter()
            batch.run(cfg.ebits)
            secs = time.perf_counter() - t
        else:
            secs = timer(batch, cfg.ebits)
        rates.append(cfg.slots * cfg.ebits / secs)
    verify(batch, cfg, moduli, exps)
    m = median(rates)
    return Score(cfg.slots, m, mad(rates), m * 3600.0 / cfg.bits)


def gpu_overhead(make: Callable, cfg: ScoreConfig) -> float:
    """Median time of run over that of run_bare on the score workload (score.rs:140-159): the cost
    of a whole step relative to its squaring."""
    moduli, exps = workload(cfg)
    batch = ModBatch(make(), moduli, 3)
    be, st = batch.backend_and_state()

    def timed(bare: bool) -> float:
        arm(batch, exps)
        t = time.perf_counter()
        if bare:
            be.run_bare(st, cfg.ebits)
        else:
            batch.run(cfg.ebits)
        return time.perf_counter() - t

    timed(False)
    timed(True)
    full = [timed(False) for _ in range(cfg.repeats)]
    bare = [timed(True) for _ in range(cfg.repeats)]
    return median(full) / median(bare)


def best_slots(make: Callable, bits: int, candidates) -> int:
    """The candidate slot count with the highest score at ebits = 200, one repeat (score.rs:125-136)."""
    if not candidates:
        raise MontMulError("no candidate slot counts")
    best = (candidates[0], 0.0)
    for slots in candidates:
        s = score(make, ScoreConfig(bits=bits, slots=slots, ebits=200, repeats=1, seed=2026))
        if s.modsq_per_s > best[1]:
            best = (slots, s.modsq_per_s)
    return best[0]
