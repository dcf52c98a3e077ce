"""Served Fermat stream: continuous batching of PRP tests and mul requests of different sizes
(no counterpart in the reference, whose backend runs one uniform batch at a time).

Requests arrive as a Poisson process. Each transform length has a lane: uniform batches
("segments") whose slots keep their Montgomery state and exponent on the device. A request is
admitted as soon as a slot of its length is free in a segment with no launch in flight; a lane
grows by one segment, while the device memory budget allows, only when no segment of it has room.
Finished slots are read back and refilled in place with waiting requests: no batch is drained.

Three launch policies run the segments:
  stream (default)  each segment cycles on its own CUDA stream: one item-list launch of its
                    length's uniform step kernel over its busy slots, each budgeted `slice_ms` of
                    device time at its length's full-GPU rate; when the launch is done the host
                    reads, refills and launches again, while the other segments keep running;
  items             ticks: every busy segment's item-list launch, then a wait for all of them;
  plan              ticks of one mixed-length persistent launch over a work list of every busy
                    slot (the slowest length runs `quantum` steps, the others as long).

A Fermat request loads 1, sets the exponent N - 1 and reports the verdict x == 1; a mul request
(a b mod N) takes two slots of the same modulus and one mul launch. Each request's time to
verdict runs from its arrival to the read-back of its result.

    python -m montmul_b200 serve [--load 0.7 0.95] [--duration 40] [--lo 10000] [--hi 200000]
"""
from __future__ import annotations

import json
import math
import os
import statistics
import time
from collections import deque
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass, field
from typing import Optional

from . import gmp
from .batch import ModBatch, MontMulError, Params

MAX_DRAW = 1 << 30
# Prime requests up to this size are seeded next_prime primes; above it a seeded next_prime search
# takes far longer than the run (minutes per prime at 16,000 bits, hours at 200,000), so a Mersenne
# prime 2^p - 1 of about the drawn size stands in.
PRIME_LIMIT_BITS = 16_000
# Exponents p of Mersenne primes 2^p - 1 (Lucas-Lehmer; the published list).
MERSENNE_P = (4253, 4423, 9689, 9941, 11213, 19937, 21701, 23209, 44497, 86243, 110503, 132049, 216091)
# next_prime(start) - start of the prime requests of the default stream, written by
# data/make_serve_primes.py (GMP's mpz_nextprime); other streams search at run time.
PRIMES_FIXTURE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "serve_primes.json")


@dataclass
class Request:
    rid: int
    kind: str             # "fermat" or "mul"
    n: int
    arrival: float        # seconds after the start of the run
    a: int = 0
    b: int = 0
    prime: str = ""       # "next_prime" or "mersenne" for a request drawn as a known prime
    length: int = 0
    admitted: Optional[float] = None
    done: Optional[float] = None
    verdict: Optional[bool] = None
    value: Optional[int] = None
    raw: Optional[int] = None
    setup: Optional[tuple] = None   # the modulus's host set-up, computed while the device runs


def fixture_offsets(seed: int, lo: int, hi: int, prime_frac: float, mul_frac: float,
                    prime_limit: int = PRIME_LIMIT_BITS) -> dict:
    """{rid: next_prime(start) - start} for the stream these parameters draw, if the fixture
    covers it; else {}."""
    try:
        with open(PRIMES_FIXTURE) as f:
            fx = json.load(f)
    except OSError:
        return {}
    if (fx["seed"], fx["lo"], fx["hi"], fx["prime_frac"], fx["mul_frac"], fx["limit_bits"]) != \
            (seed, lo, hi, prime_frac, mul_frac, prime_limit):
        return {}
    return {int(k): int(v) for k, v in fx["offsets"].items()}


def mersenne_near(bits: int, lo: int, hi: int) -> int:
    """The Mersenne exponent in [lo, hi] nearest to `bits` on a log scale."""
    cands = [p for p in MERSENNE_P if lo <= p <= hi] or list(MERSENNE_P)
    return min(cands, key=lambda p: abs(math.log(p / bits)))


def stream(count: int, rate: float, lo: int, hi: int, prime_frac: float = 0.1, mul_frac: float = 0.05,
           seed: int = 2026, prime_source=None, prime_limit: int = PRIME_LIMIT_BITS):
    """`count` requests with exponential inter-arrival times of mean 1/rate and bit sizes
    log-uniform in [lo, hi], all drawn from GMP's generator seeded `seed`: a `mul_frac` share are
    mul requests (random a, b below a random odd N), a `prime_frac` share are primes, the rest
    random odd N with the top bit set (composite but for a vanishing share). A prime request draws
    a random start of its size with the top bit set; up to `prime_limit` bits its N is
    next_prime(start) (from the fixture, else `prime_source(rid, bits, start)`, else computed),
    above it the Mersenne prime nearest its size stands in."""
    rng = gmp.RandState(seed)
    offsets = fixture_offsets(seed, lo, hi, prime_frac, mul_frac, prime_limit)
    out, t = [], 0.0
    for rid in range(count):
        u = (rng.random_below(MAX_DRAW - 1) + 1) / MAX_DRAW
        t += -math.log(u) / rate
        v = rng.random_below(MAX_DRAW) / MAX_DRAW
        bits = int(round(math.exp(math.log(lo) + v * (math.log(hi) - math.log(lo)))))
        kind_draw = rng.random_below(1000) / 1000.0
        if kind_draw < mul_frac:
            n = rng.random_bits(bits) | (1 << (bits - 1)) | 1
            out.append(Request(rid, "mul", n, t, a=rng.random_below(n), b=rng.random_below(n)))
        elif kind_draw < mul_frac + prime_frac:
            start = rng.random_bits(bits) | (1 << (bits - 1))
            if bits > prime_limit:
                out.append(Request(rid, "fermat", (1 << mersenne_near(bits, lo, hi)) - 1, t, prime="mersenne"))
                continue
            if rid in offsets:
                p = start + offsets[rid]
            elif prime_source is not None:
                p = prime_source(rid, bits, start)
            else:
                p = gmp.next_prime(start)
            out.append(Request(rid, "fermat", p, t, prime="next_prime"))
        else:
            n = rng.random_bits(bits) | (1 << (bits - 1)) | 1
            out.append(Request(rid, "fermat", n, t))
    return out


def per_slot_bytes(lib, length: int) -> int:
    return int(lib.mm_b200_batch_bytes(2, length, length // 64 + 1) - lib.mm_b200_batch_bytes(1, length, length // 64 + 1))


@dataclass
class Segment:
    batch: ModBatch
    free: list
    active: dict = field(default_factory=dict)   # slot -> Request
    inflight: bool = False                       # a launch of this segment is on the device


class Server:
    """Lanes of segments per transform length, run by one of the three launch policies."""

    def __init__(self, dev, base: int = 3, quantum: int = 128, segment_slots: int = 0, budget_frac: float = 0.5,
                 tuned: bool = True, checker: Optional["VerdictChecker"] = None, launch: str = "stream",
                 slice_ms: float = 120.0):
        from .backend import lib
        self.dev = dev
        self.lib = lib()
        self.base = base
        self.quantum = quantum
        self.lengths = dev.supported_lengths()
        self.segment_slots = segment_slots or 2 * 2 * dev.sm_count()
        self.budget = int(budget_frac * dev.free_memory())
        self.used = 0
        self.lanes = {}           # length -> [Segment]
        self.plan = None
        self.plan_dirty = False
        self.tuned = tuned
        self.steps_done = 0
        self.gpu_s = 0.0          # wall time inside plan launches (launch, run, wait)
        self.host_s = {"admit": 0.0, "list": 0.0, "read": 0.0}   # host time between launches
        self.ticks = []           # (t, busy slots, slot-steps run)
        from . import tune
        self.table = tune.load_table().get(dev.device_name(), {})
        self.seg_steps = []       # per plan batch: steps of one tick
        self.checker = checker    # receives every finished Fermat request
        if launch not in ("items", "plan", "stream"):
            raise MontMulError("launch must be 'items', 'plan' or 'stream'")
        self.launch = launch      # stream, items (ticks of per-segment launches) or plan (ticks of one mixed launch)
        self.slice_ms = slice_ms  # stream mode: device time one launch of a segment is budgeted
        self.sms = dev.sm_count()
        self.bps = {}             # length -> blocks of its step kernel per SM
        self.waiting = deque()    # requests waiting for a slot (serve() sets the live queue)
        self.last_tick_s = 0.0

    # ---- admission ----
    def _grow(self, length: int) -> Optional[Segment]:
        k = length // 2
        slots = self.segment_slots
        need = slots * per_slot_bytes(self.lib, length)
        if self.used + need > self.budget:
            slots = (self.budget - self.used) // per_slot_bytes(self.lib, length)
            if slots < 1:
                return None
            need = slots * per_slot_bytes(self.lib, length)
        bits = 32 * k - 4
        dummy = (1 << (bits - 1)) | 1
        b = ModBatch(self.dev, [dummy] * slots, self.base)
        b.set_exponents([0] * slots)
        if self.tuned:
            from . import tune
            tune.apply(b)
        seg = Segment(b, list(range(slots - 1, -1, -1)))
        self.lanes.setdefault(length, []).append(seg)
        self.used += need
        self.plan_dirty = True
        return seg

    def _slots_for(self, length: int, count: int):
        """`count` free slots of one segment of the lane that has no launch on the device. When
        only segments with a launch in flight have room, the request waits for one of them to
        finish (a refill cannot race the running launch); the lane grows only when no segment
        has room."""
        segs = self.lanes.get(length, [])
        for seg in segs:
            if not seg.inflight and len(seg.free) >= count:
                return seg, [seg.free.pop() for _ in range(count)]
        if any(len(seg.free) >= count for seg in segs):
            return None, None
        seg = self._grow(length)
        if seg is None or len(seg.free) < count:
            return None, None
        return seg, [seg.free.pop() for _ in range(count)]

    def admit(self, waiting: deque, now: float) -> None:
        """Admits waiting requests in arrival order while slots are free (a request that does not
        fit stays; later ones of other lengths may still pass it)."""
        fermat = {}   # segment id -> (segment, slots, requests)
        kept = deque()
        while waiting:
            r = waiting.popleft()
            if not r.length:
                r.length = Params.for_bits(r.n.bit_length(), self.lengths).len
            need = 2 if r.kind == "mul" else 1
            seg, slots = self._slots_for(r.length, need)
            if seg is None:
                kept.append(r)
                continue
            r.admitted = now
            if r.kind == "mul":
                self._mul(seg, slots, r)
                continue
            e = fermat.setdefault(id(seg), (seg, [], []))
            e[1].append(slots[0])
            e[2].append(r)
        waiting.extend(kept)
        for seg, slots, reqs in fermat.values():
            seg.batch.refill(slots, [r.n for r in reqs], [1] * len(reqs), [r.n - 1 for r in reqs],
                             [r.setup for r in reqs])
            for s, r in zip(slots, reqs):
                seg.active[s] = r
                r.setup = None

    def prepare(self, waiting, budget_s: float) -> None:
        """Host set-up of waiting requests (GMP: N', R mod N, R^-1 mod N) ahead of their
        admission, oldest first, for about `budget_s` seconds: done while the device runs a tick."""
        t_end = time.perf_counter() + budget_s
        for r in waiting:
            if time.perf_counter() > t_end:
                break
            if r.setup is not None or r.kind != "fermat":
                continue
            if not r.length:
                r.length = Params.for_bits(r.n.bit_length(), self.lengths).len
            seg = next(iter(self.lanes.get(r.length, [])), None)
            if seg is not None:
                r.setup = seg.batch.prepare(r.n)

    def _mul(self, seg: Segment, slots, r: Request) -> None:
        b = seg.batch
        b.refill(slots, [r.n, r.n], [r.a, r.b], [0, 0])
        b.mul(slots[0], slots[0], slots[1])
        m = b.moduli[slots[0]]
        r.value = gmp.mulmod(b.read_raw_slots(slots[:1])[0], m.rinv, m.n)
        r.done = time.perf_counter() - self.t0
        self.completed += 1
        seg.free.extend(slots)

    # ---- ticks ----
    def mixed_step_ns(self, length: int) -> float:
        """Cost of one slot-step of a length in the mixed launch (GPU time per slot-step with
        the whole GPU on that length), from the tuned table: the measured cost inside the mixed
        launch, else the uniform launch's."""
        row = self.table.get(str(length))
        if not row:
            n = length // 2
            return float(n * max(1, n.bit_length() - 1))
        return row.get("mixed_ns", row["step_ns"])

    def _plan(self):
        from .backend import Plan
        if self.plan is None or self.plan_dirty:
            if self.plan is not None:
                self.plan.close()
            segs = [s for L in sorted(self.lanes) for s in self.lanes[L]]
            self.plan = Plan([s.batch for s in segs], self.quantum)
            self.plan_segs = segs
            # An item's time per step on its worker is the GPU-wide cost per slot-step times the
            # workers sharing the GPU: a wide item (L = 16384) holds a whole block, the others
            # one of its two workers. Every length gets the steps that take as long as
            # `quantum` steps of the slowest, so no worker idles while the longest items of a
            # tick finish.
            self.blocks = self.plan.blocks()
            wide_blocks = self.plan.wide_blocks()
            wide = [self.plan.batch_wide(i) for i in range(len(segs))]
            self.seg_units = [max(1, self.blocks // wide_blocks) if w else 1 for w in wide]
            self.seg_ns = [self.mixed_step_ns(s.batch.params.len) * (wide_blocks if w else self.blocks)
                           for s, w in zip(segs, wide)]
            top = max(self.seg_ns)
            self.seg_steps = [max(1, int(round(self.quantum * top / c))) for c in self.seg_ns]
            self.plan_dirty = False
        return self.plan

    def work_list(self):
        """This tick's items (plan batch, slot, steps), longest first. Items are counted in
        worker units (a wide item holds the two workers of a block). With up to as many units as
        workers each item takes a full budget (the same time for every length). With more,
        A = q W + r units (0 < r <= W workers) split into (W - r) q units of 1/q of a budget and
        r (q + 1) units of 1/(q + 1), so every worker ends the tick at once (exactly for q = 1
        and no wide items); the slots nearest completion get the larger shares."""
        items = []
        for si, seg in enumerate(self.plan_segs):
            for s in seg.active:
                rem = seg.batch.remaining(s)
                items.append([si, s, self.seg_steps[si], rem, self.seg_ns[si], self.seg_units[si]])
        a, w = sum(it[5] for it in items), max(1, self.blocks)
        if a > w:
            q, r = divmod(a, w)
            if r == 0:
                q, r = q - 1, w
            big = (w - r) * q
            items.sort(key=lambda it: it[3] * it[4])
            units = 0
            for it in items:
                it[2] = max(1, it[2] // (q if units < big else q + 1))
                units += it[5]
        for it in items:
            it[2] = max(1, min(it[2], it[3]))
        items.sort(key=lambda it: -it[2] * it[4])
        return items

    def busy(self) -> int:
        return sum(len(s.active) for segs in self.lanes.values() for s in segs)

    def item_lat_ns(self, seg: Segment) -> float:
        """Time one busy slot of a segment's length takes per step while the GPU is full of its
        length: the uniform kernel's GPU time per slot-step times the slots resident at once."""
        length = seg.batch.params.len
        if length not in self.bps:
            be, st = seg.batch.backend_and_state()
            self.bps[length] = max(1, be.blocks_per_sm(st))
        row = self.table.get(str(length))
        ns = row["step_ns"] if row else float(length // 2 * max(1, (length // 2).bit_length() - 1))
        return ns * self.sms * self.bps[length]

    def item_lists(self):
        """This tick's launches: per segment with busy slots, (segment, slots, steps), costliest
        length first. Every item gets the steps that take as long as `quantum` steps of the
        slowest busy length; when the busy slots need more blocks than the SMs hold at once (an
        item of length L takes 1 / blocks_per_sm(L) of an SM), every budget shrinks by that
        ratio, so a tick still lasts about one quantum of the slowest length."""
        segs = [seg for segs in self.lanes.values() for seg in segs if seg.active]
        if not segs:
            return []
        lat = {id(seg): self.item_lat_ns(seg) for seg in segs}
        top = max(lat.values())
        units = sum(len(seg.active) / self.bps[seg.batch.params.len] for seg in segs)
        scale = min(1.0, self.sms / units)
        jobs = []
        for seg in sorted(segs, key=lambda sg: -lat[id(sg)]):
            base = self.quantum * top / lat[id(seg)] * scale
            slots, steps = [], []
            for s in seg.active:
                rem = seg.batch.remaining(s)
                slots.append(s)
                steps.append(max(1, min(rem, int(round(base)))))
            order = sorted(range(len(slots)), key=lambda i: -steps[i])
            jobs.append((seg, [slots[i] for i in order], [steps[i] for i in order]))
        return jobs

    def tick(self) -> int:
        """One quantum on every busy slot, then the finished slots are read and freed."""
        t = time.perf_counter()
        if self.launch == "plan":
            plan = self._plan()
            items = self.work_list()
            run = sum(it[2] for it in items)
            t1 = time.perf_counter()
            self.host_s["list"] += t1 - t
            plan.run_items([it[0] for it in items], [it[1] for it in items], [it[2] for it in items])
        else:
            jobs = self.item_lists()
            run = sum(sum(steps) for _, _, steps in jobs)
            t1 = time.perf_counter()
            self.host_s["list"] += t1 - t
            for seg, slots, steps in jobs:
                be, st = seg.batch.backend_and_state()
                be.run_items_async(st, slots, steps)
            if self.waiting:
                # The launches run on the device; prepare waiting requests meanwhile (most of a
                # tick's host work), leaving time to collect the results.
                self.prepare(self.waiting, 0.8 * self.last_tick_s)
            for seg, _, _ in jobs:
                be, st = seg.batch.backend_and_state()
                be.sync(st)
        t2 = time.perf_counter()
        self.gpu_s += t2 - t1
        self.last_tick_s = t2 - t1
        now = t2 - self.t0
        self.steps_done += run
        self.ticks.append((now, self.busy(), run))
        finished = 0
        for segs in self.lanes.values():
            for seg in segs:
                done = [s for s in seg.active if seg.batch.remaining(s) == 0]
                if not done:
                    continue
                raws = seg.batch.read_raw_slots(done)
                for s, raw in zip(done, raws):
                    r = seg.active.pop(s)
                    m = seg.batch.moduli[s]
                    r.raw = raw
                    r.verdict = raw == m.r or raw == m.r + m.n
                    r.done = now
                    if self.checker is not None:
                        self.checker.submit(r)
                    seg.free.append(s)
                    finished += 1
        self.host_s["read"] += time.perf_counter() - t2
        return finished

    def serve(self, reqs):
        """Runs the whole stream in real time; returns the requests with their results."""
        if self.launch == "stream":
            return self.serve_stream(reqs)
        pending = deque(sorted(reqs, key=lambda r: r.arrival))
        waiting = deque()
        self.waiting = waiting
        self.last_tick_s = 0.0
        self.t0 = time.perf_counter()
        self.completed = 0
        while self.completed < len(reqs):
            now = time.perf_counter() - self.t0
            while pending and pending[0].arrival <= now:
                waiting.append(pending.popleft())
            if waiting:
                t = time.perf_counter()
                self.admit(waiting, now)
                self.host_s["admit"] += time.perf_counter() - t
            if self.busy():
                self.completed += self.tick()
            elif pending and not waiting:
                time.sleep(max(0.0, min(0.05, pending[0].arrival - (time.perf_counter() - self.t0))))
            elif waiting and not self.busy():
                raise MontMulError("a request fits no lane within the memory budget")
        return reqs

    def _collect(self, seg: Segment, now: float) -> int:
        """After a segment's launch has finished: its errors, its finished slots read and freed."""
        be, st = seg.batch.backend_and_state()
        be.sync(st)
        seg.inflight = False
        done = [s for s in seg.active if seg.batch.remaining(s) == 0]
        if not done:
            return 0
        raws = seg.batch.read_raw_slots(done)
        for s, raw in zip(done, raws):
            r = seg.active.pop(s)
            m = seg.batch.moduli[s]
            r.raw = raw
            r.verdict = raw == m.r or raw == m.r + m.n
            r.done = now
            if self.checker is not None:
                self.checker.submit(r)
            seg.free.append(s)
        return len(done)

    def _launch(self, seg: Segment, slice_ns: float) -> int:
        """One launch over the segment's busy slots, each budgeted about `slice_ns` of device time
        (its length's time per step with the GPU full); returns the slot-steps enqueued."""
        steps = max(1, int(slice_ns / self.item_lat_ns(seg)))
        slots = sorted(seg.active, key=lambda s: -min(seg.batch.remaining(s), steps))
        budget = [max(1, min(seg.batch.remaining(s), steps)) for s in slots]
        be, st = seg.batch.backend_and_state()
        be.run_items_async(st, slots, budget)
        seg.inflight = True
        return sum(budget)

    def serve_stream(self, reqs):
        """The stream without ticks: every segment runs its own cycle of launch, read, refill and
        launch again on its own stream, at most one launch in flight per segment; the host
        services whichever segment's launch has finished while the others keep the device busy,
        and prepares waiting requests while it would otherwise wait."""
        pending = deque(sorted(reqs, key=lambda r: r.arrival))
        waiting = deque()
        self.waiting = waiting
        self.t0 = time.perf_counter()
        self.completed = 0
        slice_ns = self.slice_ms * 1e6
        while self.completed < len(reqs):
            now = time.perf_counter() - self.t0
            while pending and pending[0].arrival <= now:
                waiting.append(pending.popleft())
            segs = [seg for segs in self.lanes.values() for seg in segs]
            progressed = False
            t = time.perf_counter()
            for seg in segs:
                if seg.inflight and not seg.batch.backend_and_state()[0].busy(seg.batch.backend_and_state()[1]):
                    self.completed += self._collect(seg, time.perf_counter() - self.t0)
                    progressed = True
            t1 = time.perf_counter()
            self.host_s["read"] += t1 - t
            if waiting:
                self.admit(waiting, now)
                progressed = True
            t2 = time.perf_counter()
            self.host_s["admit"] += t2 - t1
            for seg in [seg for segs in self.lanes.values() for seg in segs]:
                if not seg.inflight and seg.active:
                    run = self._launch(seg, slice_ns)
                    self.steps_done += run
                    self.ticks.append((time.perf_counter() - self.t0, self.busy(), run))
                    progressed = True
            self.host_s["list"] += time.perf_counter() - t2
            if waiting:
                self.prepare(waiting, 0.002)
            if not progressed:
                if not any(seg.inflight for segs in self.lanes.values() for seg in segs):
                    if waiting:
                        raise MontMulError("a request fits no lane within the memory budget")
                    if pending:
                        time.sleep(max(0.0, min(0.05, pending[0].arrival - (time.perf_counter() - self.t0))))
                else:
                    time.sleep(0.0002)
        self.gpu_s = time.perf_counter() - self.t0 - sum(self.host_s.values())
        return reqs

    def close(self):
        if self.plan is not None:
            self.plan.close()
            self.plan = None


def capacity(reqs, step_s) -> float:
    """Fermat tests per second the GPU completes at full occupancy for this request mix:
    1 / the mean of (exponent bits x seconds per slot-step at the request's length)."""
    work = [r.n.bit_length() * step_s(Params.for_bits(r.n.bit_length(), _LENGTHS).len) for r in reqs
            if r.kind == "fermat"]
    return 1.0 / statistics.mean(work)


_LENGTHS = [1 << e for e in range(3, 25)]


def odd_primes_below(bound: int):
    """The odd primes below `bound` (sieve of Eratosthenes over odd numbers)."""
    s = bytearray([1]) * (bound // 2)   # s[i] stands for 2 i + 1
    s[0] = 0
    i = 1
    while (2 * i + 1) ** 2 < bound:
        if s[i]:
            p = 2 * i + 1
            s[p * p // 2::p] = bytes(len(range(p * p // 2, bound // 2, p)))
        i += 1
    return [2 * i + 1 for i in range(bound // 2) if s[i]]


def product(v):
    while len(v) > 1:
        v = [v[i] * v[i + 1] if i + 1 < len(v) else v[i] for i in range(0, len(v), 2)]
    return v[0]


class VerdictChecker:
    """Decides, for every served Fermat request, the verdict rug's pow_mod(3, N - 1, N) == 1 gives,
    in a host thread pool while the stream runs, and requires the served verdict to equal it.
    Each decision is exact, by the cheapest of three routes:

      - N a Mersenne prime 2^p - 1 (proven prime): 3^(N-1) = 1 mod N by Fermat's little theorem;
      - N with a factor below SMALL_PRIME_BOUND: g = gcd(N, product of those primes) > 1, and if
        3^(N-1) mod g != 1 then 3^(N-1) mod N != 1 (g divides N), so the verdict is false;
      - otherwise (no small factor, the next_prime primes, or 3^(N-1) = 1 mod g): GMP's mpz_powm
        itself, the call rug's pow_mod makes.

    GMP releases the interpreter lock inside each call, so the pool runs beside the serving loop."""

    SMALL_PRIME_BOUND = 1 << 20

    def __init__(self, threads: int = 0):
        self.threads = threads or max(1, (os.cpu_count() or 2) - 2)
        self.small = product(odd_primes_below(self.SMALL_PRIME_BOUND))
        self.ex = ThreadPoolExecutor(self.threads)
        self.futs = []

    def submit(self, r: Request) -> None:
        if r.kind == "fermat":
            self.futs.append(self.ex.submit(self._one, r))

    def _one(self, r: Request) -> str:
        if r.prime == "mersenne":
            want, how = True, "mersenne_prime"
        else:
            want, how = None, "gmp_powm"
            g = gmp.gcd(r.n, self.small)
            if g > 1 and gmp.powm(3, r.n - 1, g) != 1:
                want, how = False, "small_factor"
            if want is None:
                want = gmp.powm(3, r.n - 1, r.n) == 1
        if r.verdict != want:
            raise MontMulError(f"request {r.rid} ({r.n.bit_length()} bits): verdict {r.verdict} disagrees with "
                               f"pow_mod ({want}, by {how})")
        return how

    def finish(self) -> dict:
        out = {"mersenne_prime": 0, "small_factor": 0, "gmp_powm": 0}
        try:
            for f in self.futs:
                out[f.result()] += 1
        finally:
            self.ex.shutdown(wait=True, cancel_futures=True)
        out["verdicts"] = sum(out.values())
        return out


def check(dev, reqs, checked: dict, sample: int = 24, seed: int = 2027) -> dict:
    """The served results beyond the verdicts (`checked`, from VerdictChecker): every mul against
    a b mod N, every drawn prime a PRP, and `sample` seeded requests run again alone, one uniform
    batch per length, ending with the same raw Montgomery limbs as in the mix (the uniform batches
    are the path the test suite pins to the reference Cpu backend)."""
    out = dict(checked)
    out.update({"mul": 0, "primes": 0, "alone": 0})
    ferm = [r for r in reqs if r.kind == "fermat"]
    if out["verdicts"] != len(ferm):
        raise MontMulError(f"{out['verdicts']} verdicts checked of {len(ferm)} Fermat requests")
    for r in reqs:
        if r.kind == "mul":
            if r.value != r.a * r.b % r.n:
                raise MontMulError(f"request {r.rid}: mul disagrees")
            out["mul"] += 1
        elif r.prime:
            if not r.verdict:
                raise MontMulError(f"request {r.rid}: the prime of {r.n.bit_length()} bits was not a PRP")
            out["primes"] += 1
    rng = gmp.RandState(seed)
    pool = list(ferm)
    picked = []
    while pool and len(picked) < sample:
        picked.append(pool.pop(rng.random_below(len(pool))))
    by_len = {}
    for r in picked:
        by_len.setdefault(r.length, []).append(r)
    for group in by_len.values():
        b = ModBatch(dev, [r.n for r in group], 3)
        b.load_all([1] * len(group))
        b.set_exponents([r.n - 1 for r in group])
        while any(b.remaining(i) for i in range(len(group))):
            b.run(1 << 20)
        for i, r in enumerate(group):
            if b.read_raw(i) != r.raw:
                raise MontMulError(f"request {r.rid}: served result differs from the same test run alone")
            out["alone"] += 1
    return out


def percentile(v, q: float) -> float:
    s = sorted(v)
    if not s:
        return float("nan")
    i = min(len(s) - 1, max(0, int(math.ceil(q * len(s))) - 1))
    return s[i]


def summarize(server: Server, reqs, uniform_modsq: float, rate: float, cap: float) -> dict:
    ferm = [r for r in reqs if r.kind == "fermat"]
    muls = [r for r in reqs if r.kind == "mul"]
    lat = [r.done - r.arrival for r in ferm]
    end = max(r.done for r in reqs)
    steps = sum(r.n.bit_length() for r in ferm)
    # Steady window: the second half of the arrivals, when the stream has filled the GPU and is
    # not yet draining.
    t_b = max(r.arrival for r in reqs)
    t_a = t_b / 2
    win = [(t, run) for t, _, run in server.ticks if t_a <= t <= t_b]
    win_modsq = (sum(run for _, run in win) / (win[-1][0] - win[0][0])) if len(win) > 2 else None
    return {
        "offered_tests_per_s": rate, "capacity_tests_per_s": cap, "load": rate / cap,
        "requests": len(reqs), "fermat": len(ferm), "mul": len(muls),
        "primes": sum(1 for r in ferm if r.prime), "next_prime_primes": sum(1 for r in ferm if r.prime == "next_prime"),
        "mersenne_primes": sum(1 for r in ferm if r.prime == "mersenne"), "prp": sum(1 for r in ferm if r.verdict),
        "seconds": end, "tests_per_hour": 3600.0 * len(ferm) / end,
        "modsq_per_s": steps / end, "steady_modsq_per_s": win_modsq,
        "uniform_modsq_per_s": uniform_modsq,
        "steady_over_uniform": (win_modsq / uniform_modsq) if win_modsq else None,
        "p50_s": percentile(lat, 0.5), "p99_s": percentile(lat, 0.99),
        "mul_p50_s": percentile([r.done - r.arrival for r in muls], 0.5) if muls else None,
        "ticks": len(server.ticks), "quantum": server.quantum, "launch": server.launch, "slice_ms": server.slice_ms,
        "busy_slots_p50": percentile([b for t, b, _ in server.ticks if t_a <= t <= t_b], 0.5),
        "launch_time_frac": server.gpu_s / end,
        "host_time_frac": {k: v / end for k, v in server.host_s.items()},
        "lanes": {str(L): sum(len(s.batch.moduli) for s in segs) for L, segs in server.lanes.items()},
        "device_bytes": server.used,
    }


def main(args) -> dict:
    from .backend import B200
    from .clocks import ClockSampler
    from . import tune
    dev = B200(device=args.device)
    lengths = dev.supported_lengths()
    # Seconds per slot-step at full occupancy per length (the tuned table, measured if absent).
    need = sorted({Params.for_bits(b, lengths).len for b in (args.lo, args.hi)} | {1 << e for e in range(10, 15)})
    per = tune.tune(dev, [L for L in need if args.lo <= 16 * L and L <= 2 * Params.for_bits(args.hi, lengths).len],
                    log=lambda *_: None)

    def step_s(length):
        return per[str(length)]["step_ns"] * 1e-9

    probe = stream(2000, 1.0, args.lo, args.hi, seed=args.seed)
    cap = capacity(probe, step_s)
    # The plain uniform-batch rate of the same mix: its steps over their uniform-batch time.
    ferm = [r for r in probe if r.kind == "fermat"]
    uniform = sum(r.n.bit_length() for r in ferm) / sum(
        r.n.bit_length() * step_s(Params.for_bits(r.n.bit_length(), lengths).len) for r in ferm)
    results, pending = [], []
    for load in args.load:
        rate = load * cap
        count = max(8, int(round(rate * args.duration)))
        reqs = stream(count, rate, args.lo, args.hi, seed=args.seed)
        # Each load's verdict checks keep running (in their own host threads) while the next
        # load is served; they are all collected at the end.
        checker = None if args.no_check else VerdictChecker()
        srv = Server(dev, quantum=args.quantum, checker=checker, launch=args.launch, slice_ms=args.slice_ms)
        with ClockSampler(args.device) as clk:
            srv.serve(reqs)
        srv.close()
        s = summarize(srv, reqs, uniform, rate, cap)
        s["clocks"] = clk.summary()
        results.append(s)
        pending.append((s, reqs, checker))
    for s, reqs, checker in pending:
        s["checked"] = check(dev, reqs, checker.finish()) if checker is not None else None
    return {"workload": f"Poisson arrivals for {args.duration} s, bits log-uniform in [{args.lo}, {args.hi}], "
                        f"10% primes (seeded next_prime up to {PRIME_LIMIT_BITS} bits, Mersenne primes of about the "
                        f"drawn size above), 5% mul, full base-3 Fermat tests (seed {args.seed})",
            "loads": results}
