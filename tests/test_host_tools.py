"""Host-side logic of the tools around the kernels, without a GPU: the autotuner's fixed schedule
facts, the mixed and served workloads, the CLI's sequence and percentile helpers."""
import math

import pytest

from montmul_b200 import mixed, serve, tune
from montmul_b200.__main__ import tribonacci
from montmul_b200.batch import MontMulError, Params
from montmul_b200.gmp import powm

LENGTHS = [1 << e for e in range(3, 25)]


def test_radix_schedule_covers_every_stage():
    for m in range(1, 24):
        sched = tune.radix_schedule(m)
        assert sum(int(math.log2(r)) for r in sched) == m
        assert all(r in (2, 4, 8) for r in sched)
        if m >= 5 or m == 3:
            assert sched[-1] == 8   # the fused last pass is radix 8 (m = 4 runs [4, 4])


def test_tune_candidates_by_length():
    S, G, C = tune.SHARED, tune.GLOBAL, tune.CLUSTER
    assert tune.candidates(2048) == [(S, s, 0) for s in tune.LAUNCH_STEPS]
    assert {(c[0], c[2]) for c in tune.candidates(4096)} == {(S, 0), (S, 256)}
    assert {(c[0], c[2]) for c in tune.candidates(8192)} == {(S, 0), (S, 256), (G, 0)}
    assert {(c[0], c[2]) for c in tune.candidates(16384)} == {(S, 0), (S, 1024), (G, 0)}
    assert {c[0] for c in tune.candidates(32768)} == {G, C}
    assert {c[0] for c in tune.candidates(65536)} == {G, C}
    assert {c[0] for c in tune.candidates(131072)} == {G}
    assert tune.fixed_parts(1 << 20, True)["radix"]["global"] == tune.radix_schedule(19 - 11)
    assert tune.fixed_parts(32768, C)["cluster"] == 2 and tune.fixed_parts(65536, C)["cluster"] == 4
    assert tune.fixed_parts(32768, C, 1024)["cluster"] == 4 and tune.fixed_parts(32768, C, 1024)["blocks_per_sm"] == 2
    assert {th for g, _, th in tune.candidates(32768) if g == C} == {0, 1024}
    assert {th for g, _, th in tune.candidates(65536) if g == C} == {0}
    assert {th for g, _, th in tune.candidates(32768) if g == G} == {0}
    assert [tune.mode_name(m) for m in (S, G, C, False, True)] == ["shared", "global", "cluster", "shared", "global"]


def test_tune_table_roundtrip(tmp_path, monkeypatch):
    monkeypatch.setenv("MONTMUL_B200_SCHEDULES", str(tmp_path / "s.json"))
    tune.save_table({"dev": {"8192": {"global": False, "launch_steps": 512, "step_ns": 680.0}}})
    assert tune.schedule_for("dev", 8192)["step_ns"] == 680.0
    assert tune.schedule_for("dev", 4096) is None
    assert tune.schedule_for("other", 8192) is None


def test_cluster_row_gives_way_on_the_plain_path(tmp_path, monkeypatch):
    """A batch on the plain REDC path (no wraparound) cannot run cluster mode: it takes the
    fastest measured candidate of another mode from the same row."""
    monkeypatch.setenv("MONTMUL_B200_SCHEDULES", str(tmp_path / "s.json"))
    cands = [{"global": 1, "launch_steps": 64, "step_ns": 4903.0, "block_threads": 0},
             {"global": 1, "launch_steps": 512, "step_ns": 5211.0, "block_threads": 0},
             {"global": 2, "launch_steps": 512, "step_ns": 4118.0, "block_threads": 0}]
    tune.save_table({"dev": {"32768": {"global": 2, "launch_steps": 512, "step_ns": 4118.0, "cluster": 2,
                                       "mixed_ns": 4385.0, "candidates": cands},
                             "65536": {"global": 2, "launch_steps": 512, "step_ns": 10293.0,
                                       "candidates": cands[2:]}}})
    assert tune.schedule_for("dev", 32768)["global"] == 2
    row = tune.schedule_for("dev", 32768, cluster_ok=False)
    assert (row["global"], row["launch_steps"], row["step_ns"]) == (1, 64, 4903.0) and "mixed_ns" not in row
    assert tune.schedule_for("dev", 65536, cluster_ok=False) is None
    assert tune.load_table()["dev"]["32768"]["global"] == 2   # the table itself is unchanged


class _FakeDev:
    def device_name(self):
        return "dev"

    def sm_count(self):
        return 148


def test_tune_mixed_only_remeasures_the_mixed_cost_and_keeps_schedules(tmp_path, monkeypatch):
    """`tune --mixed-only` drops each listed row's mixed-launch cost and measures it again; the
    schedule (mode, steps per launch, uniform cost) stays."""
    monkeypatch.setenv("MONTMUL_B200_SCHEDULES", str(tmp_path / "s.json"))
    tune.save_table({"dev": {"8192": {"global": False, "launch_steps": 64, "step_ns": 709.0, "slots": 1184,
                                      "steps": 600, "mixed_ns": 787.0},
                             "16384": {"global": False, "launch_steps": 512, "step_ns": 1452.0, "slots": 1184,
                                       "steps": 300}}})
    calls = []

    def fake_mixed(dev, length, slots, steps, seed=2026):
        calls.append((length, slots, steps))
        return length * 1e-13

    monkeypatch.setattr(tune, "measure_mixed", fake_mixed)
    monkeypatch.setattr(tune, "tune_length", lambda *a, **k: pytest.fail("a schedule was re-tuned"))
    tune.tune(_FakeDev(), [8192, 16384], log=lambda *_: None, mixed_only=True)
    assert calls == [(8192, 1184, 600), (16384, 1184, 300)]
    row = tune.schedule_for("dev", 8192)
    assert row["mixed_ns"] == pytest.approx(8192 * 1e-4) and row["step_ns"] == 709.0 and row["launch_steps"] == 64
    assert tune.schedule_for("dev", 16384)["mixed_ns"] == pytest.approx(16384 * 1e-4)
    # without the flag, rows that have a mixed-launch cost keep it
    tune.tune(_FakeDev(), [8192], log=lambda *_: None)
    assert len(calls) == 2


def test_mixed_workload():
    w = mixed.workload(500, 8192, 300_000, 1000, 7)
    assert w == mixed.workload(500, 8192, 300_000, 1000, 7)
    for bits, n, c, e in w:
        assert 8192 <= bits <= 300_000 and n.bit_length() == bits and n % 2 == 1
        assert c in (2, 3, 4) and e == (n - 1) >> (bits - 1000) and e.bit_length() == 1000
    # log-uniform: about half the slots below the geometric midpoint
    mid = math.sqrt(8192 * 300_000)
    below = sum(1 for bits, *_ in w if bits < mid)
    assert 200 < below < 300
    assert {Params.for_bits(b, LENGTHS).len for b, *_ in w} == {1024, 2048, 4096, 8192, 16384, 32768}


def test_admission_waits_for_an_inflight_segment_with_room():
    """A segment whose launch is on the device takes no refill; a request of its length waits
    for it while it has room, and the lane grows only when no segment has room."""
    srv = object.__new__(serve.Server)
    grown = []

    def grow(length):
        seg = serve.Segment(batch=None, free=[0, 1])
        srv.lanes.setdefault(length, []).append(seg)
        grown.append(length)
        return seg

    srv._grow = grow
    busy = serve.Segment(batch=None, free=[5, 6], inflight=True)
    srv.lanes = {8192: [busy]}
    assert srv._slots_for(8192, 1) == (None, None) and not grown
    busy.inflight = False
    seg, slots = srv._slots_for(8192, 2)
    assert seg is busy and slots == [6, 5] and not grown
    busy.inflight = True   # full and in flight: the lane grows
    seg, slots = srv._slots_for(8192, 1)
    assert grown == [8192] and seg is srv.lanes[8192][1] and slots == [1]


def test_serve_stream():
    seen = {}

    def src(rid, bits, start):
        seen[rid] = (bits, start)
        return start | 1

    r = serve.stream(400, 10.0, 10_000, 200_000, seed=3, prime_source=src)
    assert r == serve.stream(400, 10.0, 10_000, 200_000, seed=3, prime_source=lambda rid, bits, start: start | 1)
    assert all(b.arrival > a.arrival for a, b in zip(r, r[1:]))
    gaps = [b.arrival - a.arrival for a, b in zip(r, r[1:])]
    assert 0.07 < sum(gaps) / len(gaps) < 0.13   # mean 1 / rate
    kinds = [x.kind for x in r]
    assert 5 <= kinds.count("mul") <= 40
    primes = [x for x in r if x.prime]
    assert 20 <= len(primes) <= 70
    assert {x.prime for x in primes} == {"next_prime", "mersenne"}
    for x in primes:
        if x.prime == "mersenne":
            assert x.rid not in seen
            assert x.n + 1 == 1 << x.n.bit_length() and x.n.bit_length() in serve.MERSENNE_P
        else:
            bits, start = seen[x.rid]
            assert bits <= serve.PRIME_LIMIT_BITS and start.bit_length() == bits and x.n == start | 1
    for x in r:
        assert x.n % 2 == 1
        if x.kind == "mul":
            assert 0 <= x.a < x.n and 0 <= x.b < x.n


def test_serve_primes_fixture_covers_the_default_stream():
    """Every prime request of at most PRIME_LIMIT_BITS among the fixture's requests of the default
    stream (seed 2026, [10,000, 200,000] bits) takes its prime from the fixture: a base-3 Fermat
    probable prime just above the seeded start."""
    import json
    with open(serve.PRIMES_FIXTURE) as f:
        fx = json.load(f)
    assert (fx["seed"], fx["lo"], fx["hi"], fx["limit_bits"]) == (2026, 10_000, 200_000, serve.PRIME_LIMIT_BITS)
    starts = {}

    def fail(rid, bits, start):
        raise AssertionError(f"request {rid} ({bits} bits) is not in the fixture")

    r = serve.stream(fx["requests"], 1.0, 10_000, 200_000, seed=2026, prime_source=fail)
    small = [x for x in r if x.prime == "next_prime"]
    assert len(small) == len(fx["offsets"]) > 20
    for x in small:
        off = fx["offsets"][str(x.rid)]
        assert 0 < off < 100_000 and x.n.bit_length() <= serve.PRIME_LIMIT_BITS
        assert powm(3, x.n - 1, x.n) == 1


def test_verdict_checker_routes_and_rejects():
    """The served-verdict check decides pow_mod(3, N - 1, N) == 1 exactly: Mersenne primes by
    Fermat's little theorem, composites with a small factor g by 3^(N-1) mod g, the rest with
    GMP's powm; a served verdict that differs is an error."""
    p, q = 1_000_000_007, 998_244_353          # primes above the small-prime bound
    reqs = [serve.Request(0, "fermat", (1 << 4423) - 1, 0.0, prime="mersenne", verdict=True),
            serve.Request(1, "fermat", 3 * ((1 << 5000) + 1) + 0, 0.0, verdict=False),
            serve.Request(2, "fermat", 1_000_003 * ((1 << 3000) - 1), 0.0, verdict=False),
            serve.Request(3, "fermat", p * q, 0.0, verdict=False),
            serve.Request(4, "fermat", (1 << 521) - 1, 0.0, prime="next_prime", verdict=True),
            serve.Request(5, "mul", 7, 0.0)]
    c = serve.VerdictChecker(threads=2)
    for r in reqs:
        c.submit(r)
    assert c.finish() == {"mersenne_prime": 1, "small_factor": 2, "gmp_powm": 2, "verdicts": 5}
    bad = serve.VerdictChecker(threads=1)
    bad.submit(serve.Request(9, "fermat", p * q, 0.0, verdict=True))
    with pytest.raises(MontMulError, match="request 9"):
        bad.finish()


def test_capacity_and_percentile():
    reqs = [serve.Request(0, "fermat", (1 << 9999) | 1, 0.0), serve.Request(1, "fermat", (1 << 19999) | 1, 0.0),
            serve.Request(2, "mul", 7, 0.0)]
    cap = serve.capacity(reqs, lambda length: 1e-6 * length / 1024)
    work = [10_000 * 1e-6 * 1024 / 1024, 20_000 * 1e-6 * 2048 / 1024]
    assert abs(cap - 1 / (sum(work) / 2)) < 1e-9
    assert serve.percentile([3, 1, 2, 4], 0.5) == 2
    assert serve.percentile(list(range(1, 101)), 0.99) == 99


def test_tribonacci_matches_the_reference_sequence():
    assert [tribonacci(i) for i in range(10)] == [0, 0, 1, 1, 2, 4, 7, 13, 24, 44]


class _Batch:
    def __init__(self, rem):
        self.rem = rem

    def remaining(self, s):
        return self.rem[s]


class _Seg:
    def __init__(self, rem):
        self.batch = _Batch(rem)
        self.active = {s: None for s in rem}


def _server(segs, steps, ns, blocks, units=None):
    srv = serve.Server.__new__(serve.Server)
    srv.plan_segs, srv.seg_steps, srv.seg_ns, srv.blocks = segs, steps, ns, blocks
    srv.seg_units = units or [1] * len(segs)
    return srv


def test_work_list_full_budgets_when_slots_fit():
    segs = [_Seg({0: 10_000, 1: 50}), _Seg({3: 10_000})]
    items = _server(segs, [400, 128], [700.0, 2300.0], 8).work_list()
    assert sorted((b, s, n) for b, s, n, *_ in items) == [(0, 0, 400), (0, 1, 50), (1, 3, 128)]
    durs = [n * ns for _, _, n, _, ns, _ in items]
    assert durs == sorted(durs, reverse=True)


def test_work_list_packs_blocks_evenly():
    """A = W + r busy slots on W blocks: W - r full budgets and 2r half budgets, whose work fills
    every block for one budget's time."""
    w, a = 10, 14
    segs = [_Seg({s: 1_000_000 + s for s in range(a)})]
    items = _server(segs, [100], [1.0], w).work_list()
    budgets = sorted(n for _, _, n, *_ in items)
    assert budgets == [50] * 8 + [100] * 6
    assert sum(budgets) == w * 100
    # longest first, so the greedy queue pairs the halves on the remaining blocks
    assert [n for _, _, n, *_ in items] == [100] * 6 + [50] * 8


def test_work_list_larger_shares_go_to_slots_nearest_completion():
    segs = [_Seg({0: 5_000, 1: 90_000, 2: 80_000})]
    items = _server(segs, [1000], [1.0], 2).work_list()
    got = {s: n for _, s, n, *_ in items}
    assert got[0] == 1000 and got[1] == got[2] == 500


def test_work_list_counts_wide_items_as_two_workers():
    """Wide items (a whole block: both workers) count two units: 2 wide + 2 other items on
    W = 4 workers are 6 units, so the two nearest completion (the wide ones here) keep full
    budgets and the others take half; the work fills the workers for one budget's time."""
    segs = [_Seg({0: 1_000, 1: 2_000}), _Seg({0: 900_000, 1: 800_000})]
    items = _server(segs, [100, 100], [1.0, 1.0], 4, units=[2, 1]).work_list()
    got = {(b, s): n for b, s, n, *_ in items}
    assert got == {(0, 0): 100, (0, 1): 50, (1, 0): 50, (1, 1): 50}
    assert sum(n * (2 if b == 0 else 1) for (b, _), n in got.items()) == 4 * 100
