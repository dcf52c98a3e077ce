"""The stream serving loop (montmul_b200.serve.Server with launch="stream") on the host, over a fake
segment backend whose slots keep their Montgomery state as Python integers and step it exactly
(x <- x^2 c^bit R^-1 mod N per exponent bit, as the step kernels do): every request is admitted,
stepped over several launches, read back and refilled in place; every Fermat verdict is checked
by the VerdictChecker against GMP and every mul against a b mod N; and no segment takes a refill
while one of its launches is in flight."""
import pytest

from montmul_b200 import gmp, serve
from montmul_b200.batch import Params, _setup_one

LENGTHS = [1 << e for e in range(3, 25)]


class FakeDev:
    def supported_lengths(self):
        return list(LENGTHS)

    def sm_count(self):
        return 4

    def free_memory(self):
        return 1 << 30

    def device_name(self):
        return "host fake"


class FakeBackend:
    """The part of the C ABI a segment's launches use: an item-list launch that reports busy for
    the next `latency` polls, then done."""

    def __init__(self, batch, latency=2):
        self.batch, self.latency, self.pending, self.launches = batch, latency, 0, 0

    def run_items_async(self, st, slots, steps):
        assert self.pending == 0, "a second launch while one is in flight"
        assert len(set(slots)) == len(slots) and all(s > 0 for s in steps)
        self.batch.advance(slots, steps)
        self.pending = self.latency
        self.launches += 1

    def busy(self, st):
        if self.pending:
            self.pending -= 1
        return 1 if self.pending else 0

    def sync(self, st):
        self.pending = 0

    def blocks_per_sm(self, st):
        return 2


class FakeBatch:
    def __init__(self, length, slots, base):
        self.params = Params(length // 2, length)
        self.base = base
        self.be = FakeBackend(self)
        dummy = (1 << (32 * self.params.k - 5)) | 1
        self.moduli = [_setup_one(dummy, self.params.k)[3] for _ in range(slots)]
        self.x = [0] * slots
        self.exp = [0] * slots
        self.nbits = [0] * slots
        self.pos = [0] * slots

    def backend_and_state(self):
        return self.be, None

    def prepare(self, n):
        return _setup_one(n, self.params.k)

    def refill(self, slots, moduli, xs, exps, setups=None):
        assert self.be.pending == 0, "refill while a launch of the segment is in flight"
        for i, (s, n, x, e) in enumerate(zip(slots, moduli, xs, exps)):
            su = setups[i] if setups is not None and setups[i] is not None else self.prepare(n)
            m = su[3]
            assert m.n == n
            self.moduli[s] = m
            self.x[s] = x * (1 << (32 * self.params.k)) % n     # Montgomery form x R mod N
            self.exp[s], self.nbits[s], self.pos[s] = e, e.bit_length(), 0

    def remaining(self, s):
        return self.nbits[s] - self.pos[s]

    def advance(self, slots, steps):
        for s, k in zip(slots, steps):
            m = self.moduli[s]
            for _ in range(min(k, self.remaining(s))):
                bit = (self.exp[s] >> (self.nbits[s] - 1 - self.pos[s])) & 1
                self.x[s] = self.x[s] * self.x[s] * m.rinv * (self.base if bit else 1) % m.n
                self.pos[s] += 1

    def mul(self, out, a, b):
        m = self.moduli[out]
        self.x[out] = self.x[a] * self.x[b] * m.rinv % m.n

    def read_raw_slots(self, slots):
        return [self.x[s] for s in slots]


@pytest.mark.parametrize("slice_ms", [0.0005, 0.05])
def test_stream_loop_serves_and_checks_every_request(monkeypatch, slice_ms):
    reqs = serve.stream(240, 4000.0, 40, 400, prime_frac=0.2, mul_frac=0.1, seed=11)
    checker = serve.VerdictChecker(threads=2)
    srv = serve.Server(FakeDev(), segment_slots=6, tuned=False, checker=checker, launch="stream",
                       slice_ms=slice_ms)
    segs = []

    def grow(length):
        seg = serve.Segment(FakeBatch(length, srv.segment_slots, srv.base), list(range(srv.segment_slots - 1, -1, -1)))
        srv.lanes.setdefault(length, []).append(seg)
        segs.append(seg)
        return seg

    monkeypatch.setattr(srv, "_grow", grow)
    srv.serve(reqs)
    checked = checker.finish()
    ferm = [r for r in reqs if r.kind == "fermat"]
    assert checked["verdicts"] == len(ferm) and all(r.done is not None for r in reqs)
    for r in ferm:
        assert r.verdict == (gmp.powm(3, r.n - 1, r.n) == 1)
    assert sum(r.verdict for r in ferm) >= sum(1 for r in ferm if r.prime)
    for r in reqs:
        if r.kind == "mul":
            assert r.value == r.a * r.b % r.n
    # several launches per segment, and at the finer slice more than one per request
    launches = sum(s.batch.be.launches for s in segs)
    assert launches > len(segs)
    if slice_ms < 0.001:
        assert launches > len(ferm)
    assert all(not s.active for s in segs)
