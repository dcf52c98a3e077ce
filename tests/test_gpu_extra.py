"""The rest of the reference's GPU suite (montmul/tests/gpu.rs, tests/cli.rs) on the b200 backend:
no device-memory leak over create/drop cycles, two device contexts on one GPU, structured carries
at global lengths, and the CLI's bench / prp / score lines."""
import gc
import os
import subprocess
import sys

import pytest

import common
from montmul_b200 import ModBatch
from montmul_b200.gmp import RandState, powm

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dev():
    from montmul_b200 import B200
    return B200()


def test_no_leak_over_create_drop_cycles(dev):
    """tests/gpu.rs:199-225: 50 create/drop cycles leave free device memory where it was."""
    rng = RandState(3)
    moduli = [common.rand_odd(rng, 100_000) for _ in range(64)]
    b = ModBatch(dev, moduli, 3)   # tables and first-use allocations happen before the baseline
    del b
    gc.collect()
    before = dev.free_memory()
    for _ in range(50):
        b = ModBatch(dev, moduli, 3)
        b.load_all([1] * 64)
        b.set_exponent(0, 12345)
        b.run(3)
        del b
        gc.collect()
    assert before - dev.free_memory() < 64 << 20


def test_two_contexts_on_one_device():
    """tests/gpu.rs:348-357: two backends on the same GPU keep separate batches."""
    from montmul_b200 import B200
    a, b = B200(), B200()
    rng = RandState(4)
    n1, n2 = common.rand_odd(rng, 5000), common.rand_odd(rng, 40_000)
    x, y = ModBatch(a, [n1], 3), ModBatch(b, [n2], 3)
    for m, e in ((x, 77), (y, 91)):
        m.load_all([1])
        m.set_exponents([e])
    x.run(100)
    y.run(100)
    assert x.read(0) == powm(3, 77, n1) and y.read(0) == powm(3, 91, n2)


def test_carries_at_global_lengths(dev):
    """tests/gpu.rs:261-267 up to L = 65536: all-ones and sparse operands whose products carry
    through whole limb runs."""
    common.carry_stress(lambda: dev, 1 << 16)


def _cli(*args):
    env = dict(os.environ)
    return subprocess.run([sys.executable, "-m", "montmul_b200", *args], capture_output=True, text=True,
                          timeout=600, env=env)


def test_cli_bench_prints_one_result_line():
    """tests/cli.rs:1-8"""
    r = _cli("bench", "--backend", "b200", "--bits", "1000", "--slots", "2", "--steps", "20")
    assert r.returncode == 0, r.stderr
    lines = r.stdout.strip().splitlines()
    assert len(lines) == 1
    assert "backend=b200" in lines[0] and "L=64" in lines[0] and "bitsteps_per_s=" in lines[0]


def test_cli_prp_t802_is_prp():
    """tests/cli.rs:10-14"""
    r = _cli("prp", "--index", "802", "--backend", "b200")
    assert r.returncode == 0, r.stderr
    assert "prp=true" in r.stdout


def test_cli_fermat_batch_finds_the_planted_primes():
    """The CPU-sized Fermat batch on the B200: 64 x 4,096-bit moduli, 4 seeded next_prime primes,
    every value and verdict checked against pow_mod by the command itself."""
    r = _cli("fermat", "--backend", "b200")
    assert r.returncode == 0, r.stderr
    f = dict(kv.split("=", 1) for kv in r.stdout.split())
    assert f["slots"] == "64" and f["L"] == "512" and f["prp"] == "4"
    assert f["checked"] == "every_slot_pow_mod_and_verdict"


def test_cli_score_appends_to_csv(tmp_path):
    """tests/cli.rs:28-43"""
    path = tmp_path / "score.csv"
    for _ in range(2):
        r = _cli("score", "--backend", "b200", "--slots", "1", "--csv", str(path))
        assert r.returncode == 0, r.stderr
    lines = path.read_text().splitlines()
    assert len(lines) == 3
    assert lines[0].startswith("timestamp,label,device") and ",b200,1," in lines[1]


@pytest.mark.parametrize("bits", [5000, 100_000, 400_000])
def test_run_bare_leaves_x_and_advances(dev, bits):
    """Gpu::run_bare (gpu/mod.rs:109-111; lib.rs:883-927): the squaring alone, x unchanged, the
    position advanced; run then continues from the later exponent bits."""
    rng = RandState(31)
    moduli = [common.rand_odd(rng, bits) for _ in range(3)]
    exps = [common.rand_exponent(rng, 20) for _ in range(3)]
    b = ModBatch(dev, moduli, 3)
    b.load_all([7, 8, 9])
    b.set_exponents(exps)
    before = [b.read_raw(i) for i in range(3)]
    be, st = b.backend_and_state()
    be.run_bare(st, 10)
    assert [b.remaining(i) for i in range(3)] == [10, 10, 10]
    assert [b.read_raw(i) for i in range(3)] == before
    b.run(10)
    for i, (n, e) in enumerate(zip(moduli, exps)):
        x = 7 + i
        for bit in bin(e)[2:][10:]:
            x = x * x % n
            if bit == "1":
                x = x * 3 % n
        assert b.read(i) == x


def test_overhead_ratio(dev):
    """score.rs:140-159 on a small score workload: a whole step costs more than its squaring."""
    from montmul_b200.score import ScoreConfig, gpu_overhead
    r = gpu_overhead(lambda: dev, ScoreConfig(bits=100_000, slots=296, ebits=200, repeats=3, seed=2026))
    assert 1.5 < r < 6.0
