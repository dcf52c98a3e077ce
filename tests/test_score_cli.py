"""The score harness and the CLI without a GPU: montmul/src/score.rs's unit tests, tests/score.rs's
fake backends (a corrupted read must get no score; repeats are re-armed and the median is taken)
and tests/cli.rs's option handling. The backend under the harness here is the oracle."""
import subprocess
import sys
import time

import numpy as np
import pytest

from montmul_b200.batch import MontMulError
from montmul_b200.score import Score, ScoreConfig, accept, mad, median, score


def _at(rate, m):
    return Score(1, rate, m, 0.0)


def test_median_and_mad():
    """score.rs:166-174"""
    assert median([5.0, 1.0, 3.0]) == 3.0
    assert median([4.0, 1.0, 3.0, 10.0]) == 3.5
    assert mad([1.0, 5.0, 3.0, 4.0, 100.0]) == 1.0
    assert mad([1.0, 4.0, 3.0, 10.0]) == 1.5


def test_acceptance_rule():
    """score.rs:176-185"""
    assert accept(_at(100.0, 0.5), _at(103.0, 0.5))
    assert not accept(_at(100.0, 0.1), _at(101.9, 0.1))
    assert not accept(_at(100.0, 2.0), _at(103.0, 0.5))
    assert not accept(_at(100.0, 0.5), _at(103.0, 1.5))
    assert not accept(_at(100.0, 0.5), _at(97.0, 0.5))


class _Delegate:
    def __init__(self, inner):
        self.inner = inner

    def __getattr__(self, name):
        return getattr(self.inner, name)


class CorruptRead(_Delegate):
    """Flips bit 0 of limb 0 when reading slot `bad` (tests/score.rs:8-48)."""

    def __init__(self, inner, bad):
        super().__init__(inner)
        self.bad = bad

    def read(self, st, i):
        v = np.array(self.inner.read(st, i), dtype=np.uint32)
        if i == self.bad:
            v[0] ^= 1
        return v


class SlowRun(_Delegate):
    """Each run that finds work sleeps for the next scripted duration (tests/score.rs:66-107)."""

    def __init__(self, inner, ms, calls):
        super().__init__(inner)
        self.ms, self.calls = ms, calls

    def run(self, st, bits):
        if self.inner.remaining(st, 0) > 0:
            n = self.calls[0]
            self.calls[0] += 1
            time.sleep(self.ms[min(n, len(self.ms) - 1)] / 1000.0)
        self.inner.run(st, bits)


def test_score_is_positive_and_checked(oracle):
    cfg = ScoreConfig(bits=1000, slots=4, ebits=100, repeats=3, seed=1)
    s = score(lambda: oracle.OracleBackend.wraparound(), cfg)
    assert s.modsq_per_s > 0 and s.mad >= 0
    assert abs(s.fermat_tests_per_hour - s.modsq_per_s * 3600 / 1000) < 1e-6 * s.modsq_per_s


def test_wrong_backend_gets_no_score(oracle):
    cfg = ScoreConfig(bits=1000, slots=4, ebits=100, repeats=1, seed=1)
    with pytest.raises(MontMulError, match="slot 3 disagrees with pow_mod"):
        score(lambda: CorruptRead(oracle.OracleBackend.wraparound(), 3), cfg)


def test_score_is_median_rate_over_reloaded_repeats(oracle):
    cfg = ScoreConfig(bits=200, slots=4, ebits=100, repeats=3, seed=1)
    calls = [0]
    s = score(lambda: SlowRun(oracle.OracleBackend.wraparound(), [0, 200, 200, 20], calls), cfg)
    want = cfg.slots * cfg.ebits / 0.200
    assert abs(s.modsq_per_s - want) < 0.3 * want
    assert s.mad < 0.1 * want
    assert calls[0] == cfg.repeats + 1


def _cli(*args):
    return subprocess.run([sys.executable, "-m", "montmul_b200", *args], capture_output=True, text=True, timeout=120)


@pytest.mark.parametrize("args", [
    ["score", "--backend", "b200", "--slot", "8"],
    ["score", "--backend", "b200", "--label", "--ncu"],
    ["score", "--backend", "b200", "--bare"],
    ["bench", "--backend", "b200", "--bits", "1000", "--slots", "1"],
    ["prp", "--backend", "b200"],
    ["bench", "--backend", "b200", "--bits", "1000", "--bits", "2000", "--slots", "1", "--steps", "20"],
])
def test_bad_options_are_rejected(args):
    """tests/cli.rs:16-26: unknown, valueless or missing options stop the parser (exit 2)."""
    r = _cli(*args)
    assert r.returncode == 2 and "usage" in r.stderr


def test_unknown_backend_is_rejected():
    r = _cli("bench", "--backend", "cpu", "--bits", "1000", "--slots", "1", "--steps", "20")
    assert r.returncode != 0 and "unknown or unavailable backend cpu" in r.stderr


def test_help_lists_the_subcommands():
    out = _cli("--help").stdout
    for cmd in ("bench", "prp", "fermat", "score", "sweep", "mixed", "serve", "tune"):
        assert cmd in out


NCU_SAMPLE = '''==PROF== Connected to process 4242 (/usr/bin/python3.12)
==PROF== Profiling "step_kernel": 0%....50%....100% - 1 pass
"ID","Process ID","Process Name","Host Name","Kernel Name","Context","Stream","Block Size","Grid Size","Device","CC","Section Name","Metric Name","Metric Unit","Metric Value"
"0","4242","python3.12","127.0.0.1","void mm::step_kernel<12, 256>(mm::SlotArgs, unsigned int, unsigned int)","1","13","(256, 1, 1)","(296, 1, 1)","0","10.0","Command line profiler metrics","gpu__compute_memory_throughput.avg.pct_of_peak_sustained_elapsed","%","1,234.5"
"0","4242","python3.12","127.0.0.1","void mm::step_kernel<12, 256>(mm::SlotArgs, unsigned int, unsigned int)","1","13","(256, 1, 1)","(296, 1, 1)","0","10.0","Command line profiler metrics","sm__throughput.avg.pct_of_peak_sustained_elapsed","%","56.78"
==PROF== Disconnected from process 4242
'''


def test_ncu_csv_parser_reads_the_last_launch():
    """main.rs:221-245: quoted rows, "Metric Name"/"Metric Value" columns, thousands separators."""
    from montmul_b200.__main__ import parse_ncu_csv
    assert parse_ncu_csv(NCU_SAMPLE) == (56.78, 1234.5)
    two = NCU_SAMPLE + NCU_SAMPLE.splitlines()[4].replace('"56.78"', '"60.5"') + "\n"
    assert parse_ncu_csv(two)[0] == 60.5


@pytest.mark.parametrize("text", ["", "==PROF== nothing\n", '"A","B"\n"1","2"\n'])
def test_ncu_csv_parser_rejects_missing_output(text):
    from montmul_b200.__main__ import parse_ncu_csv
    with pytest.raises(ValueError):
        parse_ncu_csv(text)
