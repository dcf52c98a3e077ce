"""SM clocks and throttle reasons sampled by nvidia-smi while a measurement runs.

Every throughput figure this package prints (bench.py, and the sweep, mixed and serve commands)
carries a `clocks` record taken during its timed region: the median SM clock under load, the
maximum, and every throttle reason seen active. A figure whose record shows hw_slowdown,
hw_thermal_slowdown or sw_thermal_slowdown, or an SM clock far below the maximum with no reason,
is not a valid measurement.

    with ClockSampler(device) as clk:
        ...timed work...
    record = clk.summary()
"""
from __future__ import annotations

import os
import statistics
import subprocess
import tempfile

FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
          "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
          "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
REASONS = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")


def parse_rows(lines):
    """Rows of the nvidia-smi CSV (noheader, nounits) with at least the nine queried fields."""
    rows = []
    for line in lines:
        parts = [p.strip() for p in line.split(",")]
        if len(parts) >= 9:
            rows.append(parts)
    return rows


def summarize(rows):
    """{"sm_mhz": median, "sm_max_mhz": max, "reasons": [...], "samples": n} or None."""
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
    for r in rows:
        for name, v in zip(REASONS, r[5:9]):
            if v.lower().startswith("active"):
                reasons.add(name)
    return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
            "reasons": sorted(reasons), "samples": len(rows)}


class ClockSampler:
    """nvidia-smi polled every 200 ms on one device for the duration of a `with` block."""

    def __init__(self, device: int, period_ms: int = 200):
        self.device = device
        self.period_ms = period_ms
        self.proc = None
        self.path = None
        self.out = None

    def __enter__(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.out = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", str(self.period_ms)],
                                         stdout=self.out, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                self.proc.wait()
        if self.out is not None:
            self.out.close()

    def summary(self):
        if self.path is None:
            return None
        try:
            with open(self.path) as f:
                rows = parse_rows(f)
        finally:
            os.unlink(self.path)
            self.path = None
        return summarize(rows) if self.proc is not None else None
