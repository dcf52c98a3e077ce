"""bench.py's reference arm on the host: the reference's two CPU backends (as the oracle restates
them) run the score workload, the faster one is reported on the bench's metric, with its CPU
baseline record and a zero-copy e2e, and both pass the pow_mod gate."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_prints_one_checked_line():
    env = dict(os.environ)
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        env.pop(k, None)
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                          "--warmup", "3"], cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["metric"] == "squarings/s @100k-bit" and d["unit"] == "modsq/s"
    assert d["value"] > 0 and d["higher_is_better"] is True and d["steps"] == 1
    assert d["config"]["backend"] in ("cpu", "gmp") and d["config"]["bits"] == 100_000
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["value"] == d["value"]
    assert d["cpu_baseline_other"]["backend"] != d["config"]["backend"]
    assert d["e2e"] == {"value": d["value"], "unit": "modsq/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
