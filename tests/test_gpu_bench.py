"""bench.py's own arm on one GPU, at a small size: exactly one JSON line
carrying the whole output contract (roofline, CPU baseline, end-to-end,
launch count, clocks), with figures that agree with each other."""
import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_bench_line_contract():
    n, steps = 8192, 40
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--npoly", str(n),
                        "--steps", str(steps), "--warmup", "3", "--e2e-steps", "2",
                        "--cpu-seconds", "0.5"],
                       capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [l for l in p.stdout.splitlines() if l.strip().startswith("{")]
    assert len(lines) == 1, p.stdout
    d = json.loads(lines[0])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
                "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config",
                "roofline", "cpu_baseline", "e2e", "gpu_launches", "clocks"):
        assert key in d, key
    assert d["n_gpus"] == 1 and d["steps"] == steps and d["warmup"] == 3
    assert d["higher_is_better"] is True and d["scaling"] == "weak"
    assert "workload" in d["config"] and "model" not in d["config"]
    # value: polynomials per second over the timed steps
    assert d["value"] == pytest.approx(n / (d["ms_per_step"] * 1e-3), rel=1e-6)
    r = d["roofline"]
    assert r["bound"] == "hbm" and r["unit"] == "GB/s" and r["peak"] > 0
    assert r["frac"] == pytest.approx(r["achieved"] / r["peak"], rel=1e-6)
    assert 0 < r["frac"] < 1.5
    cb = d["cpu_baseline"]
    assert cb["kind"] in ("reference", "port") and cb["cores"] >= 1 and cb["value"] > 0
    assert cb["sample"]
    e = d["e2e"]
    assert e["value"] > 0 and e["unit"] == d["unit"]
    assert e["h2d_bytes_per_step"] == 2 * n * 512 and e["d2h_bytes_per_step"] == 2 * n * 512
    assert d["gpu_launches"] == 2 * steps               # one forward + one inverse per step
    c = d["clocks"]
    assert "sm_mhz" in c and "sm_max_mhz" in c and isinstance(c["reasons"], list)
