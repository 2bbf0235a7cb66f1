"""bench.py --impl reference on the CPU: the contract of its JSON line, in both forms (no GPU needed).

The reference arm times full solves of the reference CPU solver (oracle/_ref) on the bench workload; here on a 12^3
grid so that it ends in seconds.  Its line carries the keys of the bench contract, "impl": "reference", a cpu_baseline
describing the run, an e2e block with no host-device traffic, and the same `config` as the GPU arm on the reference's
setup, so the two lines describe one workload.  Its timed solves fit inside the run.
"""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVER = os.path.join(ROOT, "oracle", "_ref", "pgx_ref_driver")
KEYS = {"impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
        "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"}


@pytest.mark.skipif(not os.path.exists(DRIVER), reason="oracle/_ref not built")
@pytest.mark.parametrize("mode", ["latency", "throughput"])
def test_reference_arm_line(mode):
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--ref-mode", mode,
                          "--grid", "12", "--steps", "2", "--warmup", "1"],
                         capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [line for line in out.stdout.splitlines() if line.startswith("{")]
    assert len(lines) == 1, out.stdout
    d = json.loads(lines[0])
    assert KEYS <= set(d), KEYS - set(d)
    assert d["impl"] == "reference" and d["unit"] == "solves/s" and d["higher_is_better"] is True
    assert d["steps"] == 2 and d["warmup"] == 1 and d["value"] > 0 and d["vs_baseline"] is None
    assert d["detail"]["ref_mode"] == mode and "12^3" in d["config"]["workload"]
    sys.path.insert(0, ROOT)
    import bench
    bench.GRID = (12, 12, 12)
    assert d["config"] == bench.workload_config("reference")
    assert d["detail"]["iters"] > 0 and d["detail"]["true_rel_res"] <= 1e-8
    assert 0 < d["detail"]["timed_s"] <= d["detail"]["wall_s"]
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["value"] == d["value"] and cb["cores"] == (os.cpu_count() or 1)
    assert d["e2e"] == {"value": d["value"], "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
