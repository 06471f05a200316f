"""The benchmark's reference arm on the host: the JSON line it prints keeps
the fields the benchmark contract asks for, with the metric string the GPU
arm prints for the same workload (so the two arms compare), and it times
the CPU restatement with the steps it reports.  Runs on the 2000 x 7750
rank-10 workload with a small CPU budget (a few seconds)."""
from __future__ import annotations

import json
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _line(*extra):
    out = subprocess.run(
        [sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--workload", "pbmc8k",
         "--warmup", "1", "--cpu-seconds", "2", *extra],
        cwd=ROOT, capture_output=True, text=True, timeout=600, check=True)
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, out.stdout
    return json.loads(lines[0])


@pytest.mark.parametrize("method", ["lee", "brunet"])
def test_reference_arm_line(method):
    sys.path.insert(0, str(ROOT))
    import bench

    d = _line("--steps", "2", "--method", method)
    assert d["impl"] == "reference"
    assert d["metric"] == bench.iterate_metric(method, "pbmc8k")
    assert d["unit"] == "iters/s" and d["higher_is_better"] is True
    assert d["value"] > 0 and d["steps"] == 2 and d["warmup"] == 1 and d["n_gpus"] == 1
    assert d["dtype"] == "f64"
    base = d["cpu_baseline"]
    assert base["value"] == d["value"] and base["kind"] in ("port", "reference")
    assert base["cores"] >= 1 and base["sample"]
    e2e = d["e2e"]
    assert e2e["value"] == d["value"] and e2e["unit"] == d["unit"]
    assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0
    assert d["config"]["workload"] == "pbmc8k" and d["config"]["method"] == method
