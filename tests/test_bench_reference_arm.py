"""The benchmark's reference arm on the host: the JSON line it prints keeps
the fields the benchmark contract asks for, with the metric string the GPU
arm prints for the same workload (so the two arms compare), and it times
the CPU restatement with the steps it reports.  Runs on the 2000 x 7750
rank-10 workload and on the default 20000 x 200000 rank-20 one (a column
slice) with a small CPU budget (seconds)."""
from __future__ import annotations

import json
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _line(workload, *extra):
    out = subprocess.run(
        [sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--workload", workload,
         "--warmup", "1", "--cpu-seconds", "1", *extra],
        cwd=ROOT, capture_output=True, text=True, timeout=600, check=True)
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, out.stdout
    return json.loads(lines[0])


@pytest.mark.parametrize("workload,method", [("pbmc8k", "lee"), ("pbmc8k", "brunet"),
                                             ("atlas", "lee")])
def test_reference_arm_line(workload, method):
    sys.path.insert(0, str(ROOT))
    import bench

    d = _line(workload, "--steps", "2", "--method", method)
    assert d["impl"] == "reference"
    assert d["metric"] == bench.iterate_metric(method, workload)
    assert d["unit"] == "iters/s" and d["higher_is_better"] is True
    assert d["value"] > 0 and d["steps"] == 2 and d["warmup"] == 1 and d["n_gpus"] == 1
    assert d["dtype"] == "f64"
    base = d["cpu_baseline"]
    assert base["value"] == d["value"] and base["kind"] in ("port", "reference")
    assert base["cores"] >= 1 and base["sample"]
    e2e = d["e2e"]
    assert e2e["value"] == d["value"] and e2e["unit"] == d["unit"]
    assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0
    assert d["config"]["workload"] == workload and d["config"]["method"] == method
