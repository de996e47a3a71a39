"""bench.py's JSON line on a small graph: the keys of the benchmark contract
(value, roofline, CPU baseline, end-to-end rate, launch count, clocks,
accuracy) are present and consistent."""
import json
import subprocess
import sys

import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu


def test_bench_line_contract():
    cmd = [sys.executable, "bench.py", "--steps", "3", "--warmup", "3", "--scale", "16",
           "--no-tune", "--no-forms", "--no-multigraph", "--no-spmv"]
    p = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=900)
    assert p.returncode == 0, p.stderr[-3000:]
    lines = [json.loads(x) for x in p.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1
    line = lines[0]
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
              "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config"):
        assert k in line, k
    assert line["value"] > 0 and line["n_gpus"] == 1 and line["steps"] == 3
    assert line["config"]["workload"].startswith("pagerank_rmat16")
    roof = line["roofline"]
    assert roof["bound"] == "hbm" and roof["unit"] == "GB/s"
    assert roof["frac"] == pytest.approx(roof["achieved"] / roof["peak"])
    assert "traffic" in roof
    e2e = line["e2e"]
    assert e2e["value"] > 0 and e2e["unit"] == line["unit"]
    assert e2e["h2d_bytes_per_step"] > 0 and e2e["d2h_bytes_per_step"] > 0
    assert line["gpu_launches"] > 0
    assert {"sm_mhz", "sm_max_mhz", "reasons"} <= set(line["clocks"])
    cb = line["cpu_baseline"]
    assert cb["value"] > 0 and cb["cores"] >= 1 and cb["kind"] in ("reference", "port")
    acc = line["accuracy"]
    assert acc["l1_error_vs_fp64_fixed_point"] <= 1e-5
    assert acc["max_error_vs_fp64_fixed_point"] <= acc["l1_error_vs_fp64_fixed_point"]
    # the small workload (RMAT s16, tol 1e-4) beside the reference's OpenMP solver
    s16 = line["s16"]
    assert abs(s16["gpu_exact"]["sweeps"] - s16["cpu_reference"]["sweeps"]) <= 1
    assert s16["max_abs_diff_gpu_vs_reference"] <= 1e-6
    assert s16["gpu_exact"]["gteps"] > 0 and s16["gpu_e2e"]["gteps"] > 0
    assert line["form"] in ("blocked", "exact") and line["exact_order"]["gteps"] > 0
