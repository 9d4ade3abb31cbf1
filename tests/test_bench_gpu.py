"""bench.py keeps its output contract on a B200: one JSON line from a short run of the default
workload with every key the contract names, a roofline object with the measured peak, and an
end-to-end number measured separately from the device-timed value."""

from __future__ import annotations

import json
import os
import subprocess
import sys

import pytest

from conftest import cuda_ready

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not cuda_ready(), reason="needs CUDA and libdrift_pt.so")]

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_default_bench_line_has_the_contract_keys():
    r = subprocess.run([sys.executable, "bench.py", "--rounds", "20", "--steps", "2", "--warmup", "3",
                        "--no-cpu-baseline"], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    line = json.loads(lines[0])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
                "vs_baseline", "dtype", "data", "config", "roofline", "e2e", "gpu_launches", "clocks"):
        assert key in line, key
    assert line["metric"] == "spin-flips/ns" and line["higher_is_better"] is True and line["n_gpus"] == 1
    assert line["steps"] == 2 and line["warmup"] == 3 and line["value"] > 0 and line["gpu_launches"] > 0
    assert "workload" in line["config"]
    rf = line["roofline"]
    for key in ("bound", "achieved", "peak", "unit", "frac", "traffic"):
        assert key in rf, key
    assert rf["bound"] in ("hbm", "tensor") and rf["frac"] == pytest.approx(rf["achieved"] / rf["peak"])
    e2e = line["e2e"]
    for key in ("value", "unit", "h2d_bytes_per_step", "d2h_bytes_per_step"):
        assert key in e2e, key
    assert e2e["value"] > 0 and e2e["value"] != line["value"] and e2e["h2d_bytes_per_step"] > 0
    assert "sm_mhz" in line["clocks"] and "reasons" in line["clocks"]
