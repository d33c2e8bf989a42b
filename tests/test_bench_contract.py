"""The benchmark's command-line contract, checked without a GPU:

* `bench.py --impl reference` (the reference CPU backend, built from the
  reference sources into oracle/_ref) prints one JSON line with the
  contract's keys, its `cpu_baseline` (both the tile-pool and serial
  timings) and an `e2e` object of its own value;
* the CUDA arm exits non-zero without a GPU (no CPU fallback).
"""
import json
import subprocess
import sys
from pathlib import Path

import pytest

import refdrive

ROOT = Path(__file__).resolve().parents[1]
KEYS = {"metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
        "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config"}


@pytest.mark.skipif(not refdrive.available(), reason="reference library not built")
def test_reference_arm_json_line():
    p = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference",
                        "--config", "config1", "--steps", "1", "--warmup", "1"],
                       capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [l for l in p.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert KEYS <= set(d) and d["impl"] == "reference"
    assert d["metric"] == d["unit"] == "Mpix/s" and d["higher_is_better"] is True
    assert d["value"] > 0 and d["config"]["workload"].startswith("config1")
    # the driver's warm-up count is honoured, and the config object is the CUDA arm's
    assert d["warmup"] == 1 and d["steps"] >= 1
    sys.path.insert(0, str(ROOT))
    import bench
    sc, desc = bench.workload("config1")
    assert d["config"] == bench.config_dict(desc, 1, sc)
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["value"] == d["value"] and cb["cores"] >= 1
    assert "serial" in cb["modes"] and len(cb["modes"]) >= 1
    assert d["e2e"] == {"value": d["value"], "unit": "Mpix/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}


def test_cuda_arm_fails_without_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    p = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--steps", "1", "--warmup", "1",
                        "--no-cpu-baseline", "--no-forms"],
                       capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert p.returncode != 0
    assert not [l for l in p.stdout.splitlines() if l.startswith("{")]
