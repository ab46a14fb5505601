"""The benchmark's output contract, checked on the CPU.

* The reference arm (`bench.py --impl reference`): the reference's per-view training
  step, restated in C, timed on the host cores, printed as one JSON line with the same
  metric and unit as the product arm, its own `cpu_baseline` and a host-only `e2e`.
* Under a multi-rank launch only rank 0 runs the reference arm; the others exit 0 quietly.
* The product arm has no CPU fallback: without a CUDA device it stops with the library's
  error and prints no measurement.

The 200k-Gaussian single-view workload (`--config 2`) keeps the reference step to a few
seconds on a handful of cores.
"""
import json
import os
import subprocess
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(args, env_extra=None, timeout=900):
    env = dict(os.environ)
    env.update(env_extra or {})
    return subprocess.run([sys.executable, os.path.join(REPO, "bench.py"), *args], cwd=REPO, env=env,
                          capture_output=True, text=True, timeout=timeout)


def _json_lines(out):
    return [json.loads(line) for line in out.splitlines() if line.startswith("{")]


def _cuda_present():
    import torch
    return torch.cuda.is_available()


def test_reference_arm_line():
    r = _run(["--impl", "reference", "--config", "2", "--steps", "1", "--warmup", "3"])
    assert r.returncode == 0, r.stderr[-2000:]
    lines = _json_lines(r.stdout)
    assert len(lines) == 1, r.stdout[-2000:]
    d = lines[0]
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference"
    assert d["unit"] == "steps/s" and d["higher_is_better"] is True
    assert d["steps"] == 1 and d["warmup"] >= 3 and d["n_gpus"] == 1
    assert d["value"] > 0 and d["ms_per_step"] > 0
    assert d["vs_baseline"] is None
    assert "workload" in d["config"] and d["config"]["gaussians"] == 200000
    cb = d["cpu_baseline"]
    assert cb["kind"] in ("port", "reference") and cb["cores"] >= 1 and cb["sample"]
    assert cb["value"] == d["value"] and cb["unit"] == d["unit"]
    e = d["e2e"]
    assert e["value"] == d["value"] and e["unit"] == d["unit"]
    assert e["h2d_bytes_per_step"] == 0 and e["d2h_bytes_per_step"] == 0


def test_reference_arm_runs_on_rank_zero_only():
    r = _run(["--impl", "reference", "--config", "2", "--steps", "1", "--gpus", "2"],
             env_extra={"RANK": "1", "LOCAL_RANK": "1", "WORLD_SIZE": "2"}, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    assert not _json_lines(r.stdout)


@pytest.mark.skipif(_cuda_present(), reason="a CUDA device is present: the product arm runs")
def test_product_arm_needs_a_gpu():
    r = _run(["--config", "2", "--steps", "3", "--warmup", "3", "--no-cpu", "--no-plain", "--no-e2e",
              "--no-densify"], timeout=300)
    assert r.returncode != 0
    assert not _json_lines(r.stdout)
    assert "no CUDA device" in r.stderr
