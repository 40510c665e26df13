"""bench.py's command-line contract, checked on the CPU: the reference arm
(the oracle timed on the host cores) prints one JSON line with every key a
bench line carries, ranks other than 0 print nothing, and the CUDA arm stops
with an error instead of falling back to the CPU when no device is present."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def run_bench(*args, env=None, timeout=600):
    e = dict(os.environ)
    e.update(env or {})
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args], cwd=ROOT, env=e,
                          capture_output=True, text=True, timeout=timeout)


def json_lines(out):
    return [json.loads(line) for line in out.splitlines() if line.startswith("{")]


def test_reference_arm_prints_one_contract_line():
    p = run_bench("--impl", "reference", "--config", "c1", "--steps", "1", "--warmup", "0")
    assert p.returncode == 0, p.stderr[-2000:]
    lines = json_lines(p.stdout)
    assert len(lines) == 1
    j = lines[0]
    for key in ["metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
                "vs_baseline", "dtype", "data", "config", "impl", "cpu_baseline", "e2e"]:
        assert key in j, key
    assert j["impl"] == "reference" and j["metric"] == "stack MP-frames/s (align+fuse+depth)"
    assert j["unit"] == "MP-frames/s" and j["higher_is_better"] is True and j["scaling"] == "weak"
    assert j["steps"] == 1 and j["warmup"] == 0 and j["n_gpus"] == 1
    assert j["value"] > 0 and j["ms_per_step"] > 0
    # one step is one frame's work plus its share of the stack's finish: the value is the whole
    # 8-frame 1024x768 stack's, extrapolated from the per-frame time
    cb = j["cpu_baseline"]
    assert j["ms_per_step"] == pytest.approx(1e3 * (cb["per_frame_s"] + cb["finish_s"] / 8), rel=1e-9)
    assert j["value"] == pytest.approx(1024 * 768 / 1e6 / (j["ms_per_step"] / 1e3), rel=1e-9)
    assert j["config"]["workload"].startswith("c1: 8 x 1024x768")
    assert cb["value"] == j["value"] and cb["unit"] == j["unit"] and cb["kind"] == "port" and cb["cores"] >= 1
    assert cb["extrapolated"] is True and cb["sample"] and cb["one_core"]["per_frame_s"] > 0
    # the CPU arm runs the oracle alone: no part of the CUDA library is loaded
    assert j["native_so"] is not None and not any("liblapstack_b200" in p for p in j["native_so"]), j["native_so"]
    assert any("liblsb_oracle" in p for p in j["native_so"])
    assert j["e2e"] == {"value": j["value"], "unit": j["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_reference_arm_runs_on_rank_0_only():
    p = run_bench("--impl", "reference", "--config", "c1", "--steps", "1", "--warmup", "0", "--gpus", "2",
                  env={"RANK": "1", "LOCAL_RANK": "1", "WORLD_SIZE": "2"})
    assert p.returncode == 0, p.stderr[-2000:]
    assert json_lines(p.stdout) == []


def test_cuda_arm_stops_without_a_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    p = run_bench("--config", "c1", "--steps", "1", "--warmup", "0")
    assert p.returncode != 0
    assert json_lines(p.stdout) == []


def test_batch_mode_stops_without_a_device():
    """The uneven-batch line (--batch) comes from the CUDA engine only: without a device it stops with an
    error and prints no line."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    p = run_bench("--batch", "--steps", "1", "--warmup", "0")
    assert p.returncode != 0
    assert json_lines(p.stdout) == []
