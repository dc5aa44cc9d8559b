"""The benchmark's command lines run to completion and print one contract
line: the short form the benchmark is run with by default tooling
(--gpus 1 --steps 20 --warmup 5), for the 1M-GR network and for the other
workloads."""
import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def run_bench(*extra, timeout=900):
    proc = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--gpus", "1", "--steps", "20",
                           "--warmup", "5", *extra], capture_output=True, text=True, timeout=timeout, cwd=ROOT)
    assert proc.returncode == 0, proc.stderr[-2000:]
    lines = [ln for ln in proc.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, proc.stdout[-2000:]
    return json.loads(lines[0])


def test_short_run_prints_the_contract_line():
    out = run_bench()
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "dtype", "config", "roofline", "e2e", "gpu_launches", "clocks", "cpu_baseline"):
        assert key in out, key
    assert out["n_gpus"] == 1 and out["steps"] == 20 and out["warmup"] == 5 and out["value"] > 0
    roof = out["roofline"]
    assert roof["achieved"] > 0 and roof["peak"] > 0
    assert abs(roof["frac"] - roof["achieved"] / roof["peak"]) < 1e-9
    assert abs(roof["achieved"] - roof["algorithmic_bytes"] / (roof["pass_ms"] / 1000.0) / 1e9) < 1e-6 * roof["achieved"]
    assert out["e2e"]["value"] > 0 and out["e2e"]["h2d_bytes_per_step"] > 0
    assert out["cpu_baseline"]["value"] > 0 and out["cpu_baseline"]["cores"] >= 1


@pytest.mark.parametrize("extra", [("--workload", "dense4m"), ("--workload", "batch", "--instances", "4")])
def test_short_workload_runs_print_one_line(extra):
    # these workloads time whole graph chunks: at least one chunk of steps
    out = run_bench(*extra)
    assert out["value"] > 0 and out["steps"] >= 20
