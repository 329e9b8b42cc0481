"""bench.py's reference arm (host only, no GPU): one JSON line on stdout with the contract's keys, for the default
workload and for the SCC workload, on small graphs."""

from __future__ import annotations

import json
import os
import subprocess
import sys

import pytest

import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
KEYS = {"impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
        "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"}


def run_bench(*args):
    proc = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", *args], cwd=ROOT,
                          capture_output=True, text=True, timeout=600)
    assert proc.returncode == 0, proc.stderr[-2000:]
    lines = [line for line in proc.stdout.splitlines() if line.strip()]
    assert len(lines) == 1, proc.stdout  # exactly one line on stdout: the reference's own reports go to stderr
    return json.loads(lines[0])


def check_line(line, metric_word, unit):
    assert KEYS <= set(line), KEYS - set(line)
    assert line["impl"] == "reference" and metric_word in line["metric"] and line["unit"] == unit
    assert line["value"] > 0 and line["steps"] == 1 and line["warmup"] == 3
    assert line["cpu_baseline"]["value"] == line["value"] and line["cpu_baseline"]["cores"] >= 1
    assert line["e2e"] == {"value": line["value"], "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_reference_arm_default_workload():
    line = run_bench("--n", "1500", "--degree", "10", "--steps", "1", "--warmup", "3")
    check_line(line, "APSP+Brandes", "GTEPS")
    assert line["config"]["n"] == 1500 and line["cpu_baseline"]["kind"] == "port"


def test_reference_arm_scc_workload():
    if not oracle.Reference.available():
        pytest.skip("the reference build (oracle/_ref) is not here")
    line = run_bench("--workload", "scc", "--n", "1500", "--degree", "10", "--steps", "1", "--warmup", "3")
    check_line(line, "SCC", "G arcs/s")
    assert line["cpu_baseline"]["kind"] == "reference" and line["config"]["n"] == 1500
