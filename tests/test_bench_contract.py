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


def run_bench(*args, launcher=()):
    proc = subprocess.run([sys.executable, *launcher, os.path.join(ROOT, "bench.py"), "--impl", "reference", *args], cwd=ROOT,
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


def test_reference_arm_under_torchrun():
    """Launched like the multi-GPU arm (one process per GPU): rank 0 alone runs and prints; the other ranks exit 0."""
    import socket

    with socket.socket() as sock:
        sock.bind(("127.0.0.1", 0))
        port = sock.getsockname()[1]
    launcher = ("-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2", "--master-addr", "127.0.0.1",
                "--master-port", str(port))
    line = run_bench("--gpus", "2", "--vertices", "1500", "--degree", "10", "--steps", "1", "--warmup", "3", launcher=launcher)
    check_line(line, "APSP+Brandes", "GTEPS")
    assert line["n_gpus"] == 2
