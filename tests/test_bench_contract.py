"""The bench's output contract, checked on the CPU through its reference arm (the oracle timed on
the host cores), which needs no GPU: one JSON line with the required keys, the CPU-baseline and
end-to-end objects describing the same run, and under a two-rank launch exactly one line from
rank 0 with every rank exiting 0. The GPU arm's line is produced by the same writer."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ARGS = ["--impl", "reference", "--workload", "c0", "--steps", "1", "--warmup", "3"]
REQUIRED = ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
            "vs_baseline", "dtype", "data", "config", "impl", "cpu_baseline", "e2e")


def json_lines(text):
    return [json.loads(line) for line in text.splitlines() if line.startswith("{")]


def check_line(r, n_gpus):
    for k in REQUIRED:
        assert k in r, k
    assert r["impl"] == "reference" and r["n_gpus"] == n_gpus and r["steps"] == 1 and r["warmup"] == 3
    assert r["metric"] == "body-steps/s" and r["unit"] == "body-steps/s" and r["higher_is_better"] is True
    assert r["value"] > 0 and r["ms_per_step"] > 0 and r["scaling"] in ("weak", "strong")
    assert "workload" in r["config"] and "model" not in r["config"]
    cb = r["cpu_baseline"]
    assert cb["value"] == r["value"] and cb["unit"] == r["unit"] and cb["kind"] in ("port", "reference")
    assert cb["cores"] >= 1 and cb["sample"]
    e2e = r["e2e"]
    assert e2e == {"value": r["value"], "unit": r["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_reference_arm_prints_one_contract_line():
    out = subprocess.run([sys.executable, "bench.py", *ARGS], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = json_lines(out.stdout)
    assert len(lines) == 1
    check_line(lines[0], 1)


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_reference_arm_under_two_ranks_prints_once_from_rank_zero():
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2", "--master-addr",
           "127.0.0.1", "--master-port", str(free_port()), "bench.py", "--gpus", "2", *ARGS]
    out = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = json_lines(out.stdout)
    assert len(lines) == 1
    check_line(lines[0], 2)


def test_our_arm_without_a_gpu_fails_instead_of_falling_back():
    """The product arm has no CPU path: on a machine without a GPU it exits non-zero and prints no
    result line (skipped where CUDA is present, where it would run the full bench)."""
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    out = subprocess.run([sys.executable, "bench.py", "--steps", "1", "--warmup", "3"], cwd=ROOT, capture_output=True,
                         text=True, timeout=600)
    assert out.returncode != 0
    assert json_lines(out.stdout) == []
