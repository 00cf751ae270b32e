"""The bench.py contract on the CPU: the reference arm (the oracle port,
no GPU needed) prints one JSON line with every key the harness reads, alone
and under torchrun with two ranks (rank 0 alone prints; the others exit 0),
and the command line names every workload and the CG form switch."""
import json
import os
import socket
import subprocess
import sys

from conftest import ROOT

BENCH = os.path.join(ROOT, "bench.py")
KEYS = {"impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
        "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config",
        "cpu_baseline", "e2e"}


def json_lines(out: str):
    return [json.loads(l) for l in out.splitlines() if l.startswith("{")]


def check_reference_line(d, n_gpus):
    assert KEYS <= set(d), KEYS - set(d)
    assert d["impl"] == "reference" and d["n_gpus"] == n_gpus
    assert d["value"] > 0 and d["unit"] == "cell-iters/s" and d["higher_is_better"] is True
    assert d["steps"] == 1 and d["warmup"] == 1 and d["ms_per_step"] > 0
    assert d["config"]["mesh"] == [60, 120, 84]
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == d["value"]
    assert cb["sample"]
    e2e = d["e2e"]
    assert e2e["value"] == d["value"] and e2e["unit"] == d["unit"]
    assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0


def test_reference_arm_prints_the_contract_line():
    r = subprocess.run([sys.executable, BENCH, "--impl", "reference", "--steps", "1",
                        "--warmup", "1"], capture_output=True, text=True, timeout=600,
                       cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = json_lines(r.stdout)
    assert len(lines) == 1
    check_reference_line(lines[0], 1)


def test_reference_arm_under_torchrun_prints_once():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    r = subprocess.run([sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
                        "--nproc-per-node", "2", "--master-addr", "127.0.0.1",
                        "--master-port", str(port), BENCH, "--impl", "reference",
                        "--gpus", "2", "--steps", "1", "--warmup", "1"],
                       capture_output=True, text=True, timeout=900, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = json_lines(r.stdout)
    assert len(lines) == 1
    check_reference_line(lines[0], 2)


def test_command_line_names_workloads_and_forms():
    r = subprocess.run([sys.executable, BENCH, "--help"], capture_output=True, text=True,
                       timeout=300, cwd=ROOT)
    assert r.returncode == 0
    for w in ("production", "fine", "batch", "serve", "tdma", "pcorr", "assemble", "pstep",
              "one-reduction", "reference"):
        assert w in r.stdout, w
