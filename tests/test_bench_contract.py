"""CPU checks of bench.py's command-line contract that need no GPU: the reference arm of a
configuration the reference cannot run prints one `unavailable` JSON line and exits 0, and
bad arguments are refused."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def run(*args):
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args], capture_output=True, text=True,
                          timeout=120, cwd=ROOT)


def test_reference_arm_unavailable_line():
    for cfg in ("batched", "learned"):
        r = run("--impl", "reference", "--config", cfg, "--steps", "1", "--warmup", "3")
        assert r.returncode == 0, r.stderr
        line = json.loads(r.stdout.strip().splitlines()[-1])
        assert line["impl"] == "reference" and line["unavailable"]


def test_warmup_below_three_is_refused():
    r = run("--warmup", "2")
    assert r.returncode != 0 and "warmup" in r.stderr


def test_reference_arm_under_torchrun_prints_once():
    # two ranks launched the way the driver launches N > 1: rank 0 prints the line, the other
    # rank exits 0 without work
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    r = subprocess.run([sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
                        "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.join(ROOT, "bench.py"),
                        "--impl", "reference", "--config", "batched", "--gpus", "2", "--steps", "1", "--warmup", "3"],
                       capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(x) for x in r.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1 and lines[0]["impl"] == "reference"


def test_gpus_flag_without_torchrun_starts_the_ranks():
    # `--gpus 2` outside torchrun starts two ranks itself; rank 0 prints one line for 2 GPUs
    r = run("--impl", "reference", "--config", "uniform", "--gpus", "2", "--steps", "1", "--warmup", "3")
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(x) for x in r.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1 and lines[0]["n_gpus"] == 2 and lines[0]["impl"] == "reference"
    assert lines[0]["config"]["n_keys"] == 1 << 24 and lines[0]["config"]["n_query"] == 1 << 24


def test_reference_arm_count_min():
    r = run("--impl", "reference", "--config", "cm", "--steps", "1", "--warmup", "3")
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["value"] > 0 and line["cpu_baseline"]["cores"] >= 1
