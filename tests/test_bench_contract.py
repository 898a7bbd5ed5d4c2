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
