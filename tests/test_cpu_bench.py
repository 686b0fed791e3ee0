"""bench.py's reference arm runs on the host and prints one JSON line with
the contract's keys (the GPU arm is exercised on a GPU)."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(args):
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py")] + args, capture_output=True, text=True,
                         timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, out.stdout
    return json.loads(lines[0])


KEYS = ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
        "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e", "impl")


def test_reference_arm_single_pencil():
    d = _run(["--impl", "reference", "--n", "400", "--cpu-sample-n", "200", "--steps", "1", "--warmup", "0"])
    for k in KEYS:
        assert k in d, k
    assert d["impl"] == "reference" and d["unit"] == "s" and d["higher_is_better"] is False
    assert d["value"] > 0 and d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"]["h2d_bytes_per_step"] == 0


def test_reference_arm_batched():
    d = _run(["--impl", "reference", "--workload", "c5", "--batch", "16", "--steps", "1", "--warmup", "0"])
    for k in KEYS:
        assert k in d, k
    assert d["unit"] == "pencils/s" and d["higher_is_better"] is True and d["value"] > 0
