"""bench.py's host-side paths: the reference arm (whole solves of the
benchmarked pencil by the oracle port, within a budget) prints one JSON
line with the contract's keys and the same config block as the GPU arm;
the CPU-baseline sample runs the port on the same pencil for a bounded
number of AEDs; --gpus N starts N ranks itself when it is not under
torchrun (checked with --check-ranks on gloo, no GPU)."""
import json
import os
import subprocess
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(args, timeout=600):
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py")] + args, capture_output=True, text=True,
                         timeout=timeout, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, out.stdout
    return json.loads(lines[0])


KEYS = ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
        "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e", "impl")


def test_reference_arm_single_pencil(pkg):
    d = _run(["--impl", "reference", "--n", "400", "--steps", "3", "--warmup", "0", "--ref-budget", "60"])
    for k in KEYS:
        assert k in d, k
    assert d["impl"] == "reference" and d["unit"] == "s" and d["higher_is_better"] is False
    assert d["value"] > 0 and d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["cores"] >= 1
    assert 1 <= d["steps"] <= 3
    assert d["e2e"]["h2d_bytes_per_step"] == 0
    # the same config block as the GPU arm prints for this workload
    import bench
    (H, T), desc = bench.make_pencil(pkg, "c3", 400)
    assert d["config"] == bench.workload_config(pkg, "c3", 400, desc)


def test_reference_arm_budget_bounds_steps():
    """A budget smaller than one solve still runs exactly one whole solve."""
    d = _run(["--impl", "reference", "--n", "600", "--steps", "20", "--warmup", "5", "--ref-budget", "0"])
    assert d["steps"] == 1 and d["value"] > 0


def test_reference_arm_batched():
    d = _run(["--impl", "reference", "--workload", "c5", "--batch", "16", "--steps", "1", "--warmup", "0"])
    for k in KEYS:
        assert k in d, k
    assert d["unit"] == "pencils/s" and d["higher_is_better"] is True and d["value"] > 0


def test_reference_arm_of_the_steps_beside_the_solve():
    """The balancing, reordering and HT-reduction workloads time LAPACK in
    their own line (cpu_baseline); their reference arm says so and exits 0."""
    for w in ("ggbal", "tgsen", "gghrd"):
        d = _run(["--impl", "reference", "--workload", w, "--steps", "1", "--warmup", "0"], timeout=120)
        assert d["impl"] == "reference" and "unavailable" in d and "LAPACK" in d["unavailable"]


def test_cpu_baseline_sample_is_bounded_and_scaled(pkg, monkeypatch):
    """The bounded sample stops the port after K AEDs of the real pencil
    and divides by the share those AEDs took in the committed profile."""
    import bench
    fx = bench.port_fixture("c2", 4000)
    assert fx is not None and "aed_clock" in fx
    out = bench.cpu_baseline_sample(pkg, "c2", 4000, budget_s=2.0)
    assert out is not None and out["kind"] == "port" and out["value"] > 0
    assert "first" in out["sample"] and "AEDs" in out["sample"]


def test_gpus_n_starts_ranks_itself():
    """python bench.py --gpus 2 outside torchrun launches two ranks; with
    --check-ranks they join on gloo and the c5 shards partition the batch."""
    env = dict(os.environ)
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK", "MASTER_ADDR", "MASTER_PORT"):
        env.pop(k, None)
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--gpus", "2", "--workload", "c5",
                          "--batch", "64", "--check-ranks"], capture_output=True, text=True, timeout=300, cwd=ROOT,
                         env=env)
    assert out.returncode == 0, out.stderr[-3000:]
    lines = [json.loads(l) for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, out.stdout
    d = lines[0]
    assert d["n_ranks"] == 2 and d["partition_ok"] and d["pencils"] == 128
    assert sum(d["per_rank"]) == 128 and min(d["per_rank"]) > 0
