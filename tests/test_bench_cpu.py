"""bench.py on a machine without a GPU: the reference arm's JSON contract, its rank handling,
and that the B200 arm fails loudly instead of measuring anything else."""

from __future__ import annotations

import json
import os
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _bench(*args, env=None, timeout=600):
    e = dict(os.environ)
    e.update(env or {})
    return subprocess.run([sys.executable, str(ROOT / "bench.py"), *args], cwd=ROOT, env=e,
                          capture_output=True, text=True, timeout=timeout)


def test_reference_arm_prints_one_contract_line():
    res = _bench("--impl", "reference", "--steps", "1", "--warmup", "3")
    assert res.returncode == 0, res.stderr
    lines = [ln for ln in res.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["unit"] == "GLUPS" and d["value"] > 0
    assert d["metric"].startswith("GLUPS (3D 512^3 fp32 periodic FTCS")
    assert d["n_gpus"] == 1 and d["steps"] == 1 and d["warmup"] >= 3
    assert d["higher_is_better"] is True and d["scaling"] == "weak"
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": "GLUPS", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}
    sys.path.insert(0, str(ROOT))
    try:
        import bench
    finally:
        sys.path.remove(str(ROOT))
    # the same workload description as the B200 arm (one update per bench step here)
    # the same config object as the GPU arm's line; the per-step work is a separate key
    assert d["config"] == bench.workload_config(3, 512, "float32", 1)
    assert d["time_steps_per_step"] == 1


def test_reference_arm_other_ranks_exit_quietly():
    res = _bench("--impl", "reference", "--steps", "1", "--warmup", "3",
                 env={"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"})
    assert res.returncode == 0, res.stderr
    assert res.stdout.strip() == ""


@pytest.mark.skipif(__import__("torch").cuda.is_available(), reason="needs a machine without GPU")
def test_b200_arm_without_a_gpu_fails_loudly():
    res = _bench("--steps", "1", "--warmup", "3", "--no-variants", "--no-cpu", "--no-batch",
                 "--no-serve", "--no-precision", timeout=300)
    assert res.returncode != 0
    assert not [ln for ln in res.stdout.splitlines() if ln.startswith("{")]
