"""bench.py's reference arm on the CPU: the reference's own planner and render
(built for the host) on a small uneven workload, printing one JSON line with the
bench contract's keys; under torchrun only rank 0 runs and prints."""
import json
import os
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _bench(*args, env=None):
    run = subprocess.run([sys.executable, str(ROOT / "bench.py"), *args], cwd=ROOT, capture_output=True, text=True,
                         timeout=600, env={**os.environ, **(env or {})})
    assert run.returncode == 0, run.stderr[-2000:]
    return [line for line in run.stdout.splitlines() if line.startswith("{")]


@pytest.fixture(scope="module")
def reference_built():
    from oracle import reference
    if not reference.available():
        reference.build()
    if not reference.available():
        pytest.skip("the reference is not built for the host")


def test_reference_arm_prints_the_bench_line(reference_built):
    lines = _bench("--impl", "reference", "--steps", "2", "--warmup", "1", "--jobs", "4")
    assert len(lines) == 1
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and "unavailable" not in line
    assert line["unit"] == "audio-s/s" and line["value"] > 0 and line["higher_is_better"] is True
    assert (line["n_gpus"], line["steps"], line["warmup"]) == (1, 2, 1)
    assert line["config"]["jobs_per_gpu"] == 4 and line["config"]["workload"].startswith("uneven batch: 4 jobs")
    base = line["cpu_baseline"]
    assert base["kind"] == "reference" and base["value"] == line["value"] and base["cores"] >= 1
    assert "first 4 of 4 jobs" in base["sample"]
    assert line["e2e"] == {"value": line["value"], "unit": "audio-s/s", "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}


def test_reference_arm_runs_on_rank_zero_only(reference_built):
    assert _bench("--impl", "reference", "--steps", "1", "--warmup", "0", "--jobs", "4",
                  env={"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"}) == []
