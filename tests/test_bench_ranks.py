"""The multi-rank path of bench.py (one process per GPU, jobs sharded by rank, no
data-path collective): per-rank workloads differ, and the whole-job figures sum
audio over ranks and take times as the max over ranks.  Run here as two `gloo`
ranks on the CPU."""
import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    sys.path.insert(0, str(ROOT))
    import datetime
    import torch
    import torch.distributed as dist
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    try:
        assert bench.dist_info() == (rank, world, rank)
        # rank r: 100 (r + 1) audio-s in (10 + r) ms per step; e2e (0.5 + r) s for 90 (r + 1) audio-s
        totals = torch.tensor([100.0 * (rank + 1), 10.0 + rank, 0.5 + rank, 90.0 * (rank + 1)], dtype=torch.float64)
        rows = bench.gather_rows(totals, world)
        np.save(out / f"rows{rank}.npy", rows)
        np.save(out / f"combined{rank}.npy", np.array(bench.combine(rows)))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_ranks_combine_by_sum_and_max(tmp_path):
    import torch.multiprocessing as mp
    port = _free_port()
    mp.spawn(_rank, args=(2, port, tmp_path), nprocs=2, join=True)
    for rank in range(2):
        rows = np.load(tmp_path / f"rows{rank}.npy")
        assert rows.shape == (2, 4)
        np.testing.assert_array_equal(rows[:, 0], [100.0, 200.0])
        audio, ms, e2e, e2e_audio = np.load(tmp_path / f"combined{rank}.npy")
        assert (audio, ms, e2e, e2e_audio) == (300.0, 11.0, 1.5, 270.0)


def test_each_rank_renders_its_own_batch(tmp_path, monkeypatch):
    """Weak scaling: rank r generates the workload of seed + r, so ranks never render
    the same jobs."""
    import argparse
    sys.path.insert(0, str(ROOT))
    import bench
    from claysampler_b200 import workload as wl
    seeds = []

    def fake_batch(root, seed, jobs):
        seeds.append(seed)
        root.mkdir(parents=True, exist_ok=True)
        return [wl.Job(group="-", sfz=root / "preset.sfz", midi=root / "0.mid", output=root / "0.wav")]

    monkeypatch.setattr(wl, "write_plain_batch", fake_batch)
    args = argparse.Namespace(workdir=tmp_path, seed=2, jobs=1)
    a, b = bench.workload(args, 0), bench.workload(args, 1)
    assert seeds == [2, 3] and a != b


def test_serving_requests(tmp_path):
    """The serving workload: seeded requests of the small kind with lengths in
    [5, 300] s, arriving in increasing order (a Poisson process of the given rate),
    planned by the host planner."""
    import argparse
    sys.path.insert(0, str(ROOT))
    import bench
    args = argparse.Namespace(workdir=tmp_path, seed=5, serve_jobs=6, serve_rate=50.0)
    plans, arrivals, bank = bench.serving_requests(args, 0)
    again, arrivals_again, _ = bench.serving_requests(args, 0)
    assert len(plans) == 6 and bank.size > 0
    assert np.all(np.diff(arrivals) > 0) and arrivals[0] > 0
    assert np.array_equal(arrivals, arrivals_again)
    assert [p.frames for p in plans] == [p.frames for p in again]
    seconds = np.array([p.music_end for p in plans]) / 44100
    assert np.all(seconds >= 4.5) and np.all(seconds <= 300.5)
    other, arrivals_other, _ = bench.serving_requests(args, 1)
    assert not np.array_equal(arrivals, arrivals_other)
