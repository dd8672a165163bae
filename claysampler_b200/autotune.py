"""Autotuner for the end-to-end render (render_window through the C ABI).

The renderer's kernels have no free shape parameters that keep parity: the tap
count is fixed at 48, tiles are 256 frames because the tail blocks are 1024
frames, and every launch covers all of a batch's jobs.  What does change the
end-to-end rate is how the job list is cut into GPU batches (`batch_jobs`, the
CLI's --gpu-batch-jobs): larger batches launch fewer, larger grids, while smaller
ones let the renderer's two stream lanes overlap one batch's upload and download
with the other's kernels.  The best cut depends on the workload's lengths and on
its voice mix, so :func:`tune` measures it.  After one discarded warm-up, it
renders the workload through render_window for every candidate, one untimed pass
and then `repeats` timed passes, and keeps the candidate whose median pass is
fastest.  Results are cached per workload signature in
a JSON file.  Candidates change only the batching, never the audio: publish
order and PCM are the same for every cut (the renderer's invariant, tested in
tests/test_serving.py).
"""
from __future__ import annotations

import hashlib
import json
import time
from pathlib import Path

import numpy as np

from .renderer import Renderer

CANDIDATES = (16, 32, 64, 128, 256)
RATE = 44100


def signature(plans) -> str:
    """Workload key: job count and each job's frames and span count."""
    h = hashlib.sha1()
    h.update(np.array([len(plans)], np.int64).tobytes())
    h.update(np.array([(p.frames, len(p.spans)) for p in plans], np.int64).tobytes())
    return h.hexdigest()[:16]


def measure(plans, bank, batch_jobs: int, repeats: int = 2, device: int = 0) -> float:
    """Output audio-seconds per second of render_window with GPU batches of `batch_jobs`."""
    renderer = Renderer(device=device, natural=True, batch_jobs=batch_jobs)
    try:
        renderer.upload_samples(bank)
        audio = [0.0]

        def publish(batch, first):
            audio[0] += float(batch.results["frames"].sum()) / RATE

        renderer.render_window(plans, publish, copy=False)          # untimed: arenas, staging
        times = []
        for _ in range(repeats):
            audio[0] = 0.0
            start = time.perf_counter()
            renderer.render_window(plans, publish, copy=False)
            times.append(time.perf_counter() - start)
        return audio[0] / float(np.median(times))           # the median pass: host jitter aside
    finally:
        renderer.close()


def tune(plans, bank, candidates=CANDIDATES, repeats: int = 3, device: int = 0,
         cache: Path | None = None) -> dict:
    """The fastest GPU batch size for `plans` ({"batch_jobs", "sweep", "signature"})."""
    key = signature(plans)
    store = {}
    if cache is not None and cache.exists():
        store = json.loads(cache.read_text())
        if key in store:
            return store[key]
    measure(plans, bank, candidates[0], 1, device)        # one-time costs (threads, page-locking) land here
    sweep = {}
    for jobs in candidates:
        if jobs > 2 * len(plans) and sweep:
            break
        sweep[str(jobs)] = measure(plans, bank, jobs, repeats, device)
    best = max(sweep, key=sweep.get)
    result = {"batch_jobs": int(best), "sweep": sweep, "signature": key}
    if cache is not None:
        store[key] = result
        cache.parent.mkdir(parents=True, exist_ok=True)
        cache.write_text(json.dumps(store, indent=1))
    return result
