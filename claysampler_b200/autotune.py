"""Autotuner for the end-to-end render (render_window through the C ABI).

The tap count is fixed at 48 and tiles are 256 frames because the tail blocks
are 1024 frames, so neither is a free parameter.  Frames per segment are not
swept either: the renderer cuts a batch into the longest segments its chain
scratch budget holds (one segment unless filtered voices' storage exceeds it),
and shorter segments only add launches and state carries; batches of unfiltered
voices have no chain scratch to cut.  What does change the
end-to-end rate without changing a sample is how the work is cut and overlapped:

* `batch_jobs` (the CLI's --gpu-batch-jobs): how many jobs one GPU batch takes.
  Larger batches launch fewer, larger grids; smaller ones let the stream lanes
  overlap one batch's host staging, upload and download with another's kernels.
* `lanes`: how many batches are in flight at once, each on its own stream lane
  with its own arena and staging buffers.  More lanes let the host stage the next
  batches while earlier ones run and download, at the cost of device memory.
* `shared_sources`: whether each distinct resampled source is rendered once per
  batch and read by every voice that plays it, or every voice frame is resampled
  inline.  Which is faster depends on how often sources repeat in a batch.
* `ordered_compute`: whether every lane's kernels run in batch order on one stream
  (downloads start early; shared sources pooled per window) or each lane's beside
  the others (latency-bound kernels such as long filter chains overlap).

The best point depends on the workload's lengths and voice mix, so :func:`tune`
measures it.  After one discarded warm-up, it renders the workload through
render_window for every candidate, one untimed pass and then `repeats` timed
passes, and keeps the candidate whose median pass is fastest.  Results are
cached per workload signature in a JSON file.  Candidates never change the audio:
publish order and PCM are the same for every cut, lane count and source mode (the
renderer's invariants, tested in tests/test_serving.py and
tests/test_gpu_full_size.py).
"""
from __future__ import annotations

import hashlib
import json
import time
from pathlib import Path

import numpy as np

from .plans import PlanSet
from .renderer import Renderer

CANDIDATES = (16, 32, 64, 128, 256, 512)
LANES = (2, 4)
SHARED = (True, False)
RATE = 44100


def signature(plans) -> str:
    """Workload key: job count and each job's frames and span count."""
    h = hashlib.sha1()
    h.update(np.array([len(plans)], np.int64).tobytes())
    h.update(np.array([(p.frames, len(p.spans)) for p in plans], np.int64).tobytes())
    return h.hexdigest()[:16]


def measure(plans, bank, batch_jobs: int, repeats: int = 2, device: int = 0, lanes: int = 2,
            shared_sources: bool = True, ordered_compute: bool = True) -> float:
    """Output audio-seconds per second of render_window with GPU batches of
    `batch_jobs`, `lanes` batches in flight, shared sources on or off and the
    lanes' kernels ordered on one stream or side by side."""
    plans = plans if isinstance(plans, PlanSet) else PlanSet(plans)
    renderer = Renderer(device=device, natural=True, batch_jobs=batch_jobs)
    try:
        renderer.set_lanes(lanes)
        renderer.set_shared_sources(shared_sources)
        renderer.set_ordered_compute(ordered_compute)
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
         cache: Path | None = None, lanes=LANES, shared=SHARED) -> dict:
    """The fastest render_window settings for `plans`: {"batch_jobs", "lanes",
    "shared_sources", "ordered_compute", "sweep", "signature"}.  The batch size is
    swept first with two lanes and shared sources; the lane counts and the source
    mode are then tried at the two best sizes, and the lanes' kernels side by side
    at the best point."""
    key = signature(plans)
    store = {}
    if cache is not None and cache.exists():
        store = json.loads(cache.read_text())
        if key in store and "ordered_compute" in store[key]:
            return store[key]
    measure(plans, bank, candidates[0], 1, device)        # one-time costs (threads, page-locking) land here
    sweep = {}
    for jobs in candidates:
        if jobs > 2 * len(plans) and sweep:
            break
        sweep[f"{jobs}/2/shared"] = measure(plans, bank, jobs, repeats, device)
    # Lanes and source mode at the two fastest batch sizes (neighbours often
    # trade places once more batches overlap).
    leaders = sorted(sweep, key=sweep.get, reverse=True)[:2]
    for best_jobs in (name.split("/")[0] for name in leaders):
        for count in lanes:
            for mode in shared:
                name = f"{best_jobs}/{count}/{'shared' if mode else 'plain'}"
                if name not in sweep:
                    sweep[name] = measure(plans, bank, int(best_jobs), repeats, device, count, mode)
    # The lanes side by side at the best point so far.
    best = max(sweep, key=sweep.get).split("/")
    name = "/".join(best) + "/side"
    sweep[name] = measure(plans, bank, int(best[0]), repeats, device, int(best[1]), best[2] == "shared", False)
    best = max(sweep, key=sweep.get).split("/")
    result = {"batch_jobs": int(best[0]), "lanes": int(best[1]), "shared_sources": best[2] == "shared",
              "ordered_compute": len(best) < 4, "sweep": sweep, "signature": key}
    if cache is not None:
        store[key] = result
        cache.parent.mkdir(parents=True, exist_ok=True)
        cache.write_text(json.dumps(store, indent=1))
    return result
