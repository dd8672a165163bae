"""Python mirror of the reference's ``clay::Renderer`` (src/cuda/renderer.h:45-64).

The class wraps the C ABI of ``libclaysampler_b200.so`` (``include/claysampler_b200.h``)
with the same operations: ``upload_samples``, ``render_window`` with a publish
callback and an optional refill callback, and the memory getters.  There is no
fallback: if the CUDA library is missing or no sm_100 GPU is present, construction
raises.
"""
from __future__ import annotations

import ctypes
import os
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass
from pathlib import Path
from typing import Callable, Optional

import numpy as np

from . import build
from .plans import AUDIO_CONFIG, TAIL_RESULT, CPlan, Plan, c_plans, default_audio_config

_lib = None


def library() -> ctypes.CDLL:
    """Load (building first if stale) the in-tree CUDA library."""
    global _lib
    if _lib is None:
        path = build.LIBRARY
        if not path.exists():
            build.build_library()
        lib = ctypes.CDLL(str(path))
        c = ctypes
        vp, sz, i32 = c.c_void_p, c.c_size_t, c.c_int
        lib.cs_last_error.restype = c.c_char_p
        lib.cs_renderer_create.argtypes = [i32, i32, vp, i32, sz, sz, c.POINTER(vp)]
        lib.cs_renderer_destroy.argtypes = [vp]
        lib.cs_upload_samples.argtypes = [vp, vp, sz, i32]
        lib.cs_render_window.argtypes = [vp, vp, sz, vp, vp, vp]
        lib.cs_renderer_device.argtypes = [vp]
        lib.cs_renderer_device.restype = c.c_char_p
        for name in ("cs_peak_bytes", "cs_sample_cache_budget", "cs_peak_waiting_bytes", "cs_spilled_bytes",
                     "cs_downloaded_bytes"):
            getattr(lib, name).argtypes = [vp]
            getattr(lib, name).restype = sz
        lib.cs_prepare.argtypes = [vp, vp, sz, c.POINTER(vp)]
        lib.cs_run.argtypes = [vp, vp, vp]
        lib.cs_collect.argtypes = [vp, vp, vp, sz, c.POINTER(sz), vp]
        lib.cs_copy_mix.argtypes = [vp, vp, vp, sz]
        lib.cs_prepared_frames.argtypes = [vp]
        lib.cs_prepared_frames.restype = sz
        lib.cs_prepared_launches.argtypes = [vp]
        lib.cs_prepared_segments.argtypes = [vp]
        lib.cs_prepared_segments.restype = sz
        lib.cs_prepared_destroy.argtypes = [vp]
        lib.cs_renderer_set_scratch_limit.argtypes = [vp, sz]
        lib.cs_renderer_set_shared_sources.argtypes = [vp, i32]
        lib.cs_renderer_host_ms.argtypes = [vp, c.POINTER(c.c_double), i32]
        lib.cs_renderer_set_lanes.argtypes = [vp, i32]
        lib.cs_renderer_fail_allocations.argtypes = [vp, i32]
        lib.cs_renderer_set_ordered_compute.argtypes = [vp, i32]
        lib.cs_renderer_deferred_launches.argtypes = [vp]
        lib.cs_renderer_deferred_launches.restype = sz
        for name in ("cs_prepared_shared_sources", "cs_prepared_shared_frames"):
            getattr(lib, name).argtypes = [vp]
            getattr(lib, name).restype = sz
        lib.cs_prepared_shared_voice_frames.argtypes = [vp]
        lib.cs_prepared_shared_voice_frames.restype = c.c_longlong
        lib.cs_prepared_shared_sinc.argtypes = [vp, c.POINTER(c.c_longlong)]
        lib.cs_prepared_shared_sinc.restype = c.c_longlong
        lib.cs_submit.argtypes = [vp, vp, sz, c.POINTER(c.c_uint64)]
        lib.cs_poll.argtypes = [vp, i32, vp, vp, c.POINTER(sz)]
        lib.cs_pending_jobs.argtypes = [vp]
        lib.cs_pending_jobs.restype = sz
        lib.cs_prepared_set_profile.argtypes = [vp, i32]
        lib.cs_prepared_stage_ms.argtypes = [vp, vp, i32]
        lib.cs_stage_name.restype = c.c_char_p
        _lib = lib
    return _lib


_copier: Optional[ThreadPoolExecutor] = None


def _copy_out(pointer: int, count: int, dtype) -> np.ndarray:
    """An owned copy of `count` items at `pointer` (host memory).  Large copies are
    split over a few threads; numpy releases the GIL while it copies."""
    global _copier
    out = np.empty(count, dtype)
    if not count:
        return out
    src = np.ctypeslib.as_array(ctypes.cast(pointer, ctypes.POINTER(np.ctypeslib.as_ctypes_type(dtype))),
                                shape=(count,))
    if out.nbytes < (16 << 20):
        np.copyto(out, src)
        return out
    if _copier is None:
        _copier = ThreadPoolExecutor(max_workers=min(16, os.cpu_count() or 1))
    parts = _copier._max_workers
    bounds = np.linspace(0, count, parts + 1).astype(np.int64)
    list(_copier.map(lambda i: np.copyto(out[bounds[i]:bounds[i + 1]], src[bounds[i]:bounds[i + 1]]),
                     range(parts)))
    return out


def _check(status: int) -> None:
    if status:
        raise RuntimeError(library().cs_last_error().decode(errors="replace"))


class CBatch(ctypes.Structure):
    _fields_ = [("pcm", ctypes.c_void_p), ("pcm_samples", ctypes.c_size_t), ("results", ctypes.c_void_p),
                ("result_count", ctypes.c_size_t), ("kernel_seconds", ctypes.c_double),
                ("failed_scratch_bytes", ctypes.c_size_t), ("job_indices", ctypes.c_void_p),
                ("job_index_count", ctypes.c_size_t)]


PUBLISH = ctypes.CFUNCTYPE(None, ctypes.c_void_p, ctypes.POINTER(CBatch), ctypes.c_size_t)
REFILL = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p),
                          ctypes.POINTER(ctypes.c_size_t))


@dataclass
class RenderBatch:
    """clay::RenderBatch (src/cuda/renderer.h:37-43) with owned copies."""
    pcm: np.ndarray
    results: np.ndarray
    kernel_seconds: float
    failed_scratch_bytes: int
    job_indices: list


class Prepared:
    """A staged batch whose inputs stay resident on the device."""

    def __init__(self, renderer: "Renderer", plans: list[Plan]):
        self.renderer = renderer
        self.plans = plans
        self._array = c_plans(plans)
        handle = ctypes.c_void_p()
        _check(library().cs_prepare(renderer.handle, self._array, len(plans), ctypes.byref(handle)))
        self.handle = handle

    @property
    def frames(self) -> int:
        return library().cs_prepared_frames(self.handle)

    @property
    def launches(self) -> int:
        return library().cs_prepared_launches(self.handle)

    @property
    def segments(self) -> int:
        return library().cs_prepared_segments(self.handle)

    @property
    def shared(self) -> dict:
        """Shared voice sources of the batch: how many, the floats they hold and
        the voice frames that read them instead of resampling."""
        lib = library()
        voice_sinc = ctypes.c_longlong()
        sinc = lib.cs_prepared_shared_sinc(self.handle, ctypes.byref(voice_sinc))
        return {"sources": int(lib.cs_prepared_shared_sources(self.handle)),
                "floats": int(lib.cs_prepared_shared_frames(self.handle)),
                "voice_frames": int(lib.cs_prepared_shared_voice_frames(self.handle)),
                "sinc_floats": int(sinc), "voice_sinc_floats": int(voice_sinc.value)}

    def set_profile(self, enable: bool = True) -> None:
        _check(library().cs_prepared_set_profile(self.handle, int(enable)))

    def stage_ms(self) -> dict[str, float]:
        """Device time of each stage of the last profiled run (CUDA events)."""
        out = (ctypes.c_float * 16)()
        count = library().cs_prepared_stage_ms(self.handle, out, 16)
        if count < 0:
            _check(1)
        return {library().cs_stage_name(i).decode(): float(out[i]) for i in range(count)}

    def run(self, stream: int | None = None) -> None:
        _check(library().cs_run(self.renderer.handle, self.handle, stream))

    def collect(self) -> tuple[np.ndarray, np.ndarray]:
        samples = ctypes.c_size_t()
        results = np.zeros(len(self.plans), TAIL_RESULT)
        _check(library().cs_collect(self.renderer.handle, self.handle, None, 0, ctypes.byref(samples),
                                    results.ctypes.data))
        pcm = np.zeros(samples.value, np.int16)
        _check(library().cs_collect(self.renderer.handle, self.handle, pcm.ctypes.data if pcm.size else None,
                                    pcm.size, ctypes.byref(samples), results.ctypes.data))
        return pcm, results

    def mix(self) -> np.ndarray:
        dtype = np.float32 if self.renderer.natural else np.int16
        out = np.zeros((self.frames, 2), dtype)
        _check(library().cs_copy_mix(self.renderer.handle, self.handle, out.ctypes.data, out.nbytes))
        return out

    def close(self) -> None:
        if self.handle:
            library().cs_prepared_destroy(self.handle)
            self.handle = None

    def __del__(self):
        self.close()


class Renderer:
    """clay::Renderer over the B200 kernels."""

    def __init__(self, device: int = 0, natural: bool = True, audio: Optional[np.ndarray] = None,
                 group_minimum: int = 0, waiting_limit: int = 256 << 20, batch_jobs: int = 64):
        self.natural = natural
        self.audio = default_audio_config() if audio is None else np.asarray(audio, AUDIO_CONFIG)
        handle = ctypes.c_void_p()
        _check(library().cs_renderer_create(device, int(natural), self.audio.ctypes.data, group_minimum,
                                            waiting_limit, batch_jobs, ctypes.byref(handle)))
        self.handle = handle
        self._bank = None

    def close(self) -> None:
        if getattr(self, "handle", None):
            library().cs_renderer_destroy(self.handle)
            self.handle = None

    def __del__(self):
        self.close()

    def upload_samples(self, bank: np.ndarray, fresh: bool = False) -> None:
        bank = np.ascontiguousarray(bank, np.float32)
        self._bank = bank
        _check(library().cs_upload_samples(self.handle, bank.ctypes.data if bank.size else None, bank.size,
                                           int(fresh)))

    def set_scratch_limit(self, nbytes: int) -> None:
        _check(library().cs_renderer_set_scratch_limit(self.handle, nbytes))

    def set_lanes(self, lanes: int) -> None:
        """Batches in flight at most (1-4); submit / poll publishes them as they finish."""
        _check(library().cs_renderer_set_lanes(self.handle, lanes))

    def set_ordered_compute(self, ordered: bool) -> None:
        """True (default): every lane's kernels in batch order on one stream, shared
        sources pooled per render window; False: lanes compute side by side."""
        _check(library().cs_renderer_set_ordered_compute(self.handle, int(bool(ordered))))

    def fail_allocations(self, count: int) -> None:
        """Test hook: the next `count` batch-arena allocations report out of memory
        (host-side fault injection; the device is not touched)."""
        _check(library().cs_renderer_fail_allocations(self.handle, count))

    @property
    def deferred_launches(self) -> int:
        return int(library().cs_renderer_deferred_launches(self.handle))

    def host_ms(self) -> dict[str, float]:
        """Host milliseconds spent staging batches so far, per phase, then the device
        milliseconds of the published batches' downloads and kernels."""
        out = (ctypes.c_double * 16)()
        count = library().cs_renderer_host_ms(self.handle, out, 16)
        names = ("index", "budget", "segments", "shared", "arena", "pieces", "copy", "wait", "d2h_device",
                 "kernels_device")
        return {names[i] if i < len(names) else str(i): float(out[i]) for i in range(count)}

    def set_shared_sources(self, enable: bool) -> None:
        """Render each voice source shared by several voices once per batch (the
        default), or resample every voice frame inline (the plain path)."""
        _check(library().cs_renderer_set_shared_sources(self.handle, int(enable)))

    def prepare(self, plans: list[Plan]) -> Prepared:
        return Prepared(self, plans)

    def render_window(self, plans: list[Plan], publish: Callable[[RenderBatch, int], None],
                      refill: Optional[Callable[[bool], list[Plan]]] = None, copy: bool = True) -> None:
        """Render every plan; ``publish(batch, first)`` receives each finished batch.

        ``refill(wait)`` may return more plans (or an empty list when none are ready),
        like the reference's Refill callback.  With ``copy=False`` the batch's PCM is
        a view of the renderer's page-locked download buffer, valid only until
        ``publish`` returns (copy what must outlive the call), as in the C ABI.
        """
        array = c_plans(plans)
        keep = [array]
        errors = []

        def on_publish(_user, batch_ptr, first):
            try:
                b = batch_ptr.contents
                if copy:
                    pcm = _copy_out(b.pcm, b.pcm_samples, np.int16)
                elif b.pcm_samples:
                    pcm = np.ctypeslib.as_array(ctypes.cast(b.pcm, ctypes.POINTER(ctypes.c_int16)),
                                                shape=(b.pcm_samples,))
                else:
                    pcm = np.zeros(0, np.int16)
                results = np.frombuffer(ctypes.string_at(b.results, b.result_count * TAIL_RESULT.itemsize),
                                        TAIL_RESULT).copy() if b.result_count else np.zeros(0, TAIL_RESULT)
                indices = [ctypes.cast(b.job_indices, ctypes.POINTER(ctypes.c_size_t))[i]
                           for i in range(b.job_index_count)] if b.job_index_count else []
                publish(RenderBatch(pcm, results, b.kernel_seconds, b.failed_scratch_bytes, indices), first)
            except Exception as exc:  # surfaced after the C call returns
                errors.append(exc)

        def on_refill(_user, wait, plans_out, count_out):
            if refill is None:
                return 0
            more = refill(bool(wait))
            if not more:
                return 0
            extra = c_plans(more)
            keep.append((extra, more))
            plans_out[0] = ctypes.cast(extra, ctypes.c_void_p)
            count_out[0] = len(more)
            return 1

        publish_cb, refill_cb = PUBLISH(on_publish), REFILL(on_refill)
        status = library().cs_render_window(self.handle, array, len(plans), ctypes.cast(publish_cb, ctypes.c_void_p),
                                            ctypes.cast(refill_cb, ctypes.c_void_p), None)
        if errors:
            raise errors[0]
        _check(status)

    # ---- serving: non-blocking submission (continuous batching) -------------------

    def submit(self, plans: list[Plan]) -> int:
        """Queues plans for rendering and returns at once (after launching what the
        free stream lanes take); returns the ticket of the first plan.  Tickets
        number submitted plans in order."""
        array = c_plans(plans)
        ticket = ctypes.c_uint64()
        _check(library().cs_submit(self.handle, array, len(plans), ctypes.byref(ticket)))
        if not hasattr(self, "_submitted"):
            self._submitted = {}
        self._submitted[ticket.value] = (ticket.value + len(plans), array, plans)
        return ticket.value

    def poll(self, publish: Callable[[RenderBatch, int], None], wait: bool = False) -> int:
        """Publishes finished batches in order (``publish(batch, first_ticket)``),
        waiting for the oldest one when ``wait``, and admits queued plans into the
        freed lanes; returns the jobs published."""
        errors = []

        def on_publish(_user, batch_ptr, first):
            try:
                b = batch_ptr.contents
                pcm = _copy_out(b.pcm, b.pcm_samples, np.int16)
                results = np.frombuffer(ctypes.string_at(b.results, b.result_count * TAIL_RESULT.itemsize),
                                        TAIL_RESULT).copy() if b.result_count else np.zeros(0, TAIL_RESULT)
                publish(RenderBatch(pcm, results, b.kernel_seconds, b.failed_scratch_bytes, []), first)
            except Exception as exc:
                errors.append(exc)

        callback = PUBLISH(on_publish)
        count = ctypes.c_size_t()
        status = library().cs_poll(self.handle, int(wait), ctypes.cast(callback, ctypes.c_void_p), None,
                                   ctypes.byref(count))
        if errors:
            raise errors[0]
        _check(status)
        # Release the arrays of submissions whose jobs have all been published.
        done = self.pending_jobs == 0
        for key in [k for k, v in getattr(self, "_submitted", {}).items() if done]:
            del self._submitted[key]
        return count.value

    @property
    def pending_jobs(self) -> int:
        return library().cs_pending_jobs(self.handle)

    @property
    def device(self) -> str:
        return library().cs_renderer_device(self.handle).decode()

    @property
    def peak_bytes(self) -> int:
        return library().cs_peak_bytes(self.handle)

    @property
    def sample_cache_budget(self) -> int:
        return library().cs_sample_cache_budget(self.handle)

    @property
    def peak_waiting_bytes(self) -> int:
        return library().cs_peak_waiting_bytes(self.handle)

    @property
    def spilled_bytes(self) -> int:
        return library().cs_spilled_bytes(self.handle)

    @property
    def downloaded_bytes(self) -> int:
        return library().cs_downloaded_bytes(self.handle)
