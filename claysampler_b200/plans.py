"""Planned render jobs as numpy arrays.

A :class:`Plan` holds one job's ``cs_plan`` arrays (the reference's
``clay::RenderPlan``, src/render/plan.h:9-20).  The record dtypes below are
byte-compatible with the C structs in ``include/claysampler_b200.h`` (and with the
reference's src/cuda/render_types.h), so arrays pass through ctypes unchanged.
"""
from __future__ import annotations

import ctypes
import struct
from dataclasses import dataclass, field

import numpy as np

VOICE_FILTER = np.dtype([("type", "<i4"), ("cutoff", "<f4"), ("resonance", "<f4"),
                         ("bandwidth", "<f4"), ("gain", "<f4")], align=True)
ENVELOPE_SHAPE = np.dtype(
    [(n, "<i4") for n in ("attackStart", "holdStart", "decayStart", "releaseStart", "fadeStart")]
    + [(n, "<f4") for n in ("start", "attackStep", "decayRate", "sustain", "releaseValue", "releaseRate",
                             "fadeValue", "fadeStep", "depth", "releaseSeconds")], align=True)
VOICE_SPAN = np.dtype(
    [("sample", "<u8"), ("position", "<f8"), ("step", "<f8"), ("pitchSlope", "<f8")]
    + [(n, "<i4") for n in ("channels", "begin", "end", "sourceEnd", "loopFirst", "loopEnd", "loopCrossfade",
                             "stereoMatrix", "generator")]
    + [("noiseSeed", "<u4")]
    + [(n, "<i4") for n in ("noiseStart", "firstModulation", "modulationCount", "firstLfo", "lfoCount",
                             "filterTrack", "nextFilteredSpan")]
    + [("filteredOffset", "<u8"), ("phaseOffset", "<u8"), ("variablePitch", "<i4"), ("minimumPitchRatio", "<f4"),
       ("filterControls", "<i4", (4,)), ("sampleRate", "<i4"), ("filters", VOICE_FILTER, (5,)),
       ("extraEnvelope", ENVELOPE_SHAPE, (2,)), ("activeEnvelope", "<i4", (2,))]
    + [(n, "<i4") for n in ("attackStart", "holdStart", "decayStart", "releaseStart", "fadeStart", "bendEnd")]
    + [(n, "<f4") for n in ("gain", "pan", "left", "right", "start", "attackStep", "decayRate", "sustain",
                             "releaseValue", "releaseRate", "fadeValue", "fadeStep", "widthDirect", "widthCross",
                             "positionLeft", "positionRight", "width", "stereoPosition")], align=True)
CONTROL_POINT = np.dtype([("frame", "<i4"), ("value", "<f4"), ("step", "<f4")], align=True)
VOICE_MODULATION = np.dtype([("first", "<i4"), ("last", "<i4"), ("target", "<i4"), ("depth", "<f4"),
                             ("shapeFirst", "<i4"), ("shapeLast", "<i4")], align=True)
AUDIO_METRICS = np.dtype([(n, "<f8") for n in ("median", "quartile", "silentFraction", "clippedFraction",
                                                "bodyRms", "targetRms", "gain")]
                         + [("longestSilence", "<i4"), ("clipped", "<i4"), ("verdict", "<i4"),
                            ("measured", "u1")], align=True)
TAIL_RESULT = np.dtype([("offset", "<u8")]
                       + [(n, "<i4") for n in ("frames", "dataFrames", "fade", "peak", "first", "last", "status")]
                       + [("scale", "<f4"), ("audio", AUDIO_METRICS)], align=True)
AUDIO_CONFIG = np.dtype([(n, "<i4") for n in ("rate", "window", "maxFrames", "minPeak")] + [("enabled", "u1")]
                        + [(n, "<f8") for n in ("minMedian", "minQuartile", "silencePower", "maxSilentFraction",
                                                 "maxSilentFrames", "maxClippedFraction")], align=True)

assert VOICE_SPAN.itemsize == 472 and CONTROL_POINT.itemsize == 12
assert VOICE_MODULATION.itemsize == 24 and TAIL_RESULT.itemsize == 112 and AUDIO_CONFIG.itemsize == 72

TAIL_STATUS = ["ok", "duration", "nonfinite", "peak", "audioDuration", "quietPerformance", "excessiveSilence",
               "silentAudio", "clipping", "silentBody", "incompleteGroup", "scratchMemory"]

_HEADER = struct.Struct("<4sI12iQQ")


class CPlan(ctypes.Structure):
    """ctypes mirror of ``cs_plan``."""
    _fields_ = [("spans", ctypes.c_void_p), ("points", ctypes.c_void_p), ("track_offsets", ctypes.c_void_p),
                ("modulation", ctypes.c_void_p), ("onsets", ctypes.c_void_p),
                ("span_count", ctypes.c_int32), ("track_count", ctypes.c_int32),
                ("modulation_count", ctypes.c_int32), ("onset_count", ctypes.c_int32),
                ("filter_tracks", ctypes.c_int32), ("frames", ctypes.c_int32), ("music_end", ctypes.c_int32),
                ("limit", ctypes.c_int32), ("fade_frames", ctypes.c_int32), ("tail_clipped", ctypes.c_int32),
                ("body_frames", ctypes.c_int32), ("volume_group", ctypes.c_uint64)]


@dataclass
class Plan:
    spans: np.ndarray
    points: np.ndarray
    track_offsets: np.ndarray
    modulation: np.ndarray
    onsets: np.ndarray
    filter_tracks: int = 0
    frames: int = 0
    music_end: int = 0
    limit: int = 0
    fade_frames: int = 0
    tail_clipped: int = 0
    body_frames: int = 0
    volume_group: int = 0
    _keep: list = field(default_factory=list, repr=False)

    @classmethod
    def from_blob(cls, blob: bytes) -> "Plan":
        (magic, version, filter_tracks, frames, music_end, limit, fade_frames, tail_clipped, body_frames,
         spans, tracks, mods, onsets, _, group, points) = _HEADER.unpack_from(blob, 0)
        if magic != b"CSPL" or version != 1:
            raise ValueError("not a plan image")
        offset = _HEADER.size

        def take(dtype, count):
            # Copy raw bytes (numpy's copy of a padded record dtype drops the padding).
            nonlocal offset
            nbytes = np.dtype(dtype).itemsize * count
            array = np.frombuffer(bytearray(blob[offset:offset + nbytes]), dtype=dtype, count=count)
            offset += nbytes
            return array
        plan = cls(take(VOICE_SPAN, spans), None, None, None, None, filter_tracks, frames, music_end, limit,
                   fade_frames, tail_clipped, body_frames, group)
        plan.track_offsets = take(np.int64, tracks + 1)
        plan.points = take(CONTROL_POINT, points)
        plan.modulation = take(VOICE_MODULATION, mods)
        plan.onsets = take(np.int32, onsets)
        if offset != len(blob):
            raise ValueError("truncated plan image")
        return plan

    def to_blob(self) -> bytes:
        head = _HEADER.pack(b"CSPL", 1, self.filter_tracks, self.frames, self.music_end, self.limit,
                            self.fade_frames, self.tail_clipped, self.body_frames, len(self.spans),
                            len(self.track_offsets) - 1, len(self.modulation), len(self.onsets), 0,
                            self.volume_group, len(self.points))
        return b"".join([head, self.spans.tobytes(), self.track_offsets.astype(np.int64).tobytes(),
                         self.points.tobytes(), self.modulation.tobytes(), self.onsets.astype(np.int32).tobytes()])

    def pin(self) -> "Plan":
        """Moves the plan's arrays into page-locked host memory, from which the
        renderer's copy engines upload them directly (no staging copy)."""
        import torch
        keep = []
        for name in ("spans", "points", "track_offsets", "modulation", "onsets"):
            array = np.ascontiguousarray(getattr(self, name))
            buffer = torch.empty(max(array.nbytes, 1), dtype=torch.uint8, pin_memory=True)
            pinned = buffer.numpy()[:array.nbytes].view(array.dtype)
            pinned[...] = array
            setattr(self, name, pinned)
            keep.append(buffer)
        self._pinned = keep
        return self

    @property
    def track_count(self) -> int:
        return len(self.track_offsets) - 1

    def track(self, index: int) -> np.ndarray:
        return self.points[self.track_offsets[index]:self.track_offsets[index + 1]]

    def _c_key(self) -> tuple:
        return (id(self.spans), id(self.points), id(self.track_offsets), id(self.modulation), id(self.onsets),
                self.filter_tracks, self.frames, self.music_end, self.limit, self.fade_frames, self.tail_clipped,
                self.body_frames, self.volume_group)

    def as_c(self) -> CPlan:
        """The plan as a ``cs_plan`` view of its arrays, cached until a field or an
        array of the plan is replaced (the cache holds the arrays it points to)."""
        key = self._c_key()
        cached = self.__dict__.get("_c")
        if cached is not None and cached[0] == key:
            return cached[1]
        arrays = [np.ascontiguousarray(a) for a in (self.spans, self.points, self.track_offsets.astype(np.int64),
                                                    self.modulation, self.onsets.astype(np.int32))]
        ptr = [a.ctypes.data if a.size else None for a in arrays]
        view = CPlan(ptr[0], ptr[1], ptr[2], ptr[3], ptr[4], len(self.spans), self.track_count,
                     len(self.modulation), len(self.onsets), self.filter_tracks, self.frames, self.music_end,
                     self.limit, self.fade_frames, self.tail_clipped, self.body_frames, self.volume_group)
        self._keep = arrays
        self._c = (key, view)
        return view

    def voice_frames(self) -> int:
        return int(np.sum(self.spans["end"].astype(np.int64) - self.spans["begin"]))


class PlanSet(tuple):
    """An immutable sequence of plans with its ``cs_plan`` array built once, for
    callers that render the same plans repeatedly (as a C caller keeps its plan
    array); the renderer's calls take it wherever they take a list of plans."""

    def __new__(cls, plans=()):
        self = super().__new__(cls, plans)
        self.array = _build_array(self)
        return self


def _build_array(plans):
    return (CPlan * len(plans))(*[plan.as_c() for plan in plans])


def c_plans(plans: list[Plan]):
    """A ctypes array of ``cs_plan`` views (the plans keep their buffers alive)."""
    if isinstance(plans, PlanSet):
        return plans.array
    return _build_array(plans)


def default_audio_config(rate: int = 44100, quality: bool = False) -> np.ndarray:
    """audioConfig() of the reference CLI (src/main.cpp:169-187)."""
    power = lambda dbfs: 4294967296.0 * 10.0 ** (dbfs / 10)  # noqa: E731
    config = np.zeros((), AUDIO_CONFIG)
    config["rate"] = rate
    config["window"] = int(np.rint(rate / 20.0))
    config["maxFrames"] = 375 * rate
    config["minPeak"] = 32
    config["enabled"] = 1 if quality else 0
    config["minMedian"] = -38
    config["minQuartile"] = -45
    config["silencePower"] = power(-70)
    config["maxSilentFraction"] = 0.75
    config["maxSilentFrames"] = 10.0 * rate
    config["maxClippedFraction"] = 0.0001
    return config
