"""Python access to the C++ host library (``include/claysampler_host.h``).

:class:`Host` mirrors the reference CLI's planning step (src/main.cpp:298-361):
an SFZ instrument and a Standard MIDI File become a :class:`~.plans.Plan` whose
spans index into the host's shared float32 sample bank.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import build
from .plans import Plan

TAIL = {"natural": 0, "orig": 1, "custom": 2}
_lib = None


def library() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not build.HOST_LIBRARY.exists():
            build.build_host()
        lib = ctypes.CDLL(str(build.HOST_LIBRARY))
        vp, sz = ctypes.c_void_p, ctypes.c_size_t
        lib.cs_host_last_error.restype = ctypes.c_char_p
        lib.cs_host_create.argtypes = [ctypes.POINTER(vp)]
        lib.cs_host_destroy.argtypes = [vp]
        lib.cs_host_free.argtypes = [vp]
        lib.cs_host_plan.argtypes = [vp, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int, ctypes.c_int,
                                     ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                     ctypes.c_uint64, ctypes.POINTER(vp), ctypes.POINTER(sz)]
        lib.cs_host_bank.argtypes = [vp, ctypes.POINTER(vp), ctypes.POINTER(sz)]
        lib.cs_host_release_bank.argtypes = [vp]
        lib.cs_write_wave.argtypes = [ctypes.c_char_p, vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        lib.cs_wave_complete.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int]
        _lib = lib
    return _lib


def _check(status: int) -> None:
    if status:
        raise RuntimeError(library().cs_host_last_error().decode(errors="replace"))


class Host:
    """Planner + sample bank, one per render session."""

    def __init__(self):
        handle = ctypes.c_void_p()
        _check(library().cs_host_create(ctypes.byref(handle)))
        self.handle = handle

    def close(self) -> None:
        if getattr(self, "handle", None):
            library().cs_host_destroy(self.handle)
            self.handle = None

    def __del__(self):
        self.close()

    def plan(self, sfz, midi, rate: int = 44100, tail: str = "natural", max_audio: float = -1.0,
             tail_max: float = -1.0, tail_fade_ms: int = -1, quality: bool = False, group_volume: bool = False,
             group: int = 0) -> Plan:
        image = ctypes.c_void_p()
        size = ctypes.c_size_t()
        _check(library().cs_host_plan(self.handle, str(sfz).encode(), str(midi).encode(), rate, TAIL[tail],
                                      max_audio, tail_max, tail_fade_ms, int(quality), int(group_volume), group,
                                      ctypes.byref(image), ctypes.byref(size)))
        try:
            return Plan.from_blob(ctypes.string_at(image.value, size.value))
        finally:
            library().cs_host_free(image)

    def bank(self) -> np.ndarray:
        pointer = ctypes.c_void_p()
        floats = ctypes.c_size_t()
        _check(library().cs_host_bank(self.handle, ctypes.byref(pointer), ctypes.byref(floats)))
        if not floats.value:
            return np.zeros(0, np.float32)
        return np.ctypeslib.as_array(ctypes.cast(pointer, ctypes.POINTER(ctypes.c_float)),
                                     shape=(floats.value,)).copy()

    def release_bank(self) -> None:
        _check(library().cs_host_release_bank(self.handle))


def write_wave(path, pcm: np.ndarray, data_frames: int, frames: int, rate: int, channels: int) -> None:
    pcm = np.ascontiguousarray(pcm, np.int16)
    _check(library().cs_write_wave(str(path).encode(), pcm.ctypes.data if pcm.size else None, data_frames, frames,
                                   rate, channels))


def wave_complete(path, rate: int, channels: int) -> bool:
    return bool(library().cs_wave_complete(str(path).encode(), rate, channels))
