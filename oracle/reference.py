"""Test infrastructure: Python access to the reference's own code built for the host.

``oracle/_ref/libclayref.so`` (built by ``oracle/ref/Makefile`` from the
reference sources) exposes the reference planner and the reference's per-voice
render math (src/cuda/render.cu compiled as host C++).  Only tests and the
CPU-baseline leg of ``bench.py`` use this module; the GPU product never does.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

from claysampler_b200.plans import Plan, c_plans

HERE = Path(__file__).resolve().parent
REF_DIR = HERE / "_ref"
TAIL = {"natural": 0, "orig": 1, "custom": 2}


def build(root=None, quiet: bool = True) -> bool:
    """Compile oracle/_ref from the reference checkout at `root` (default: the
    CLAY_REFERENCE_ROOT environment variable) when its sources are present; without
    them the prebuilt oracle/_ref is used as it is."""
    root = root or os.environ.get("CLAY_REFERENCE_ROOT")
    if not root or not (Path(root) / "src" / "cuda" / "render.cu").exists():
        return available()
    result = subprocess.run(["make", "-s", "-C", str(HERE / "ref"), f"REF={root}"],
                            capture_output=quiet, text=True)
    if result.returncode:
        raise RuntimeError("oracle/_ref build failed:\n" + (result.stdout or "") + (result.stderr or ""))
    return available()


def available() -> bool:
    return (REF_DIR / "libclayref.so").exists() and (REF_DIR / "libsndfile_shim.so").exists()


_lib = None
_gpu = None


def gpu_available() -> bool:
    return (REF_DIR / "libclayref_gpu.so").exists()


def gpu_lib():
    global _gpu
    if _gpu is None:
        if not gpu_available():
            raise RuntimeError("oracle/_ref/libclayref_gpu.so is not built")
        _gpu = ctypes.CDLL(str(REF_DIR / "libclayref_gpu.so"))
        _gpu.ref_gpu_last_error.restype = ctypes.c_char_p
        _gpu.ref_gpu_synthesize.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_size_t,
                                            ctypes.c_void_p]
        _gpu.ref_gpu_synthesize_timed.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_size_t,
                                                  ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_float)]
    return _gpu


def synthesize_gpu(plans: list[Plan], bank: np.ndarray) -> np.ndarray:
    """The reference's own render kernels (src/cuda/render.cu built for the GPU with
    its NVRTC defaults) on the current CUDA device: the float mix, (frames, 2)."""
    frames = sum(p.frames for p in plans)
    out = np.zeros((frames, 2), np.float32)
    array = c_plans(plans)
    bank = np.ascontiguousarray(bank, np.float32)
    if gpu_lib().ref_gpu_synthesize(array, len(plans), bank.ctypes.data if bank.size else None, bank.size,
                                    out.ctypes.data):
        raise RuntimeError(gpu_lib().ref_gpu_last_error().decode())
    return out


def time_gpu(plans: list[Plan], bank: np.ndarray, repeats: int = 5) -> float:
    """Mean device milliseconds of the reference's synthesis launches (render.cu on
    this GPU, one segment) over `repeats` runs after a first one."""
    frames = sum(p.frames for p in plans)
    out = np.zeros((frames, 2), np.float32)
    array = c_plans(plans)
    bank = np.ascontiguousarray(bank, np.float32)
    ms = ctypes.c_float()
    if gpu_lib().ref_gpu_synthesize_timed(array, len(plans), bank.ctypes.data if bank.size else None, bank.size,
                                          out.ctypes.data, repeats, ctypes.byref(ms)):
        raise RuntimeError(gpu_lib().ref_gpu_last_error().decode())
    return float(ms.value)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise RuntimeError("oracle/_ref is not built")
        _lib = ctypes.CDLL(str(REF_DIR / "libclayref.so"))
        _lib.ref_session_create.restype = ctypes.c_void_p
        _lib.ref_session_create.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_size_t]
        _lib.ref_session_destroy.argtypes = [ctypes.c_void_p]
        _lib.ref_free.argtypes = [ctypes.c_void_p]
        _lib.ref_session_plan.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int,
                                          ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                          ctypes.c_int, ctypes.c_int, ctypes.c_ulonglong,
                                          ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_size_t),
                                          ctypes.c_char_p, ctypes.c_size_t]
        _lib.ref_session_bank.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p),
                                          ctypes.POINTER(ctypes.c_size_t)]
        _lib.ref_sinc_table.argtypes = [ctypes.c_void_p]
        _lib.ref_synthesize.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int,
                                        ctypes.c_int, ctypes.c_void_p]
    return _lib


class RefSession:
    """The reference planner with one shared sample bank (clay::AudioBank)."""

    def __init__(self):
        error = ctypes.create_string_buffer(1024)
        self.handle = lib().ref_session_create(str(REF_DIR / "libsndfile_shim.so").encode(), error, 1024)
        if not self.handle:
            raise RuntimeError(error.value.decode())

    def close(self):
        if self.handle:
            lib().ref_session_destroy(self.handle)
            self.handle = None

    def __del__(self):
        self.close()

    def plan(self, sfz, midi, rate=44100, tail="natural", max_audio=-1.0, tail_max=-1.0, tail_fade_ms=-1,
             quality=False, group_volume=False, group=0) -> Plan:
        blob = ctypes.c_void_p()
        size = ctypes.c_size_t()
        error = ctypes.create_string_buffer(4096)
        status = lib().ref_session_plan(self.handle, str(sfz).encode(), str(midi).encode(), rate, TAIL[tail],
                                        max_audio, tail_max, tail_fade_ms, int(quality), int(group_volume),
                                        group, ctypes.byref(blob), ctypes.byref(size), error, 4096)
        if status:
            raise RuntimeError(error.value.decode())
        try:
            data = ctypes.string_at(blob.value, size.value)
        finally:
            lib().ref_free(blob)
        return Plan.from_blob(data)

    def bank(self) -> np.ndarray:
        pointer = ctypes.c_void_p()
        floats = ctypes.c_size_t()
        lib().ref_session_bank(self.handle, ctypes.byref(pointer), ctypes.byref(floats))
        if not floats.value:
            return np.zeros(0, np.float32)
        return np.ctypeslib.as_array(ctypes.cast(pointer, ctypes.POINTER(ctypes.c_float)),
                                     shape=(floats.value,)).copy()


def sinc_table() -> np.ndarray:
    out = np.zeros(48 * 2049, np.float32)
    lib().ref_sinc_table(out.ctypes.data)
    return out.reshape(48, 2049)


def synthesize(plans: list[Plan], bank: np.ndarray, natural: bool = True, threads: int = 0) -> np.ndarray:
    """Reference mix: (frames, 2) float32 in natural mode, (frames, 2) int16 otherwise."""
    frames = sum(p.frames for p in plans)
    out = np.zeros((frames, 2), np.float32 if natural else np.int16)
    array = c_plans(plans)
    bank = np.ascontiguousarray(bank, np.float32)
    lib().ref_synthesize(array, len(plans), bank.ctypes.data if bank.size else None, int(natural),
                         threads or os.cpu_count() or 1, out.ctypes.data)
    return out
