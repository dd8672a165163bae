"""ORACLE (test infrastructure): Python access to the plain-C restatement.

``oracle/liboracle.so`` (built by ``oracle/Makefile`` from ``oracle/cs_oracle*.c``)
restates the reference's render path on the CPU.  Only tests/,
``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg use it; the GPU product
never calls it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

from claysampler_b200.plans import TAIL_RESULT, Plan, c_plans

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"
_lib = None


def build() -> Path:
    sources = list(HERE.glob("cs_oracle*.c")) + [HERE.parent / "include" / "claysampler_b200.h"]
    if not LIB.exists() or any(s.stat().st_mtime > LIB.stat().st_mtime for s in sources):
        result = subprocess.run(["make", "-s", "-C", str(HERE)], capture_output=True, text=True)
        if result.returncode:
            raise RuntimeError("oracle build failed:\n" + result.stdout + result.stderr)
    return LIB


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        build()
        _lib = ctypes.CDLL(str(LIB))
        vp, i32 = ctypes.c_void_p, ctypes.c_int
        _lib.oracle_finish_natural.restype = ctypes.c_size_t
        _lib.oracle_finish_natural.argtypes = [vp, vp, i32, i32, i32, i32, vp, vp]
        _lib.oracle_finish_stereo.restype = ctypes.c_size_t
        _lib.oracle_finish_stereo.argtypes = [vp, vp, i32, i32, vp, vp]
        if hasattr(_lib, "oracle_synthesize"):
            _lib.oracle_synthesize.argtypes = [vp, i32, vp, i32, i32, vp]
            _lib.oracle_synthesize_fp64_resampler.argtypes = [vp, i32, vp, i32, i32, vp]
        _lib.oracle_assess.restype = ctypes.c_size_t
        _lib.oracle_assess.argtypes = [vp, i32, vp, i32, vp, i32, vp, vp]
        _lib.oracle_match_group.argtypes = [vp, i32, i32]
        _lib.oracle_pack_accepted.restype = ctypes.c_size_t
        _lib.oracle_pack_accepted.argtypes = [vp, i32, vp, i32, vp, vp]
    return _lib


def finish(mix: np.ndarray, plans: list[Plan], natural: bool = True, rate: int = 44100, window: int = 2205,
           quality: bool = False) -> tuple[np.ndarray, np.ndarray]:
    """(packed PCM16, results) of the reference finishing stages for a batch mix."""
    array = c_plans(plans)
    results = np.zeros(len(plans), TAIL_RESULT)
    frames = sum(p.frames for p in plans)
    packed = np.zeros(frames * (1 if natural else 2), np.int16)
    if natural:
        mix = np.ascontiguousarray(mix, np.float32)
        n = lib().oracle_finish_natural(mix.ctypes.data, array, len(plans), rate, window, int(quality),
                                        results.ctypes.data, packed.ctypes.data)
    else:
        mix = np.ascontiguousarray(mix, np.int16)
        n = lib().oracle_finish_stereo(mix.ctypes.data, array, len(plans), int(quality), results.ctypes.data,
                                       packed.ctypes.data)
    return packed[:n], results


def synthesize(plans: list[Plan], bank: np.ndarray, natural: bool = True, threads: int = 0,
               fp64_resampler: bool = False) -> np.ndarray:
    """Restated mix: (frames, 2) float32 in natural mode, int16 otherwise.  With
    `fp64_resampler` the 48-tap interpolation runs in FP64 on the unrounded sinc
    table (the rest of the voice math stays FP32), which bounds the FP32
    resampler's rounding error independently of the reference's arithmetic."""
    frames = sum(p.frames for p in plans)
    out = np.zeros((frames, 2), np.float32 if natural else np.int16)
    array = c_plans(plans)
    bank = np.ascontiguousarray(bank, np.float32)
    call = lib().oracle_synthesize_fp64_resampler if fp64_resampler else lib().oracle_synthesize
    call(array, len(plans), bank.ctypes.data if bank.size else None, int(natural), threads or os.cpu_count() or 1,
         out.ctypes.data)
    return out


def assess(finished: np.ndarray, results: np.ndarray, plans: list[Plan], natural: bool = True, config=None,
           group_minimum: int = 0) -> tuple[np.ndarray, np.ndarray]:
    """(accepted PCM16, results) of the reference's quality gate, group volume and
    accepted packing (src/cuda/quality.cu) applied to a finished batch."""
    from claysampler_b200.plans import default_audio_config
    config = default_audio_config() if config is None else np.asarray(config)
    finished = np.ascontiguousarray(finished, np.int16)
    out = np.array(results, TAIL_RESULT, copy=True)
    accepted = np.zeros(max(finished.size, 1), np.int16)
    array = c_plans(plans)
    n = lib().oracle_assess(finished.ctypes.data, 1 if natural else 2, array, len(plans), config.ctypes.data,
                            group_minimum, out.ctypes.data, accepted.ctypes.data)
    return accepted[:n], out
