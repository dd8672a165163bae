"""The allocation-free natural finishing entry point (cs_finish_natural_static).

It serves callers that cannot allocate device memory while rendering — a
real-time audio host calling from its audio callback, where a device allocation
can block or synchronise past the callback's deadline, or an application that
owns the device-memory budget itself — by keeping the stage's intermediates in a
fixed static device array.  This test renders a batch through the regular
renderer, then finishes the same device-resident float mix through the
allocation-free entry point twice in a row (the array keeps the previous call's
contents) and requires the same PCM16 and results, within the tolerance the other
GPU tests use (<= 1 LSB).  It runs last so that a failure here cannot hide others.
"""
import ctypes

import numpy as np
import pytest

from conftest import gpu_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not gpu_available(), reason="needs a CUDA GPU")]


class FinishJob(ctypes.Structure):
    _fields_ = [("frames", ctypes.c_int32), ("music_end", ctypes.c_int32), ("limit", ctypes.c_int32),
                ("fade_frames", ctypes.c_int32)]


def test_static_finishing_matches_renderer(plain_small, batch_mini):
    import torch

    from claysampler_b200.host import Host
    from claysampler_b200.plans import TAIL_RESULT
    from claysampler_b200.renderer import Renderer, library

    host = Host()
    plans = [host.plan(j.sfz, j.midi) for j in plain_small + batch_mini]
    bank = host.bank()
    renderer = Renderer(natural=True)
    renderer.upload_samples(bank)
    prepared = renderer.prepare(plans)
    prepared.run()
    expected_pcm, expected = prepared.collect()
    mix = prepared.mix()
    prepared.close()
    renderer.close()

    lib = library()
    lib.cs_finish_natural_static.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                             ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    lib.cs_finish_natural_static_error.restype = ctypes.c_char_p
    jobs = (FinishJob * len(plans))(*[FinishJob(p.frames, p.music_end, p.limit, p.fade_frames) for p in plans])
    frames = sum(p.frames for p in plans)
    mix_d = torch.from_numpy(mix).cuda()
    # Both calls' outputs are allocated up front, so that device memory can be
    # compared across the second call: after the first call on a device (which
    # loads the module holding the static array), a call allocates nothing.
    packed_d = [torch.full((frames,), 12345, dtype=torch.int16, device="cuda") for _ in range(2)]
    results_d = [torch.zeros(len(plans) * TAIL_RESULT.itemsize, dtype=torch.uint8, device="cuda") for _ in range(2)]
    free_before = None
    for call in range(2):
        torch.cuda.synchronize()
        if call == 1:
            free_before = torch.cuda.mem_get_info()[0]
        status = lib.cs_finish_natural_static(mix_d.data_ptr(), jobs, len(plans), 44100, 2205,
                                              packed_d[call].data_ptr(), results_d[call].data_ptr(), None)
        assert status == 0, lib.cs_finish_natural_static_error().decode()
        torch.cuda.synchronize()
        if call == 1:
            assert torch.cuda.mem_get_info()[0] == free_before, "the second call changed free device memory"
        results = np.frombuffer(results_d[call].cpu().numpy().tobytes(), TAIL_RESULT)
        for field in ("status", "frames", "dataFrames", "fade", "offset", "peak", "first", "last"):
            np.testing.assert_array_equal(results[field], expected[field], err_msg=f"call {call}: {field}")
        pcm = packed_d[call].cpu().numpy()[:expected_pcm.size]
        assert int(np.max(np.abs(pcm.astype(np.int32) - expected_pcm.astype(np.int32)))) <= 1, f"call {call}"


def test_static_finishing_rejects_oversized_calls():
    from claysampler_b200.renderer import library
    lib = library()
    lib.cs_finish_natural_static.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                             ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    lib.cs_finish_natural_static_error.restype = ctypes.c_char_p
    jobs = (FinishJob * 1)(FinishJob((1 << 23) + 1, 1, (1 << 23) + 2, 0))
    # No buffer is touched: the size check fails before anything is enqueued.
    status = lib.cs_finish_natural_static(ctypes.c_void_p(16), jobs, 1, 44100, 2205, ctypes.c_void_p(16),
                                          ctypes.c_void_p(16), None)
    assert status != 0
    assert b"exceed the limit" in lib.cs_finish_natural_static_error()
