"""Host-side helpers on the CPU: the seeded workload generators' file formats and
length distribution, and the plan image / cs_plan marshalling the renderer's
Python calls go through."""
import struct
import wave

import numpy as np
import pytest

from claysampler_b200 import plans as P
from claysampler_b200 import workload as W


def test_pareto_lengths_are_truncated_heavy_tailed_and_seeded():
    draw = lambda seed: W.pareto_seconds(np.random.default_rng(seed), 100_000)
    lengths = draw(7)
    assert np.array_equal(lengths, draw(7))
    assert not np.array_equal(lengths, draw(8))
    assert lengths.min() >= 2.0 and lengths.max() <= 600.0
    assert np.median(lengths) < lengths.mean()
    # P(X > 60 s) of a Pareto(1.5) on [2, 600]: about 0.59 %; the count is binomial.
    ratio = (2.0 / 600.0) ** 1.5
    tail = ((2.0 / 60.0) ** 1.5 - ratio) / (1 - ratio)
    expected = tail * len(lengths)
    assert abs(np.count_nonzero(lengths > 60.0) - expected) < 5 * np.sqrt(expected)


@pytest.mark.parametrize("value, encoded", [(0, b"\x00"), (0x40, b"\x40"), (0x7F, b"\x7f"), (0x80, b"\x81\x00"),
                                            (0x2000, b"\xc0\x00"), (0x3FFF, b"\xff\x7f"),
                                            (0x4000, b"\x81\x80\x00"), (0x0FFFFFFF, b"\xff\xff\xff\x7f")])
def test_midi_variable_length_quantities(value, encoded):
    assert W._varlen(value) == encoded


def test_midi_file_layout(tmp_path):
    path = tmp_path / "t.mid"
    on, off = b"\x90\x3c\x64", b"\x80\x3c\x00"
    # Out of order on purpose: the writer sorts by tick, then by the tie order.
    W.write_midi(path, [(960, 1, on), (0, 1, on), (960, 0, off)], end_tick=1920)
    data = path.read_bytes()
    assert data[:4] == b"MThd" and struct.unpack(">IHHH", data[4:14]) == (6, 0, 1, W.PPQ)
    assert data[14:18] == b"MTrk"
    (length,) = struct.unpack(">I", data[18:22])
    track = data[22:]
    assert len(track) == length
    tempo = b"\x00\xff\x51\x03" + W.TEMPO_US.to_bytes(3, "big")
    # delta 0 on, delta 960 (0x87 0x40) off before the second on, then the end of track after 960 more.
    assert track == tempo + b"\x00" + on + b"\x87\x40" + off + b"\x00" + on + b"\x87\x40\xff\x2f\x00"
    assert W.seconds_to_tick(1.0) == int(W.TICKS_PER_SECOND) == 960


@pytest.mark.parametrize("bits", [16, 24])
def test_wav_writer_round_trips(tmp_path, bits):
    rng = np.random.default_rng(3)
    data = rng.uniform(-1, 1, (257, 2)).astype(np.float64)
    data[0] = [-1.0, 0.99999999]                     # the clipped ends of the range
    path = tmp_path / f"t{bits}.wav"
    W.write_wav(path, data, rate=48000, bits=bits)
    with wave.open(str(path)) as f:
        assert (f.getnchannels(), f.getsampwidth(), f.getframerate(), f.getnframes()) == (2, bits // 8, 48000, 257)
        raw = f.readframes(257)
    scale = float(1 << (bits - 1))
    want = np.clip(np.round(data * scale), -scale, scale - 1).astype(np.int64)
    if bits == 16:
        got = np.frombuffer(raw, "<i2").astype(np.int64)
    else:
        b = np.frombuffer(raw, np.uint8).reshape(-1, 3).astype(np.int64)
        got = b[:, 0] | (b[:, 1] << 8) | (b[:, 2] << 16)
        got = np.where(got >= 1 << 23, got - (1 << 24), got)
    assert np.array_equal(got.reshape(257, 2), want)


def _plan(seed=0):
    rng = np.random.default_rng(seed)
    spans = np.zeros(3, P.VOICE_SPAN)
    spans["begin"] = [0, 100, 250]
    spans["end"] = [400, 300, 900]
    points = np.zeros(4, P.CONTROL_POINT)
    points["frame"] = [0, 0, 0, 500]
    points["value"] = rng.uniform(0, 1, 4)
    modulation = np.zeros(1, P.VOICE_MODULATION)
    modulation["depth"] = 0.5
    return P.Plan(spans, points, np.array([0, 1, 2, 4], np.int64), modulation, np.array([10, 20], np.int32),
                  frames=1000, music_end=900, limit=1500, fade_frames=64, body_frames=800, volume_group=2)


def test_plan_image_round_trips():
    plan = _plan()
    blob = plan.to_blob()
    again = P.Plan.from_blob(blob)
    assert again.to_blob() == blob
    assert (again.frames, again.music_end, again.limit, again.fade_frames, again.volume_group) == (1000, 900, 1500,
                                                                                                  64, 2)
    assert again.track_count == 3 and np.array_equal(again.track(2)["frame"], [0, 500])
    assert again.voice_frames() == 400 + 200 + 650
    with pytest.raises(ValueError):
        P.Plan.from_blob(blob[:-1])
    with pytest.raises(ValueError):
        P.Plan.from_blob(b"XXXX" + blob[4:])


def test_cs_plan_views_are_cached_until_the_plan_changes():
    plan = _plan()
    view = plan.as_c()
    assert plan.as_c() is view
    assert view.span_count == 3 and view.track_count == 3 and view.frames == 1000
    assert view.spans == plan.spans.ctypes.data
    plan.points = plan.points.copy()                 # a replaced array is a new view
    fresh = plan.as_c()
    assert fresh is not view and fresh.points == plan.points.ctypes.data
    plan.frames = 999                                # so is a changed field
    assert plan.as_c().frames == 999


def test_plan_set_builds_its_array_once():
    plans = P.PlanSet([_plan(1), _plan(2)])
    assert P.c_plans(plans) is plans.array is P.c_plans(plans)
    listed = P.c_plans(list(plans))
    assert listed is not plans.array
    for a, b in zip(listed, plans.array):
        assert (a.spans, a.points, a.frames) == (b.spans, b.points, b.frames)
