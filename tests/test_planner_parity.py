"""The C++ host planner against the reference's own planner (oracle/_ref: the
reference's src/sfz, src/io/midi.cpp and src/render/plan.cpp built for the host).

Event scheduling, region and velocity-layer selection, voice stealing (choke and
note_polyphony), integer sample positions and output lengths are checked by
comparing the two plan images byte for byte, together with the decoded banks.
"""
import struct
import wave

import numpy as np
import pytest

from claysampler_b200 import workload
from claysampler_b200.host import Host


def same_plans(jobs, ref_session, **options):
    host = Host()
    for job in jobs:
        mine = host.plan(job.sfz, job.midi, **options)
        theirs = ref_session.plan(job.sfz, job.midi, **options)
        assert mine.to_blob() == theirs.to_blob(), f"{job.midi.name} {options}"
    assert np.array_equal(host.bank(), ref_session.bank())
    host.close()


@pytest.mark.parametrize("tail", ["natural", "orig"])
def test_plain_small_plans_match(plain_small, tail):
    from oracle import reference
    session = reference.RefSession() if reference.available() or reference.build() else pytest.skip("no oracle/_ref")
    same_plans(plain_small, session, tail=tail)


@pytest.mark.parametrize("tail", ["natural", "orig"])
def test_filtered_batch_plans_match(batch_mini, tail):
    from oracle import reference
    session = reference.RefSession() if reference.available() or reference.build() else pytest.skip("no oracle/_ref")
    same_plans(batch_mini, session, tail=tail)


def test_uneven_batch_plans_match(tmp_path):
    from oracle import reference
    session = reference.RefSession() if reference.available() or reference.build() else pytest.skip("no oracle/_ref")
    jobs = workload.write_uneven_batch(tmp_path, seed=9, jobs=6, presets=2, high=40.0)
    same_plans(jobs, session)


def _midi(path, data):
    path.write_bytes(b"MThd" + struct.pack(">IHHH", 6, 0, 1, 480) + b"MTrk" + struct.pack(">I", len(data)) + data)


def _tone(path, frames_a, value_a, frames_b, value_b):
    with wave.open(str(path), "wb") as stream:
        stream.setparams((1, 2, 44100, 0, "NONE", "not compressed"))
        stream.writeframes(struct.pack("<h", value_a) * frames_a + struct.pack("<h", value_b) * frames_b)


@pytest.mark.parametrize("options", [
    {"tail": "natural"}, {"tail": "orig"}, {"tail": "custom", "tail_max": 1.0, "tail_fade_ms": 100},
    {"tail": "custom", "tail_max": 4.0}, {"tail": "natural", "max_audio": 0.5},
])
def test_tail_fixture_plans_match(tmp_path, options):
    """The reference's tests/check_tail.py inputs: one-shot, looping with pedals
    and sostenuto, filter + LFO to pitch, hot volume with a pan CC."""
    from oracle import reference
    session = reference.RefSession() if reference.available() or reference.build() else pytest.skip("no oracle/_ref")
    _tone(tmp_path / "sample.wav", 44100 * 2 // 5, 1600, 44100 * 3, 12)
    presets = {
        "one": "<region> sample=sample.wav key=60 loop_mode=one_shot amp_veltrack=0\n",
        "loop": "<region> sample=sample.wav key=60 loop_mode=loop_continuous loop_start=0 loop_end=800 "
                "ampeg_release=0.1 amp_veltrack=0\n",
        "processed": "<region> sample=sample.wav key=60 loop_mode=loop_continuous loop_start=0 loop_end=800 "
                     "ampeg_release=0.1 amp_veltrack=0 fil_type=lpf_2p cutoff=1200 lfo1_freq=3 lfo1_pitch=120\n",
        "hot": "<region> sample=sample.wav key=60 loop_mode=one_shot amp_veltrack=0 pan_oncc10=0 volume=33\n",
    }
    midis = {
        "source": "00 90 3c 64 60 80 3c 00 a5 40 ff 2f 00",
        "regular": "00 90 3c 64 60 80 3c 00 00 ff 2f 00",
        "held": "00 b0 40 7f 00 90 3c 64 60 80 3c 00 00 b0 78 00 a5 40 ff 2f 00",
        "later": "00 b0 40 7f 00 90 3c 64 60 80 3c 00 82 68 b0 40 00 00 ff 2f 00",
        "sostenuto": "00 90 3c 64 30 b0 42 7f 30 80 3c 00 82 68 b0 42 00 00 ff 2f 00",
    }
    host = Host()
    for name, text in presets.items():
        sfz = tmp_path / f"{name}.sfz"
        sfz.write_text(text, encoding="ascii")
        for midi_name, hexdata in midis.items():
            midi = tmp_path / f"{midi_name}.mid"
            _midi(midi, bytes.fromhex(hexdata))
            outcome = []
            for planner in (host, session):
                try:
                    outcome.append(planner.plan(sfz, midi, **options).to_blob())
                except RuntimeError as error:
                    outcome.append(str(error).split(": ")[-1])
            assert outcome[0] == outcome[1], (name, midi_name, options)
    host.close()


def test_segment_fixture_plans_match(tmp_path):
    """The reference's tests/check_segments.py voice: loop, release, resonant
    cutoff and pitch on CC1, bends and pedal across a long note."""
    from oracle import reference
    session = reference.RefSession() if reference.available() or reference.build() else pytest.skip("no oracle/_ref")
    rate = 44100
    with wave.open(str(tmp_path / "sample.wav"), "wb") as stream:
        stream.setparams((1, 2, rate, 0, "NONE", "not compressed"))
        stream.writeframes(b"".join(struct.pack("<h", round(3000 * np.sin(i * .04))) for i in range(rate)))
    sfz = tmp_path / "voice.sfz"
    sfz.write_text("<region> sample=sample.wav key=60 loop_mode=loop_continuous loop_start=0 loop_end=44099 "
                   "amp_veltrack=0 ampeg_release=1.7 cutoff=1800 resonance=3 "
                   "cutoff_oncc1=3000 pitch_oncc1=37\n", encoding="ascii")
    _midi(tmp_path / "long.mid", bytes.fromhex(
        "00 b0 40 7f 00 90 3c 64 87 40 b0 01 40 87 40 e0 00 50 87 40 80 3c 00 87 40 b0 40 00 00 ff 2f 00"))
    _midi(tmp_path / "short.mid", bytes.fromhex("00 90 3c 64 60 80 3c 00 00 ff 2f 00"))
    host = Host()
    for tail in ("natural", "orig"):
        for name in ("short", "long"):
            mine = host.plan(sfz, tmp_path / f"{name}.mid", tail=tail)
            theirs = session.plan(sfz, tmp_path / f"{name}.mid", tail=tail)
            assert mine.to_blob() == theirs.to_blob(), (tail, name)
    assert np.array_equal(host.bank(), session.bank())
