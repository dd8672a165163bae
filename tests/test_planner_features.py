"""The C++ host planner against the reference's own planner on the SFZ and MIDI
features beyond the benchmark presets.

Each case builds small instruments that exercise one family of opcodes — key
switches, round robins, velocity layers and curves, release triggers with
rt_decay, choke groups (off_by with each off_mode), note_polyphony with and
without self-masking, CC-triggered regions, key / velocity / CC crossfades,
#define / #include / <control> / <curve>, random offsets, pitch and amplitude
randomisation, filters with key / velocity tracking, EQ bands, LFOs (numbered and
the legacy pitch/amp/fil forms, with CC-driven frequency), filter and pitch
envelopes with velocity tracking, flex envelopes on pitch, CC modulation with
curves and smoothing, dynamic amplitude envelopes, sustain and sostenuto pedals,
pitch bend with smoothing, loops with crossfades and sustain loops — and a
performance that touches them, then compares the two planners' plan images
byte for byte (with the decoded bank) in the natural and orig tail policies.
"""
import struct

import numpy as np
import pytest

from claysampler_b200 import workload
from claysampler_b200.host import Host


@pytest.fixture
def session():
    """A fresh reference session per case: sample offsets in a plan follow the
    session's bank, which the case's host starts empty as well."""
    from oracle import reference
    if not (reference.available() or reference.build()):
        pytest.skip("oracle/_ref (the reference built for the host) is not available")
    s = reference.RefSession()
    yield s
    s.close()


def tone(seconds, f0, channels=1, seed=0):
    rng = np.random.default_rng(seed)
    t = np.arange(int(seconds * 44100)) / 44100
    wave = 0.4 * np.sin(2 * np.pi * f0 * t) * np.exp(-t / 1.2) + 0.01 * rng.standard_normal(t.size)
    return np.stack([wave, np.roll(wave, 7)], axis=1) if channels == 2 else wave


def write_samples(root):
    samples = root / "zoo_samples"
    samples.mkdir(parents=True, exist_ok=True)
    for i, (name, channels, bits) in enumerate([("a", 1, 16), ("b", 2, 24), ("c", 1, 24), ("d", 2, 16),
                                                 ("e", 1, 16), ("f", 2, 16)]):
        workload.write_wav(samples / f"{name}.wav", tone(1.5 + 0.25 * i, 110 * (i + 1), channels, i), bits=bits)


ARTICULATIONS = """\
<control> default_path=zoo_samples/ set_cc1=20 set_hdcc74=0.5
#define $VOL -3
<global> ampeg_release=0.2 volume=$VOL amp_veltrack=80
<master> pitch_keytrack=100
<group> sw_lokey=24 sw_hikey=26 sw_last=24 sw_default=24
<region> sample=a.wav lokey=36 hikey=59 pitch_keycenter=48 seq_length=2 seq_position=1 ampeg_attack=0.01 ampeg_decay=0.3 ampeg_sustain=50
<region> sample=b.wav lokey=36 hikey=59 pitch_keycenter=48 seq_length=2 seq_position=2 tune=-10 pan=-30
<group> sw_last=25 loop_mode=loop_continuous loop_start=1000 loop_end=30000 loop_crossfade=0.01
<region> sample=c.wav lokey=36 hikey=59 pitch_keycenter=50 lovel=1 hivel=80
<region> sample=d.wav lokey=36 hikey=59 pitch_keycenter=50 lovel=81 hivel=127 amp_velcurve_100=0.8 amp_velcurve_64=0.3
<group> sw_last=26
<region> sample=e.wav lokey=36 hikey=59 pitch_keycenter=52 offset=500 offset_random=200 pitch_random=20 amp_random=2
<group> trigger=release rt_decay=6
<region> sample=f.wav lokey=36 hikey=59 pitch_keycenter=48 volume=-12
<group> group=1 off_by=2 off_mode=normal
<region> sample=a.wav lokey=60 hikey=71 note_polyphony=2
<group> group=2 off_by=1 off_mode=time off_time=0.05
<region> sample=b.wav lokey=72 hikey=83 note_polyphony=1 note_selfmask=off
<group> group=3
<region> sample=c.wav key=-1 on_locc20=64 on_hicc20=127 pitch_keycenter=60
<region> sample=d.wav lokey=85 hikey=95 xfin_lokey=85 xfin_hikey=90 xfout_lokey=90 xfout_hikey=95 xf_keycurve=gain
<region> sample=e.wav lokey=96 hikey=108 xfin_lovel=1 xfin_hivel=60 xfin_locc1=0 xfin_hicc1=100 loop_mode=loop_sustain loop_start=2000 loop_end=20000
<region> sample=f.wav lokey=96 hikey=108 lorand=0 hirand=0.5 trigger=first
<region> sample=a.wav lokey=96 hikey=108 lorand=0.5 hirand=1 trigger=legato delay=0.02 ampeg_delay=0.01 ampeg_hold=0.05 ampeg_start=20
"""

MODULATION = """\
<control> default_path=zoo_samples/
#include "zoo_common.sfzh"
<global> fil_type=lpf_2p cutoff=1200 resonance=3 fil_keytrack=50 fil_veltrack=1200 fil_random=100
<region> sample=a.wav lokey=36 hikey=60 fileg_attack=0.02 fileg_decay=0.4 fileg_sustain=40 fileg_release=0.3 fileg_depth=2400 fileg_vel2depth=-600 fileg_vel2attack=0.01 lfo1_freq=5 lfo1_cutoff=600 lfo1_freq_oncc1=3 lfo2_freq=2 lfo2_wave=1 lfo2_pitch=30 lfo2_delay=0.1 lfo2_fade=0.2 cutoff_oncc74=1200 cutoff_curvecc74=4 volume_oncc11=-6 pan_oncc10=50 pan_smoothcc10=20 amplitude_oncc7=100 amplitude_curvecc7=7
<region> sample=b.wav lokey=61 hikey=90 fil_type=hpf_2p cutoff=300 eq1_freq=800 eq1_gain=6 eq1_bw=1.5 eq2_gain=-4 pitcheg_attack=0.05 pitcheg_decay=0.2 pitcheg_sustain=0 pitcheg_depth=100 pitchlfo_freq=6 pitchlfo_depth=15 amplfo_freq=4 amplfo_depth=2 fillfo_freq=3 fillfo_depth=500 width=60 position=20 lfo3_freq=1 lfo3_wave=3 lfo3_width=30 resonance_oncc1=6
<region> sample=c.wav lokey=91 hikey=108 eg1_time1=0.05 eg1_level1=1 eg1_time2=0.2 eg1_level2=0 eg1_pitch=200 eg1_sustain=2 eg1_time1_oncc1=0.1 bend_up=200 bend_down=-1200 ampeg_vel2attack=0.05 ampeg_dynamic=on ampeg_release_oncc1=2 fil2_type=bpf_2p cutoff2=2000 fil_type=lpf_1p
<region> sample=d.wav lokey=20 hikey=35 bend_smooth=30 bend_up=700 pitch_oncc1=50 tune_smoothcc1=10 lfo4_freq=0.5 lfo4_wave=6 lfo4_volume=3 lfo4_position=20 lfo4_phase=0.25 offset_oncc1=100
<curve> curve_index=7 v000=0 v064=0.3 v127=1
"""

COMMON = "<master> ampeg_attack=0.005 ampeg_release=0.25 ampeg_vel2release=0.1\n"


def message(delta, *data):
    return workload._varlen(delta) + bytes(data)


def performance(path, pedal_cc66):
    """A single-channel performance: key switches, repeated notes, chords, CC
    sweeps, pedals, pitch bends, a CC-triggered region and a controller reset."""
    ev = []
    t = 0

    def at(dt, *data):
        nonlocal t
        ev.append(message(dt, *data))
        t += dt
    at(0, 0xB0, 1, 30)
    at(0, 0xB0, 74, 40)
    for sw, notes in ((24, (40, 48, 52)), (25, (44, 50, 57)), (26, (38, 55))):
        at(10, 0x90, sw, 100)
        at(30, 0x80, sw, 0)
        for k, key in enumerate(notes):
            at(40, 0x90, key, 40 + 30 * k)
            at(20, 0xB0, 1, 30 + 20 * k)
        at(120, 0xE0, 0x00, 0x50)
        at(60, 0xE0, 0x00, 0x40)
        for key in notes:
            at(30, 0x80, key, 0)
    for rep in range(4):                       # polyphony and choke groups
        at(40, 0x90, 62, 60 + 10 * rep)
        at(25, 0x90, 75, 90 - 10 * rep)
        at(25, 0x80, 62, 0)
    at(30, 0x80, 75, 0)
    at(10, 0xB0, 64, 127)                      # sustain pedal over a chord
    for key in (64, 88, 100):
        at(15, 0x90, key, 100)
    at(60, 0xB0, 11, 80)
    at(10, 0xB0, 10, 20)
    for key in (64, 88, 100):
        at(20, 0x80, key, 0)
    at(40, 0xB0, 64, 0)
    if pedal_cc66:
        at(10, 0x90, 30, 90)
        at(10, 0xB0, 66, 127)
        at(30, 0x80, 30, 0)
        at(10, 0x90, 33, 80)
        at(30, 0x80, 33, 0)
        at(40, 0xB0, 66, 0)
    at(20, 0xB0, 20, 100)                      # CC-triggered region
    at(20, 0xB0, 20, 10)
    at(10, 0x90, 98, 50)                       # first / legato / sustain loop
    at(20, 0x90, 100, 70)
    at(40, 0x80, 100, 0)
    at(20, 0x80, 98, 0)
    at(10, 0x90, 93, 110)
    at(30, 0xB0, 1, 100)                       # dynamic release change mid-release
    at(10, 0x80, 93, 0)
    at(5, 0xB0, 1, 10)
    at(20, 0xB0, 121, 0)                       # reset all controllers
    at(10, 0x90, 45, 64)
    at(60, 0x80, 45, 0)
    at(200, 0xFF, 0x2F, 0x00)
    data = b"\x00\xff\x51\x03" + (500000).to_bytes(3, "big") + b"".join(ev)
    path.write_bytes(b"MThd" + struct.pack(">IHHH", 6, 0, 1, 96) + b"MTrk" + struct.pack(">I", len(data)) + data)


@pytest.mark.parametrize("preset", ["articulations", "modulation"])
@pytest.mark.parametrize("tail", ["natural", "orig"])
def test_planner_feature_zoo(tmp_path, session, preset, tail):
    write_samples(tmp_path)
    (tmp_path / "zoo_common.sfzh").write_text(COMMON)
    sfz = tmp_path / f"{preset}.sfz"
    sfz.write_text(ARTICULATIONS if preset == "articulations" else MODULATION)
    midi = tmp_path / "zoo.mid"
    performance(midi, pedal_cc66=tail == "natural")
    host = Host()
    mine = host.plan(sfz, midi, tail=tail)
    theirs = session.plan(sfz, midi, tail=tail)
    assert len(mine.spans) > 10
    assert mine.to_blob() == theirs.to_blob()
    bank = host.bank()
    ref_bank = session.bank()
    assert np.array_equal(bank, ref_bank[:bank.size]) and bank.size > 0
    host.close()
