"""Generates tests/golden/*.npz from the reference's own code built for the host.

Inputs are the fixtures of the reference's tests/check_tail.py (its WAV, SFZ and
hex-encoded MIDI, restated here as data) plus one short excerpt of the plain
12-region preset.  For each case the reference planner (oracle/_ref) makes the
plan, the reference's render.cu (oracle/_ref) makes the mix, and the oracle's
restatement of tail.cu finishes it.  Stored per case: the plan image, the decoded
bank, the packed PCM16 and the per-job results.

Run from the repository root:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import struct
import sys
import tempfile
import wave
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
OUT = Path(__file__).resolve().parent
RATE = 44100

MIDI = {
    "source": "00 90 3c 64 60 80 3c 00 a5 40 ff 2f 00",
    "regular": "00 90 3c 64 60 80 3c 00 00 ff 2f 00",
    "held": "00 b0 40 7f 00 90 3c 64 60 80 3c 00 00 b0 78 00 a5 40 ff 2f 00",
    "later": "00 b0 40 7f 00 90 3c 64 60 80 3c 00 82 68 b0 40 00 00 ff 2f 00",
    "sostenuto": "00 90 3c 64 30 b0 42 7f 30 80 3c 00 82 68 b0 42 00 00 ff 2f 00",
    "gap": "00 90 3c 64 8b 20 80 3c 00 00 ff 2f 00",
}
ONE_SHOT = "<region> sample=sample.wav key=60 loop_mode=one_shot amp_veltrack=0"
LOOP = ("<region> sample=sample.wav key=60 loop_mode=loop_continuous loop_start=0 loop_end=800 "
        "ampeg_release=0.1 amp_veltrack=0")
PRESETS = {
    "one": ONE_SHOT + "\n",
    "loop": LOOP + "\n",
    "processed": LOOP + " fil_type=lpf_2p cutoff=1200 lfo1_freq=3 lfo1_pitch=120\n",
    "hot": ONE_SHOT + " pan_oncc10=0 volume=33\n",
    "tooHot": ONE_SHOT + " pan_oncc10=0 volume=42\n",
    "short": ONE_SHOT.replace("sample.wav", "short.wav") + "\n",
}
# case -> (preset, midi, tail, options)
CASES = {
    "natural": ("one", "source", "natural", {}),
    "orig": ("one", "source", "orig", {}),
    "custom": ("one", "source", "custom", {"tail_max": 1.0, "tail_fade_ms": 100}),
    "custom_dry": ("one", "source", "custom", {"tail_max": 1.0, "tail_fade_ms": 0}),
    "custom_uncut": ("one", "source", "custom", {"tail_max": 4.0}),
    "limited": ("one", "source", "natural", {"max_audio": 0.5}),
    "pedal_regular": ("loop", "regular", "natural", {}),
    "pedal_held": ("loop", "held", "natural", {}),
    "pedal_later": ("loop", "later", "natural", {}),
    "pedal_sostenuto": ("loop", "sostenuto", "natural", {}),
    "filtered_regular": ("processed", "regular", "natural", {}),
    "filtered_later": ("processed", "later", "natural", {}),
    "repaired": ("hot", "source", "natural", {}),
    "too_hot": ("tooHot", "source", "natural", {}),
    "padded": ("short", "gap", "natural", {}),
}


def write_inputs(root: Path) -> None:
    with wave.open(str(root / "sample.wav"), "wb") as stream:
        stream.setparams((1, 2, RATE, 0, "NONE", "not compressed"))
        stream.writeframes(struct.pack("<h", 1600) * (RATE * 2 // 5) + struct.pack("<h", 12) * (RATE * 3))
    with wave.open(str(root / "short.wav"), "wb") as stream:
        stream.setparams((1, 2, RATE, 0, "NONE", "not compressed"))
        stream.writeframes(struct.pack("<h", 1600) * (RATE * 2 // 5))
    for name, text in PRESETS.items():
        (root / f"{name}.sfz").write_text(text, encoding="ascii")
    for name, hexdata in MIDI.items():
        data = bytes.fromhex(hexdata)
        (root / f"{name}.mid").write_bytes(b"MThd" + struct.pack(">IHHH", 6, 0, 1, 480) + b"MTrk"
                                           + struct.pack(">I", len(data)) + data)


def main() -> None:
    from claysampler_b200 import workload
    from oracle import oracle, reference
    if not (reference.available() or reference.build()):
        raise SystemExit("oracle/_ref is not built (needs the reference sources)")
    with tempfile.TemporaryDirectory() as tmp:
        root = Path(tmp)
        write_inputs(root)
        for case, (preset, midi, tail, options) in CASES.items():
            session = reference.RefSession()
            plan = session.plan(root / f"{preset}.sfz", root / f"{midi}.mid", tail=tail, **options)
            bank = session.bank()
            natural = tail == "natural"
            mix = reference.synthesize([plan], bank, natural)
            pcm, results = oracle.finish(mix, [plan], natural)
            np.savez_compressed(OUT / f"{case}.npz", plan=np.frombuffer(plan.to_blob(), np.uint8), bank=bank,
                                pcm=pcm, results=results.view(np.uint8), natural=natural, tail=tail)
            session.close()
        # An excerpt of the plain 12-region preset (resampled voices, 48-tap sinc).
        (root / "plain").mkdir()
        sfz = workload.write_plain_small_preset(root / "plain", seed=11)
        notes = [(0.05, 0.4, 60, 100), (0.3, 0.6, 67, 80), (0.9, 0.3, 42, 110), (1.2, 0.8, 88, 60),
                 (1.5, 0.2, 25, 127), (2.0, 0.7, 103, 90)]
        workload._note_midi(notes, [], 3.0, root / "plain" / "excerpt.mid")
        session = reference.RefSession()
        plan = session.plan(sfz, root / "plain" / "excerpt.mid")
        bank = session.bank()
        mix = reference.synthesize([plan], bank, True)
        pcm, results = oracle.finish(mix, [plan], True)
        np.savez_compressed(OUT / "plain_excerpt.npz", plan=np.frombuffer(plan.to_blob(), np.uint8), bank=bank,
                            pcm=pcm, results=results.view(np.uint8), natural=True, tail="natural")
    print("wrote", sorted(p.name for p in OUT.glob("*.npz")))


if __name__ == "__main__":
    main()
