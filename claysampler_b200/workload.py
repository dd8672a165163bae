"""Seeded synthetic SFZ instruments, WAV samples and Standard MIDI Files.

The reference measures on sample libraries and MIDI collections that are not
redistributable.  These generators build instruments and performances of the
same shapes from a seed so that every run sees identical inputs:

* ``plain_small``   - 12 mono 16-bit regions (2 s, 8-partial harmonic sums with
  exponential decay), ``pitch_keycenter`` every 8 semitones, ampeg 5 ms / 200 ms /
  60 % / 300 ms, no filter, no loops; one 30 s MIDI file with 64 notes.
* ``plain_batch``   - 88 keys x 4 velocity layers of stereo 24-bit samples (4 s,
  harmonic plus noise), half of them ``loop_continuous``; ``lpf_2p`` with a random
  cutoff in 200-8000 Hz, a +-2400 cent filter envelope and a 5 Hz LFO on the cutoff;
  MIDI lengths log-uniform 10-180 s, Poisson 4 notes/s, at most 64 held notes and a
  CC64 sustain pedal toggled every ~8 s.
* ``uneven_batch``  - jobs of the ``plain_small`` kind with Pareto(1.5) lengths from
  2 s to 600 s over several presets.

Everything here is plain file generation (numpy); it never touches the GPU.
"""
from __future__ import annotations

import math
import struct
from dataclasses import dataclass
from pathlib import Path

import numpy as np

RATE = 44100
PPQ = 480
TEMPO_US = 500000          # 120 bpm -> one tick is 1/960 s
TICKS_PER_SECOND = 1_000_000 * PPQ / TEMPO_US


# --------------------------------------------------------------------------- files

def write_wav(path: Path, data: np.ndarray, rate: int = RATE, bits: int = 16) -> None:
    """Write ``data`` (frames x channels, floats in [-1, 1)) as PCM16 or PCM24 WAV."""
    if data.ndim == 1:
        data = data[:, None]
    frames, channels = data.shape
    scale = float(1 << (bits - 1))
    ints = np.clip(np.round(data * scale), -scale, scale - 1).astype(np.int32)
    if bits == 16:
        payload = ints.astype("<i2").tobytes()
    elif bits == 24:
        raw = ints.astype("<i4").reshape(-1).view(np.uint8).reshape(-1, 4)[:, :3]
        payload = np.ascontiguousarray(raw).tobytes()
    else:
        raise ValueError("bits must be 16 or 24")
    block = channels * bits // 8
    header = b"RIFF" + struct.pack("<I", 36 + len(payload)) + b"WAVE"
    header += b"fmt " + struct.pack("<IHHIIHH", 16, 1, channels, rate, rate * block, block, bits)
    header += b"data" + struct.pack("<I", len(payload))
    path.write_bytes(header + payload)


def _varlen(value: int) -> bytes:
    out = [value & 0x7F]
    value >>= 7
    while value:
        out.append(0x80 | (value & 0x7F))
        value >>= 7
    return bytes(reversed(out))


def write_midi(path: Path, events: list[tuple[int, int, bytes]], end_tick: int) -> None:
    """Write a format-0 SMF at 480 PPQ / 120 bpm.

    ``events`` holds ``(tick, order, message)``; ``order`` breaks ties so that
    note-offs precede note-ons at the same tick.
    """
    data = bytearray()
    data += b"\x00\xff\x51\x03" + TEMPO_US.to_bytes(3, "big")
    last = 0
    for tick, _, message in sorted(events, key=lambda e: (e[0], e[1])):
        data += _varlen(tick - last) + message
        last = tick
    data += _varlen(max(0, end_tick - last)) + b"\xff\x2f\x00"
    path.write_bytes(b"MThd" + struct.pack(">IHHH", 6, 0, 1, PPQ)
                     + b"MTrk" + struct.pack(">I", len(data)) + bytes(data))


def seconds_to_tick(seconds: float) -> int:
    return int(round(seconds * TICKS_PER_SECOND))


def key_frequency(key: float) -> float:
    return 440.0 * 2.0 ** ((key - 69) / 12.0)


# --------------------------------------------------------------------------- jobs

@dataclass
class Job:
    group: str
    sfz: Path
    midi: Path
    output: Path


def write_manifest(path: Path, jobs: list[Job]) -> None:
    """The reference's --jobs TSV: group, SFZ, MIDI, output (relative to the manifest)."""
    root = path.parent
    lines = [f"{j.group}\t{j.sfz.relative_to(root)}\t{j.midi.relative_to(root)}\t{j.output.relative_to(root)}\n"
             for j in jobs]
    path.write_text("".join(lines), encoding="utf-8")


def _note_midi(notes: list[tuple[float, float, int, int]], pedals: list[tuple[float, int]],
               end_seconds: float, path: Path) -> None:
    events = []
    for onset, duration, key, velocity in notes:
        events.append((seconds_to_tick(onset), 2, bytes([0x90, key, velocity])))
        events.append((seconds_to_tick(onset + duration), 0, bytes([0x80, key, 0])))
    for time, value in pedals:
        events.append((seconds_to_tick(time), 1, bytes([0xB0, 64, value])))
    end_tick = max(seconds_to_tick(end_seconds), max(e[0] for e in events))
    write_midi(path, events, end_tick)


def _performance(rng: np.random.Generator, seconds: float, rate_per_second: float | None,
                 count: int | None, low_vel: int, high_vel: int, mean_duration: float,
                 max_held: int = 64) -> list[tuple[float, float, int, int]]:
    """Random notes without same-key overlap and with at most ``max_held`` held keys."""
    if count is None:
        count = max(1, int(rng.poisson(rate_per_second * seconds)))
    onsets = np.sort(rng.uniform(0.0, seconds, count))
    held: list[tuple[float, int]] = []
    notes = []
    for onset in onsets:
        held = [(end, key) for end, key in held if end > onset]
        if len(held) >= max_held:
            continue
        busy = {key for _, key in held}
        key = int(rng.integers(21, 109))
        while key in busy:
            key = int(rng.integers(21, 109))
        duration = max(0.03, float(rng.exponential(mean_duration)))
        duration = min(duration, seconds - onset + 1.0)
        velocity = int(rng.integers(low_vel, high_vel + 1))
        notes.append((float(onset), duration, key, velocity))
        held.append((onset + duration + 0.01, key))
    return notes


# --------------------------------------------------------------------------- presets

def _harmonic(rng: np.random.Generator, f0: float, seconds: float, partials: int = 8,
              tau: float | None = None) -> np.ndarray:
    t = np.arange(int(seconds * RATE)) / RATE
    tau = float(rng.uniform(0.5, 1.5)) if tau is None else tau
    out = np.zeros_like(t)
    for k in range(1, partials + 1):
        if k * f0 >= RATE / 2:
            break
        amp = float(rng.uniform(0.5, 1.0)) / k
        out += amp * np.sin(2 * np.pi * k * f0 * t + float(rng.uniform(0, 2 * np.pi)))
    out *= np.exp(-t / tau)
    return 0.5 * out / max(1e-9, float(np.max(np.abs(out))))


def write_plain_small_preset(root: Path, seed: int, name: str = "plain") -> Path:
    """12 mono PCM16 regions; returns the SFZ path."""
    rng = np.random.default_rng(seed)
    samples = root / f"{name}_samples"
    samples.mkdir(parents=True, exist_ok=True)
    lines = ["<group> ampeg_attack=0.005 ampeg_decay=0.2 ampeg_sustain=60 ampeg_release=0.3 "
             "loop_mode=no_loop\n"]
    for i in range(12):
        center = 21 + 8 * i
        wav = samples / f"r{i:02d}.wav"
        write_wav(wav, _harmonic(rng, key_frequency(center), 2.0), bits=16)
        lo, hi = max(21, center - 4), min(108, center + 3)
        lines.append(f"<region> sample={wav.relative_to(root).as_posix()} lokey={lo} hikey={hi} "
                     f"pitch_keycenter={center}\n")
    sfz = root / f"{name}.sfz"
    sfz.write_text("".join(lines), encoding="ascii")
    return sfz


def write_plain_small(root: Path, seed: int = 1) -> list[Job]:
    """One 30 s MIDI file of 64 notes through the 12-region mono preset."""
    root.mkdir(parents=True, exist_ok=True)
    sfz = write_plain_small_preset(root, seed)
    rng = np.random.default_rng(seed + 1000)
    notes = _performance(rng, 30.0, None, 64, 40, 120, 0.5)
    midi = root / "plain_small.mid"
    _note_midi(notes, [], 30.0, midi)
    return [Job("-", sfz, midi, root / "out" / "plain_small.wav")]


def write_plain_batch_preset(root: Path, seed: int, keys: range = range(21, 109),
                             layers: int = 4, seconds: float = 4.0, name: str = "batch") -> Path:
    """Stereo PCM24 multisample with loops, lpf_2p, filter envelope and LFO."""
    rng = np.random.default_rng(seed)
    samples = root / f"{name}_samples"
    samples.mkdir(parents=True, exist_ok=True)
    frames = int(seconds * RATE)
    t = np.arange(frames) / RATE
    edges = np.linspace(0, 128, layers + 1).astype(int)
    lines = ["<global> ampeg_attack=0.005 ampeg_decay=1.5 ampeg_sustain=50 ampeg_release=0.5 "
             "fil_type=lpf_2p fileg_attack=0.01 fileg_decay=0.6 fileg_sustain=30 fileg_release=0.4 "
             "lfo1_freq=5\n"]
    for key in keys:
        f0 = key_frequency(key)
        partials = []
        for k in range(1, 9):
            if k * f0 >= RATE / 2:
                break
            phase_l, phase_r = rng.uniform(0, 2 * np.pi, 2)
            partials.append((np.sin(2 * np.pi * k * f0 * t + phase_l),
                             np.sin(2 * np.pi * k * f0 * t + phase_r), k))
        tau = float(rng.uniform(1.5, 4.0))
        decay = np.exp(-t / tau)
        for layer in range(layers):
            bright = 0.4 + 0.6 * layer / max(1, layers - 1)
            left = np.zeros(frames)
            right = np.zeros(frames)
            for wave_l, wave_r, k in partials:
                amp = bright ** (k - 1) * float(rng.uniform(0.6, 1.0)) / k
                left += amp * wave_l
                right += amp * wave_r
            noise = rng.standard_normal((frames, 2)) * 0.02 * np.exp(-t / 0.05)[:, None]
            data = np.stack([left, right], axis=1) * decay[:, None] + noise
            data *= (0.3 + 0.5 * layer / max(1, layers - 1)) / max(1e-9, float(np.max(np.abs(data))))
            wav = samples / f"k{key:03d}_v{layer}.wav"
            write_wav(wav, data, bits=24)
            lo_vel, hi_vel = max(1, int(edges[layer])), int(edges[layer + 1]) - 1
            opcodes = [f"sample={wav.relative_to(root).as_posix()}", f"key={key}",
                       f"lovel={lo_vel}", f"hivel={hi_vel}",
                       f"cutoff={rng.uniform(200, 8000):.1f}",
                       f"fileg_depth={int(rng.choice([-2400, 2400]))}",
                       f"lfo1_cutoff={int(rng.integers(300, 1201))}"]
            if (key + layer) % 2 == 0:
                first = int(rng.integers(RATE // 2, RATE))
                opcodes += ["loop_mode=loop_continuous", f"loop_start={first}",
                            f"loop_end={frames - 1 - int(rng.integers(0, RATE // 2))}"]
            else:
                opcodes.append("loop_mode=no_loop")
            lines.append("<region> " + " ".join(opcodes) + "\n")
    sfz = root / f"{name}.sfz"
    sfz.write_text("".join(lines), encoding="ascii")
    return sfz


def write_plain_batch(root: Path, seed: int = 2, jobs: int = 64, min_seconds: float = 10.0,
                      max_seconds: float = 180.0, keys: range = range(21, 109),
                      layers: int = 4) -> list[Job]:
    """The 64-job batch: lengths log-uniform, Poisson 4 notes/s, CC64 every ~8 s."""
    root.mkdir(parents=True, exist_ok=True)
    sfz = write_plain_batch_preset(root, seed, keys, layers)
    rng = np.random.default_rng(seed + 1000)
    out = []
    for j in range(jobs):
        seconds = float(math.exp(rng.uniform(math.log(min_seconds), math.log(max_seconds))))
        notes = _performance(rng, seconds, 4.0, None, 1, 127, 0.5)
        notes = [n for n in notes if keys.start <= n[2] < keys.stop] or \
            [(0.1, 0.5, keys.start, 100)]
        pedals = []
        time, down = float(rng.uniform(2, 8)), True
        while time < seconds:
            pedals.append((time, 127 if down else 0))
            down = not down
            time += float(rng.uniform(6, 10))
        midi = root / f"batch_{j:03d}.mid"
        _note_midi(notes, pedals, seconds, midi)
        out.append(Job("-", sfz, midi, root / "out" / f"batch_{j:03d}.wav"))
    return out


def pareto_seconds(rng: np.random.Generator, count: int, alpha: float = 1.5,
                   low: float = 2.0, high: float = 600.0) -> np.ndarray:
    """Truncated Pareto lengths by inverse-CDF sampling."""
    u = rng.uniform(0, 1, count)
    ratio = (low / high) ** alpha
    return low / (1 - u * (1 - ratio)) ** (1 / alpha)


def write_uneven_batch(root: Path, seed: int = 3, jobs: int = 1024, presets: int = 4,
                       high: float = 600.0) -> list[Job]:
    """Jobs of the small kind over several presets with Pareto(1.5) lengths."""
    root.mkdir(parents=True, exist_ok=True)
    sfzs = [write_plain_small_preset(root, seed + p, name=f"preset{p}") for p in range(presets)]
    rng = np.random.default_rng(seed + 1000)
    lengths = pareto_seconds(rng, jobs, high=high)
    out = []
    for j, seconds in enumerate(lengths):
        count = max(1, int(round(64 * seconds / 30.0)))
        notes = _performance(rng, float(seconds), None, count, 40, 120, 0.5)
        midi = root / f"uneven_{j:04d}.mid"
        _note_midi(notes, [], float(seconds), midi)
        out.append(Job("-", sfzs[j % presets], midi, root / "out" / f"uneven_{j:04d}.wav"))
    return out


def write_serving_jobs(root: Path, seed: int = 5, jobs: int = 200, presets: int = 8, low: float = 5.0,
                       high: float = 300.0, rate: float = 50.0, large: bool = False) -> tuple[list[Job], np.ndarray]:
    """Render requests of the serving kind: jobs over several presets of the small
    kind (`large`: of the HBM-bank kind, about 1.5 GB of float samples each), MIDI
    lengths log-uniform in [low, high] seconds at the small kind's note density,
    arriving by a Poisson process of `rate` jobs per second.  Returns the jobs and
    their arrival times in seconds."""
    root.mkdir(parents=True, exist_ok=True)
    if large:
        sfzs = [write_hbm_preset(root, seed + p, name=f"serve_large{p}") for p in range(presets)]
    else:
        sfzs = [write_plain_small_preset(root, seed + p, name=f"serve{p}") for p in range(presets)]
    rng = np.random.default_rng(seed + 2000)
    lengths = np.exp(rng.uniform(np.log(low), np.log(high), jobs))
    arrivals = np.cumsum(rng.exponential(1.0 / rate, jobs))
    out = []
    for j, seconds in enumerate(lengths):
        count = max(1, int(round(64 * seconds / 30.0)))
        notes = _performance(rng, float(seconds), None, count, 40, 120, 0.5)
        midi = root / f"serve_{j:04d}.mid"
        _note_midi(notes, [], float(seconds), midi)
        out.append(Job("-", sfzs[j % presets], midi, root / "out" / f"serve_{j:04d}.wav"))
    return out, arrivals


def write_hbm_preset(root: Path, seed: int, name: str, centers: range = range(23, 109, 4), layers: int = 8,
                     seconds: float = 48.0) -> Path:
    """A large mono 16-bit multisample: a region per keycenter (every 4 semitones,
    keys -2..+1 around it) and velocity layer, each `seconds` long.  Each sample
    tiles one period of an 8-partial wavetable (brighter for louder layers) under an
    exponential decay, which keeps generating gigabytes of samples fast."""
    rng = np.random.default_rng(seed)
    samples = root / f"{name}_samples"
    samples.mkdir(parents=True, exist_ok=True)
    frames = int(seconds * RATE)
    edges = np.linspace(0, 128, layers + 1).astype(int)
    lines = ["<group> ampeg_attack=0.005 ampeg_decay=0.2 ampeg_sustain=60 ampeg_release=0.3 loop_mode=no_loop\n"]
    t = np.arange(frames) / RATE
    for center in centers:
        period = max(2, int(round(RATE / key_frequency(center))))
        phase = np.arange(period) / period
        decay = np.exp(-t / float(rng.uniform(4.0, 12.0)))
        for layer in range(layers):
            bright = 0.3 + 0.7 * layer / max(1, layers - 1)
            table = np.zeros(period)
            for k in range(1, 9):
                table += (bright ** (k - 1)) * float(rng.uniform(0.6, 1.0)) / k * \
                    np.sin(2 * np.pi * k * phase + float(rng.uniform(0, 2 * np.pi)))
            table *= 0.45 / max(1e-9, float(np.max(np.abs(table))))
            data = np.resize(table, frames) * decay
            wav = samples / f"c{center:03d}_v{layer}.wav"
            write_wav(wav, data, bits=16)
            lo, hi = max(21, center - 2), min(108, center + 1)
            lines.append(f"<region> sample={wav.relative_to(root).as_posix()} lokey={lo} hikey={hi} "
                         f"pitch_keycenter={center} lovel={max(1, int(edges[layer]))} hivel={int(edges[layer + 1]) - 1}\n")
    sfz = root / f"{name}.sfz"
    sfz.write_text("".join(lines), encoding="ascii")
    return sfz


def write_uneven_hbm_batch(root: Path, seed: int = 3, jobs: int = 1024, presets: int = 4,
                           high: float = 600.0) -> list[Job]:
    """The uneven batch over four large presets (about 6 GB of float samples in
    all, far above the L2): Pareto(1.5) lengths from 2 to 600 s, notes as in the
    small kind with velocities spanning the layers."""
    root.mkdir(parents=True, exist_ok=True)
    sfzs = [write_hbm_preset(root, seed + p, name=f"large{p}") for p in range(presets)]
    rng = np.random.default_rng(seed + 1000)
    lengths = pareto_seconds(rng, jobs, high=high)
    out = []
    for j, seconds in enumerate(lengths):
        count = max(1, int(round(64 * seconds / 30.0)))
        notes = _performance(rng, float(seconds), None, count, 1, 127, 0.5)
        midi = root / f"uneven_hbm_{j:04d}.mid"
        _note_midi(notes, [], float(seconds), midi)
        out.append(Job("-", sfzs[j % presets], midi, root / "out" / f"uneven_hbm_{j:04d}.wav"))
    return out
