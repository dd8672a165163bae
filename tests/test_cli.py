"""The `claysampler` command line: the reference CLI's flags, --jobs manifest, line
protocol and exit codes (src/main.cpp), checked with the reference's own CLI test
scenarios restated (tests/check_tail.py, check_group_audio.py, check_segments.py).

Argument, manifest, --check-sfz and fully-resumed runs never reach the GPU and run
on the CPU; everything that renders is gpu-marked.
"""
import itertools
import math
import struct
import subprocess
import wave
from pathlib import Path

import numpy as np
import pytest

from conftest import gpu_available

RATE = 44100
gpu = [pytest.mark.gpu, pytest.mark.skipif(not gpu_available(), reason="needs a CUDA GPU")]


@pytest.fixture(scope="module")
def clay():
    from claysampler_b200 import build
    build.build_library()
    build.build_host()
    assert build.CLI.exists()
    return build.CLI


def run(clay, *args, expected=None):
    result = subprocess.run([str(clay), *map(str, args)], capture_output=True, text=True, timeout=600)
    if expected is not None:
        assert result.returncode == expected, result.stdout + result.stderr
    return result


def midi(path, data):
    path.write_bytes(b"MThd" + struct.pack(">IHHH", 6, 0, 1, 480) + b"MTrk" + struct.pack(">I", len(data)) + data)


def write_wav(path, frames_bytes, channels=1):
    with wave.open(str(path), "wb") as stream:
        stream.setparams((channels, 2, RATE, 0, "NONE", "not compressed"))
        stream.writeframes(frames_bytes)


def read_wav(path):
    with wave.open(str(path), "rb") as stream:
        return stream.getnchannels(), stream.getnframes(), stream.readframes(stream.getnframes())


def pcm(path):
    return np.frombuffer(read_wav(path)[2], "<i2").astype(np.int64)


def transfer(result):
    line = next(line for line in result.stdout.splitlines() if line.startswith("TRANSFER\t"))
    return tuple(map(int, line.split("\t")[2:]))


@pytest.fixture(scope="module")
def tail_inputs(tmp_path_factory):
    """check_tail.py:27-36 — 0.4 s at 1600 then 3 s at 12; a 0.1 s note, 5 s to EOT."""
    root = tmp_path_factory.mktemp("tail")
    write_wav(root / "sample.wav", struct.pack("<h", 1600) * (RATE * 2 // 5) + struct.pack("<h", 12) * (RATE * 3))
    (root / "sample.sfz").write_text("<region> sample=sample.wav key=60 loop_mode=one_shot amp_veltrack=0\n",
                                     encoding="ascii")
    midi(root / "source.mid", bytes.fromhex("00 90 3c 64 60 80 3c 00 a5 40 ff 2f 00"))
    return root


# ---- CPU: options, manifests, presets, resume -----------------------------------------

def test_usage_and_option_errors(clay, tail_inputs, tmp_path):
    assert "Usage: claysampler" in run(clay, "--help", expected=0).stdout
    cases = [
        ((), "provide --sfz, --output, and at least one MIDI path"),
        (("--sfz", "a.sfz", "--output", "o", "--tail-policy", "long", "x.mid"), "expected --tail-policy"),
        (("--sfz", "a.sfz", "--output", "o", "--qa-min-peak", "3", "x.mid"), "quality thresholds require"),
        (("--sfz", "a.sfz", "--output", "o", "--group-volume", "mean", "x.mid"), "--group-volume mean requires --jobs"),
        (("--sfz", "a.sfz", "--output", "o", "--tail-policy", "custom", "x.mid"), "custom tail requires"),
        (("--sfz", "a.sfz", "--output", "o", "--max-audio-seconds", "1", "--tail-policy", "orig", "x.mid"),
         "--max-audio-seconds requires"),
        (("--sfz", "a.sfz", "--output", "o", "--samplerate", "7999", "x.mid"), "invalid numeric argument"),
        (("--sfz", "a.sfz", "--output", "o", "--frobnicate", "1", "x.mid"), "unknown option --frobnicate"),
        (("--jobs", "j.tsv", "--sfz", "a.sfz"), "--jobs supplies"),
    ]
    for args, message in cases:
        result = run(clay, *args, expected=1)
        assert result.stderr.startswith("ERROR\t") and message in result.stderr, (args, result.stderr)


def test_manifest_errors(clay, tmp_path):
    cases = [
        ("-\ta.sfz\tb.mid\n", "expected group, SFZ, MIDI and output on manifest line 1"),
        ("-\ta.sfz\t\tc.wav\n", "expected group, SFZ, MIDI and output on manifest line 1"),
        ("\n-\ta.sfz\tb.mid\tc.wav\textra\n", "invalid job manifest line 2"),
        ("-\ta.sfz\tb.mid\tc.flac\n", "expected a .wav output on manifest line 1"),
        ("-\ta.sfz\tb.mid\tc.wav\n-\ta.sfz\tb.mid\t./c.wav\n", "duplicate output path"),
        ("", "job manifest is empty"),
    ]
    for text, message in cases:
        manifest = tmp_path / "jobs.tsv"
        manifest.write_bytes(text.encode())
        result = run(clay, "--jobs", manifest, expected=1)
        assert message in result.stderr, (text, result.stderr)


def test_check_sfz(clay, tail_inputs, tmp_path):
    result = run(clay, "--check-sfz", tail_inputs / "sample.sfz", expected=0)
    assert result.stdout == "SFZ\tOK\t1\n"
    result = run(clay, "--check-sfz", tail_inputs / "sample.sfz", tmp_path / "missing.sfz", expected=2)
    lines = result.stdout.splitlines()
    assert lines[0] == "SFZ\tOK\t1" and lines[1].startswith("SFZ\tREJECT\t")


def test_resume_skips_complete_groups_without_a_device(clay, tail_inputs, tmp_path):
    """A fully written manifest resumes to SKIP lines only: no renderer, no DEVICE."""
    out = tmp_path / "out"
    out.mkdir()
    for name in ("a", "b"):
        write_wav(out / f"{name}.wav", b"\0\0" * 100)
    manifest = tmp_path / "jobs.tsv"
    manifest.write_text(f"g\t{tail_inputs / 'sample.sfz'}\t{tail_inputs / 'source.mid'}\tout/a.wav\n"
                        f"g\t{tail_inputs / 'sample.sfz'}\t{tail_inputs / 'source.mid'}\tout/b.wav\n")
    result = run(clay, "--jobs", manifest, "--group-volume", "mean", "--resume", expected=0)
    assert result.stdout.count("SKIP\t") == 2 and "DEVICE\t" not in result.stdout


# ---- GPU: rendering through the CLI ------------------------------------------------------

def test_tail_policies(clay, tail_inputs, tmp_path):
    """check_tail.py:38-120."""
    root, sfz, source = tail_inputs, tail_inputs / "sample.sfz", tail_inputs / "source.mid"

    def render(name, *flags, inputs=(source,), preset=sfz, expected=0):
        output = tmp_path / name
        return output, run(clay, "--sfz", preset, "--output", output, *flags, *inputs, expected=expected)

    natural, log = render("default")
    explicit, _ = render("natural", "--tail-policy", "natural")
    wave_path = natural / "source.wav"
    assert wave_path.read_bytes() == (explicit / "source.wav").read_bytes()
    channels, frames, samples = read_wav(wave_path)
    assert (channels, frames) == (1, round(.65 * RATE))
    values = np.frombuffer(samples, "<i2").astype(np.int64)
    assert values[frames - 5000] > 3 and values[-1] == 0
    audible = np.nonzero(np.abs(values) > 3)[0]
    ok = next(line.split("\t") for line in log.stdout.splitlines() if line.startswith("OK\t"))
    assert ok[1] == "source.wav"
    assert list(map(int, ok[2:])) == [frames, int(np.abs(values).max()), int(audible[0]), int(audible[-1])]
    assert log.stdout.startswith("DEVICE\t") and "\nINIT\t" in log.stdout and "\nPASS\t1\t" in log.stdout

    orig, _ = render("orig", "--tail-policy", "orig")
    assert read_wav(orig / "source.wav")[:2] == (2, round(5.1 * RATE))
    custom, _ = render("custom", "--tail-policy", "custom", "--tail-max-seconds", "1", "--tail-fade-ms", "100")
    dry, _ = render("custom-dry", "--tail-policy", "custom", "--tail-max-seconds", "1", "--tail-fade-ms", "0")
    channels, frames, samples = read_wav(custom / "source.wav")
    dry_samples = read_wav(dry / "source.wav")[2]
    assert (channels, frames) == (2, round(1.1 * RATE) + 1)
    assert samples[:-4410 * 4] == dry_samples[:-4410 * 4]
    assert samples[-4:] == b"\0\0\0\0" and dry_samples[-4:] != samples[-4:]
    uncut, _ = render("custom-uncut", "--tail-policy", "custom", "--tail-max-seconds", "4")
    channels, frames, samples = read_wav(uncut / "source.wav")
    assert (channels, frames) == (2, round(3.4 * RATE))
    assert samples == read_wav(orig / "source.wav")[2][:frames * 4]
    limited, result = render("limited", "--max-audio-seconds", "0.5", expected=2)
    assert "tail or audio duration limit" in result.stderr and not (limited / "source.wav").exists()

    loop = root / "loop.sfz"
    loop.write_text("<region> sample=sample.wav key=60 loop_mode=loop_continuous loop_start=0 "
                    "loop_end=800 ampeg_release=0.1 amp_veltrack=0\n", encoding="ascii")
    names = ("regular", "held", "later", "sostenuto")
    data = ("00 90 3c 64 60 80 3c 00 00 ff 2f 00",
            "00 b0 40 7f 00 90 3c 64 60 80 3c 00 00 b0 78 00 a5 40 ff 2f 00",
            "00 b0 40 7f 00 90 3c 64 60 80 3c 00 82 68 b0 40 00 00 ff 2f 00",
            "00 90 3c 64 30 b0 42 7f 30 80 3c 00 82 68 b0 42 00 00 ff 2f 00")
    for name, hexdata in zip(names, data):
        midi(root / f"{name}.mid", bytes.fromhex(hexdata))
    pedals, _ = render("pedals", inputs=[root / f"{n}.mid" for n in names], preset=loop)
    assert (pedals / "regular.wav").read_bytes() == (pedals / "held.wav").read_bytes()
    assert (pedals / "later.wav").read_bytes() == (pedals / "sostenuto.wav").read_bytes()
    assert read_wav(pedals / "later.wav")[1] > read_wav(pedals / "held.wav")[1] + RATE // 4
    assert read_wav(pedals / "held.wav")[1] % 1024 == 0

    processed = root / "processed.sfz"
    processed.write_text(loop.read_text().strip() + " fil_type=lpf_2p cutoff=1200 lfo1_freq=3 lfo1_pitch=120\n")
    filtered, _ = render("filtered", inputs=(root / "regular.mid", root / "later.mid"), preset=processed)
    assert (filtered / "regular.wav").read_bytes() != (pedals / "regular.wav").read_bytes()

    hot = root / "hot.sfz"
    centered = sfz.read_text().strip() + " pan_oncc10=0"
    hot.write_text(centered + " volume=33\n")
    repaired, _ = render("repaired", preset=hot)
    assert abs(int(np.abs(pcm(repaired / "source.wav")).max()) - round(32768 * 10 ** (-1 / 20))) <= 1
    hot.write_text(centered + " volume=42\n")
    rejected, result = render("too-hot", preset=hot, expected=2)
    assert "excessive_peak" in result.stderr and not (rejected / "source.wav").exists()

    write_wav(root / "short.wav", struct.pack("<h", 1600) * (RATE * 2 // 5))
    short = root / "short.sfz"
    short.write_text(sfz.read_text().replace("sample.wav", "short.wav"))
    midi(root / "gap.mid", bytes.fromhex("00 90 3c 64 8b 20 80 3c 00 00 ff 2f 00"))
    padded, _ = render("padded", inputs=(root / "gap.mid",), preset=short)
    channels, frames, samples = read_wav(padded / "gap.wav")
    assert (channels, frames) == (1, 65 * 1024) and not any(samples[(RATE * 2 // 5) * 2:])

    many = [root / f"batch-{i}.mid" for i in range(66)]
    for path in many:
        path.write_bytes((root / "regular.mid").read_bytes())
    many[64].write_bytes(b"invalid MIDI")
    output, result = render("pipeline", "--passes", "2", inputs=many, preset=short, expected=2)
    assert len(list(output.glob("*.wav"))) == 65
    assert sum(line.startswith("OK\t") for line in result.stdout.splitlines()) == 130
    assert (output / "batch-0.wav").read_bytes() == (output / "batch-65.wav").read_bytes()


@pytest.fixture(scope="module")
def group_inputs(tmp_path_factory):
    """check_group_audio.py:23-32."""
    root = tmp_path_factory.mktemp("group")
    midi(root / "melody.mid", bytes.fromhex("00 90 3c 64 83 60 80 3c 00 00 ff 2f 00"))
    for name, value in [("soft", 1600), ("loud", 6400), ("quiet", 100), ("tiny", 8)]:
        write_wav(root / f"{name}.wav", struct.pack("<h", value) * RATE)
        (root / f"{name}.sfz").write_text(f"<region> sample={name}.wav key=60 loop_mode=one_shot amp_veltrack=0\n")
    (root / "invalid.mid").write_bytes(b"not MIDI")
    return root


ROWS = [("pair", "soft", "melody", "soft"), ("-", "loud", "melody", "independent"),
        ("pair", "quiet", "melody", "quiet"), ("pair", "loud", "melody", "loud")]


def render_jobs(clay, root, directory, rows, *flags, expected=0):
    manifest = root / f"{directory}.tsv"
    manifest.write_text("".join(f"{g}\t{p}.sfz\t{m}.mid\t{directory}/{o}.wav\n" for g, p, m, o in rows))
    return run(clay, "--jobs", manifest, *flags, expected=expected)


def test_group_volume_and_quality_gate(clay, group_inputs):
    """check_group_audio.py:51-124."""
    root = group_inputs
    render_jobs(clay, root, "off", ROWS)
    accepted = [row for row in ROWS if row[1] != "quiet"]
    render_jobs(clay, root, "resume", accepted, "--group-volume", "mean")
    member = root / "resume/soft.wav"
    reference = member.read_bytes()
    member.write_bytes(reference[:len(reference) // 2])
    resumed = render_jobs(clay, root, "resume", accepted, "--group-volume", "mean", "--resume")
    assert resumed.stdout.count("SKIP\t") == 1 and resumed.stdout.count("OK\t") == 2
    assert member.read_bytes() == reference
    complete = render_jobs(clay, root, "resume", accepted, "--group-volume", "mean", "--resume")
    assert complete.stdout.count("SKIP\t") == 3 and "DEVICE\t" not in complete.stdout

    grouped = render_jobs(clay, root, "on", ROWS, "--group-volume", "mean", "--quality-gate", "clayengine",
                          expected=2)
    assert "quiet_performance" in grouped.stderr and not (root / "on/quiet.wav").exists()
    assert (root / "off/independent.wav").read_bytes() == (root / "on/independent.wav").read_bytes()
    assert len([line for line in grouped.stdout.splitlines() if line.startswith("VOLUME\t")]) == 2
    soft, loud = (pcm(root / f"off/{name}.wav") for name in ("soft", "loud"))
    body = RATE // 2
    levels = [math.sqrt(sum(int(x) * int(x) for x in s[:body]) / body) for s in (soft, loud)]
    target = sum(levels) / 2
    for name, samples, level in zip(("soft", "loud"), (soft, loud), levels):
        assert list(pcm(root / f"on/{name}.wav")) == [round(int(x) * (target / level)) for x in samples]
    downloaded, spilled, waiting = transfer(grouped)
    assert 0 < downloaded <= sum((root / f"on/{n}.wav").stat().st_size - 44 for n in ("soft", "loud", "independent"))
    assert (spilled, waiting) == (0, 0)

    quiet = [("-", "quiet", "melody", "out")]
    rejected = render_jobs(clay, root, "rejected", quiet, "--quality-gate", "clayengine", expected=2)
    assert "quiet_performance" in rejected.stderr and transfer(rejected) == (0, 0, 0)
    render_jobs(clay, root, "custom", quiet, "--quality-gate", "custom", "--qa-min-onset-median-dbfs", "-70",
                "--qa-min-onset-quartile-dbfs", "-75")
    assert (root / "custom/out.wav").read_bytes() == (root / "off/quiet.wav").read_bytes()
    short = render_jobs(clay, root, "too-long", ROWS[:1], "--quality-gate", "custom", "--qa-max-seconds", ".6",
                        expected=2)
    assert "rendered_audio_too_long" in short.stderr and transfer(short) == (0, 0, 0)
    incomplete = render_jobs(clay, root, "incomplete", [("pair", "soft", "melody", "one"),
                                                        ("pair", "loud", "invalid", "two")],
                             "--group-volume", "mean", expected=2)
    assert "insufficient_qualified_group_members" in incomplete.stderr and transfer(incomplete) == (0, 0, 0)
    tiny = render_jobs(clay, root, "tiny", [("-", "tiny", "melody", "out")], "--quality-gate", "custom",
                       "--qa-min-onset-median-dbfs", "-120", "--qa-min-onset-quartile-dbfs", "-120",
                       "--qa-max-silence-fraction", "1", expected=2)
    assert "effectively_silent_audio" in tiny.stderr and transfer(tiny) == (0, 0, 0)
    midi(root / "gap.mid", bytes.fromhex("00 90 3c 64 60 80 3c 00 96 40 90 3c 64 60 80 3c 00 00 ff 2f 00"))
    silent = render_jobs(clay, root, "gap", [("-", "soft", "gap", "out")], "--quality-gate", "custom",
                         "--qa-max-silence-seconds", "1", expected=2)
    assert "excessive_audio_silence" in silent.stderr and transfer(silent) == (0, 0, 0)

    stereo = render_jobs(clay, root, "stereo", ROWS, "--tail-policy", "orig", "--group-volume", "mean",
                         "--quality-gate", "clayengine", expected=2)
    assert "quiet_performance" in stereo.stderr and read_wav(root / "stereo/soft.wav")[0] == 2
    (root / "hot.sfz").write_text((root / "loud.sfz").read_text().strip() + " volume=30\n")
    clipped = render_jobs(clay, root, "clipped", [("-", "hot", "melody", "out")], "--tail-policy", "orig",
                          "--quality-gate", "clayengine", expected=2)
    assert "excessive_audio_clipping" in clipped.stderr and transfer(clipped) == (0, 0, 0)

    write_wav(root / "spiky.wav", struct.pack("<h", 12000) * (RATE // 1000) + struct.pack("<h", 100) * RATE)
    (root / "spiky.sfz").write_text((root / "soft.sfz").read_text().strip().replace("soft.wav", "spiky.wav")
                                    + " volume=10\n")
    limited = render_jobs(clay, root, "peak-limit", [("pair", "loud", "melody", "loud"),
                                                     ("pair", "spiky", "melody", "spiky")], "--group-volume", "mean")
    levels = [list(map(float, line.split("\t")[2:])) for line in limited.stdout.splitlines()
              if line.startswith("VOLUME\t")]
    assert levels[0][1] == levels[1][1] < (levels[0][0] + levels[1][0]) / 2
    assert int(np.abs(pcm(root / "peak-limit/spiky.wav")).max()) == round(32767 * 10 ** (-1 / 20))


def test_group_split_across_batches(clay, group_inputs):
    """check_group_audio.py:126-147: a group larger than a GPU batch."""
    root = group_inputs
    large = [("-", "soft", "melody", "solo")]
    large += [("large", "loud" if i % 2 else "soft", "melody", f"out-{i}") for i in range(65)]
    large += [("large", "quiet", "melody", "quiet"), ("small", "soft", "melody", "small-1"),
              ("small", "loud", "melody", "small-2")]
    flags = ("--group-volume", "mean", "--quality-gate", "clayengine")
    device = render_jobs(clay, root, "device", large, *flags, expected=2)
    host = render_jobs(clay, root, "host", large, *flags, "--group-wait-mib", "0", expected=2)
    wide = render_jobs(clay, root, "wide", large, *flags, "--cpu-batch-jobs", "1", "--gpu-batch-jobs", "128",
                       expected=2)
    device_bytes, device_spill, device_wait = transfer(device)
    host_bytes, host_spill, host_wait = transfer(host)
    assert device_bytes == host_bytes > device_wait > 0
    assert (device_spill, host_wait, host_spill) == (0, 0, device_wait)
    assert transfer(wide) == (device_bytes, 0, 0)
    assert device.stdout.index("solo.wav") < device.stdout.index("out-0.wav")
    for _, _, _, output in large:
        if output != "quiet":
            expected = (root / f"device/{output}.wav").read_bytes()
            assert (root / f"host/{output}.wav").read_bytes() == expected
            assert (root / f"wide/{output}.wav").read_bytes() == expected


def test_outputs_identical_across_batching_modes(clay, tmp_path):
    """check_segments.py: a held, bent, CC-modulated voice renders byte-identically
    whatever the GPU batch size, planning batch size and grouping."""
    write_wav(tmp_path / "sample.wav", b"".join(struct.pack("<h", round(3000 * math.sin(i * .04)))
                                                for i in range(RATE)))
    (tmp_path / "voice.sfz").write_text(
        "<region> sample=sample.wav key=60 loop_mode=loop_continuous loop_start=0 loop_end=44099 "
        "amp_veltrack=0 ampeg_release=1.7 cutoff=1800 resonance=3 cutoff_oncc1=3000 pitch_oncc1=37\n")
    midi(tmp_path / "long.mid", bytes.fromhex("00 b0 40 7f 00 90 3c 64 87 40 b0 01 40 87 40 e0 00 50 "
                                              "87 40 80 3c 00 87 40 b0 40 00 00 ff 2f 00"))
    midi(tmp_path / "short.mid", bytes.fromhex("00 90 3c 64 60 80 3c 00 00 ff 2f 00"))
    for tail, grouped in itertools.product(("natural", "orig"), (False, True)):
        outputs = []
        for name, cap, cpu in (("wide", 32, 64), ("single", 1, 64), ("pairs", 2, 64), ("prefetch", 2, 1)):
            directory = f"{name}-{tail}-{grouped}"
            manifest = tmp_path / f"{directory}.tsv"
            manifest.write_text("".join(f"{'pair' if grouped else '-'}\tvoice.sfz\t{source}.mid\t{directory}/{i}.wav\n"
                                        for i, source in enumerate(("short", "long", "short", "long"))))
            command = ["--jobs", manifest, "--tail-policy", tail, "--gpu-batch-jobs", cap, "--cpu-batch-jobs", cpu,
                       "--quality-gate", "off"]
            if grouped:
                command += ["--group-volume", "mean"]
            run(clay, *command, expected=0)
            outputs.append([(tmp_path / directory / f"{i}.wav").read_bytes() for i in range(4)])
        assert all(output == outputs[0] for output in outputs[1:]), (tail, grouped)


for _name in ("test_tail_policies", "test_group_volume_and_quality_gate", "test_group_split_across_batches",
              "test_outputs_identical_across_batching_modes"):
    for _mark in gpu:
        globals()[_name] = _mark(globals()[_name])
