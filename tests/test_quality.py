"""Quality gate, group volume and accepted-PCM packing (the reference's
src/cuda/quality.cu).

* CPU: the oracle's restatement, fed by the reference's own planner and render
  (oracle/_ref), meets every expectation of the reference's group/quality test
  (tests/check_group_audio.py): verdict strings, exact group gains
  round(x * target / level), the -1 dBFS group ceiling, minimum group members.
* GPU (gpu-marked): the sm_100a assessment of a finished batch equals the oracle's
  assessment of the same finished PCM bit for bit (verdicts, levels, gains,
  offsets, accepted PCM), in-batch and for a group split across batches.
"""
import math
import struct
import wave

import numpy as np
import pytest

from claysampler_b200.plans import TAIL_STATUS, default_audio_config
from conftest import gpu_available

RATE = 44100
# check_group_audio.py:25 — one 0.5 s note at key 60.
MELODY = bytes.fromhex("00 90 3c 64 83 60 80 3c 00 00 ff 2f 00")
# check_group_audio.py:104 — two 0.1 s notes three seconds apart.
GAP = bytes.fromhex("00 90 3c 64 60 80 3c 00 96 40 90 3c 64 60 80 3c 00 00 ff 2f 00")


def write_midi(path, data):
    path.write_bytes(b"MThd" + struct.pack(">IHHH", 6, 0, 1, 480) + b"MTrk" + struct.pack(">I", len(data)) + data)


def write_mono(path, samples):
    with wave.open(str(path), "wb") as stream:
        stream.setparams((1, 2, RATE, 0, "NONE", "not compressed"))
        stream.writeframes(b"".join(struct.pack("<h", v) for v in samples) if not isinstance(samples, bytes)
                           else samples)


@pytest.fixture(scope="module")
def presets(tmp_path_factory):
    """Constant-level one-shot presets (soft 1600, loud 6400, quiet 100, tiny 8),
    a hot and a spiky variant, and the melody / gap MIDI files."""
    root = tmp_path_factory.mktemp("quality")
    for name, value in [("soft", 1600), ("loud", 6400), ("quiet", 100), ("tiny", 8)]:
        write_mono(root / f"{name}.wav", struct.pack("<h", value) * RATE)
        (root / f"{name}.sfz").write_text(
            f"<region> sample={name}.wav key=60 loop_mode=one_shot amp_veltrack=0\n", encoding="ascii")
    (root / "hot.sfz").write_text("<region> sample=loud.wav key=60 loop_mode=one_shot amp_veltrack=0 volume=30\n",
                                  encoding="ascii")
    write_mono(root / "spiky.wav", struct.pack("<h", 12000) * (RATE // 1000) + struct.pack("<h", 100) * RATE)
    (root / "spiky.sfz").write_text("<region> sample=spiky.wav key=60 loop_mode=one_shot amp_veltrack=0 volume=10\n",
                                    encoding="ascii")
    write_midi(root / "melody.mid", MELODY)
    write_midi(root / "gap.mid", GAP)
    return root


def custom_config(**thresholds):
    """audioConfig() with --quality-gate custom and --qa-* options (src/main.cpp:169-187)."""
    config = default_audio_config(RATE, quality=True)
    power = lambda dbfs: 4294967296.0 * 10.0 ** (dbfs / 10)  # noqa: E731
    for name, value in thresholds.items():
        if name == "max_seconds":
            config["maxFrames"] = int(math.floor(value * RATE))
        elif name == "min_median":
            config["minMedian"] = value
        elif name == "min_quartile":
            config["minQuartile"] = value
        elif name == "silence_dbfs":
            config["silencePower"] = power(value)
        elif name == "max_silence_fraction":
            config["maxSilentFraction"] = value
        elif name == "max_silence_seconds":
            config["maxSilentFrames"] = value * RATE
        else:
            raise KeyError(name)
    return config


def schedule(rows, group_volume):
    """Manifest rows (group name or '-', preset, midi) in the order the reference CLI
    renders them, with their group ids: a group takes a slot at its first member and
    collects its later members there; ungrouped rows take a slot each
    (src/main.cpp:208-246)."""
    slots, index = [], {}
    for group, preset, midi in rows:
        if group_volume and group != "-":
            if group not in index:
                index[group] = len(slots)
                slots.append([])
            slots[index[group]].append((index[group] + 1, preset, midi))
        else:
            slots.append([(0, preset, midi)])
    return [row for slot in slots for row in slot]


def plan_rows(session, root, rows, tail="natural", quality=False, group_volume=False):
    return [session.plan(root / f"{preset}.sfz", root / f"{midi}.mid", tail=tail, quality=quality,
                         group_volume=group_volume, group=gid)
            for gid, preset, midi in schedule(rows, group_volume)]


def oracle_render(session, root, rows, config=None, group_minimum=0, tail="natural"):
    """The reference's render (oracle/_ref) finished and assessed by the oracle."""
    from oracle import oracle, reference
    natural = tail == "natural"
    quality = config is not None and bool(config["enabled"])
    plans = plan_rows(session, root, rows, tail, quality, group_minimum > 0)
    mix = reference.synthesize(plans, session.bank(), natural)
    finished, results = oracle.finish(mix, plans, natural, quality=quality)
    if config is None and not group_minimum:
        return plans, finished, results
    config = default_audio_config(RATE) if config is None else config
    accepted, results = oracle.assess(finished, results, plans, natural, config, group_minimum)
    return plans, accepted, results


def job_pcm(pcm, results, i, channels=1):
    r = results[i]
    first = int(r["offset"]) * channels
    return pcm[first:first + int(r["dataFrames"]) * channels].astype(np.int64)


def status(results, i):
    return TAIL_STATUS[int(results[i]["status"])]


ROWS = [("pair", "soft", "melody"), ("-", "loud", "melody"), ("pair", "quiet", "melody"), ("pair", "loud", "melody")]
# Rendered (scheduled) order of ROWS with group volume on: soft, quiet, loud (the
# pair), then the independent loud job.
SOFT, QUIET, LOUD, INDEPENDENT = range(4)


def test_schedule_keeps_groups_together():
    assert schedule(ROWS, True) == [(1, "soft", "melody"), (1, "quiet", "melody"), (1, "loud", "melody"),
                                    (0, "loud", "melody")]
    assert schedule(ROWS, False) == [(0, p, m) for _, p, m in ROWS]


def test_oracle_group_gain_and_quiet_verdict(ref_session, presets):
    # check_group_audio.py:51, 70-80
    _, off_pcm, off = oracle_render(ref_session, presets, [("-", p, m) for _, p, m in schedule(ROWS, True)])
    _, on_pcm, on = oracle_render(ref_session, presets, ROWS, default_audio_config(RATE, quality=True), 2)
    assert status(on, QUIET) == "quietPerformance" and on[QUIET]["dataFrames"] == 0
    assert np.array_equal(job_pcm(off_pcm, off, INDEPENDENT), job_pcm(on_pcm, on, INDEPENDENT))
    assert [float(on[i]["audio"]["gain"]) > 0 for i in range(4)] == [True, False, True, False]
    body = RATE // 2
    soft, loud = job_pcm(off_pcm, off, SOFT), job_pcm(off_pcm, off, LOUD)
    levels = [math.sqrt(sum(int(x) * int(x) for x in s[:body]) / body) for s in (soft, loud)]
    target = sum(levels) / 2
    for i, samples, level in ((SOFT, soft, levels[0]), (LOUD, loud, levels[1])):
        assert on[i]["audio"]["bodyRms"] == level
        assert list(job_pcm(on_pcm, on, i)) == [round(int(x) * (target / level)) for x in samples]


def test_oracle_custom_thresholds_and_verdicts(ref_session, presets):
    quiet = [("-", "quiet", "melody")]
    _, _, rejected = oracle_render(ref_session, presets, quiet, default_audio_config(RATE, quality=True))
    assert status(rejected, 0) == "quietPerformance"                               # :82-84
    _, off_pcm, off = oracle_render(ref_session, presets, quiet)
    _, pcm, accepted = oracle_render(ref_session, presets, quiet, custom_config(min_median=-70, min_quartile=-75))
    assert status(accepted, 0) == "ok" and np.array_equal(job_pcm(pcm, accepted, 0), job_pcm(off_pcm, off, 0))
    _, _, long = oracle_render(ref_session, presets, ROWS[:1], custom_config(max_seconds=.6))
    assert status(long, 0) == "audioDuration"                                     # :88-89
    _, _, tiny = oracle_render(ref_session, presets, [("-", "tiny", "melody")],
                               custom_config(min_median=-120, min_quartile=-120, max_silence_fraction=1))
    assert status(tiny, 0) == "silentAudio"                                       # :94-97
    _, _, gap = oracle_render(ref_session, presets, [("-", "soft", "gap")], custom_config(max_silence_seconds=1))
    assert status(gap, 0) == "excessiveSilence"                                   # :101-103
    assert gap[0]["audio"]["longestSilence"] > RATE


def test_oracle_incomplete_group(ref_session, presets):
    # :90-93 — the second member's MIDI fails to plan, so the group keeps one member.
    _, _, results = oracle_render(ref_session, presets, [("pair", "soft", "melody")], None, 2)
    assert status(results, 0) == "incompleteGroup"


def test_oracle_stereo_and_clipping(ref_session, presets):
    # :105-112
    _, _, stereo = oracle_render(ref_session, presets, ROWS, default_audio_config(RATE, quality=True), 2, "orig")
    assert status(stereo, QUIET) == "quietPerformance"
    _, _, hot = oracle_render(ref_session, presets, [("-", "hot", "melody")],
                              default_audio_config(RATE, quality=True), tail="orig")
    assert status(hot, 0) == "clipping"


def test_oracle_group_peak_ceiling(ref_session, presets):
    # :119-124 — the spiky member limits the group target to -1 dBFS of its peak.
    rows = [("pair", "loud", "melody"), ("pair", "spiky", "melody")]
    _, pcm, results = oracle_render(ref_session, presets, rows, None, 2)
    audio = results["audio"]
    assert audio["targetRms"][0] == audio["targetRms"][1] < audio["bodyRms"].mean()
    assert int(np.abs(job_pcm(pcm, results, 1)).max()) == round(32767 * 10 ** (-1 / 20))


# ---- GPU ---------------------------------------------------------------------------

gpu = [pytest.mark.gpu, pytest.mark.skipif(not gpu_available(), reason="needs a CUDA GPU")]


def gpu_render(plans, bank, natural, config=None, group_minimum=0, batch_jobs=64, waiting=256 << 20):
    """Every batch render_window publishes, in job order: (pcm per job, results)."""
    from claysampler_b200.plans import TAIL_RESULT
    from claysampler_b200.renderer import Renderer
    renderer = Renderer(natural=natural, audio=config, group_minimum=group_minimum, batch_jobs=batch_jobs,
                        waiting_limit=waiting)
    renderer.upload_samples(bank)
    channels = 1 if natural else 2
    jobs = [None] * len(plans)
    results = np.zeros(len(plans), TAIL_RESULT)

    def publish(batch, first):
        assert not batch.failed_scratch_bytes
        for i, r in enumerate(batch.results):
            results[first + i] = r
            start = int(r["offset"]) * channels
            jobs[first + i] = batch.pcm[start:start + int(r["dataFrames"]) * channels].copy()

    renderer.render_window(plans, publish)
    counters = (renderer.downloaded_bytes, renderer.spilled_bytes, renderer.peak_waiting_bytes)
    renderer.close()
    return jobs, results, counters


def concat(jobs, results, channels):
    """Jobs' PCM packed at their result offsets (one batch)."""
    total = max((int(r["offset"]) + int(r["dataFrames"])) * channels for r in results) if len(results) else 0
    out = np.zeros(total, np.int16)
    for pcm, r in zip(jobs, results):
        out[int(r["offset"]) * channels:int(r["offset"]) * channels + pcm.size] = pcm
    return out


def compare_assessed(results, expected):
    exact = ("offset", "frames", "dataFrames", "fade", "peak", "first", "last", "status")
    for field in exact:
        np.testing.assert_array_equal(results[field], expected[field], err_msg=field)
    for field in ("silentFraction", "clippedFraction", "bodyRms", "targetRms", "gain", "longestSilence",
                  "clipped", "verdict", "measured"):
        np.testing.assert_array_equal(results["audio"][field], expected["audio"][field], err_msg=field)
    for field in ("median", "quartile"):                   # log10 on device and host
        np.testing.assert_allclose(results["audio"][field], expected["audio"][field], rtol=1e-12, atol=1e-12)


def assess_case(plans, bank, natural, config, group_minimum):
    from oracle import oracle
    channels = 1 if natural else 2
    plain_jobs, plain, _ = gpu_render(plans, bank, natural)
    finished = concat(plain_jobs, plain, channels)
    expected_pcm, expected = oracle.assess(finished, plain, plans, natural,
                                           config if config is not None else default_audio_config(RATE),
                                           group_minimum)
    jobs, results, _ = gpu_render(plans, bank, natural, config, group_minimum)
    compare_assessed(results, expected)
    assert np.array_equal(concat(jobs, results, channels), expected_pcm)
    return results


@pytest.mark.parametrize("tail", ["natural", "orig"])
def test_gpu_assessment_matches_oracle(ref_session, presets, tail):
    natural = tail == "natural"
    config = default_audio_config(RATE, quality=True)
    rows = ROWS + [("trio", "soft", "gap"), ("trio", "spiky", "melody"), ("trio", "loud", "gap"),
                   ("-", "tiny", "melody"), ("-", "hot", "melody")]
    plans = plan_rows(ref_session, presets, rows, tail, True, True)
    results = assess_case(plans, ref_session.bank(), natural, config, 2)
    assert status(results, QUIET) == "quietPerformance"


def test_gpu_assessment_real_music(ref_session, batch_mini, plain_small):
    """Dense music: onset percentiles over many notes, silence runs, both groups."""
    config = default_audio_config(RATE, quality=True)
    plans = [ref_session.plan(j.sfz, j.midi, quality=True, group_volume=True, group=1 + i // 2)
             for i, j in enumerate(list(batch_mini) + list(plain_small))]
    results = assess_case(plans, ref_session.bank(), True, config, 2)
    assert results["audio"]["measured"].all()


def test_gpu_group_split_across_batches(ref_session, presets):
    """A 66-member group with a rejected member is rendered in chunks (64-job
    batches): the waiting PCM on the device, or spilled to host memory, packs to
    the same output as one wide batch (check_group_audio.py:126-147)."""
    config = default_audio_config(RATE, quality=True)
    rows = [("-", "soft", "melody")]
    rows += [("large", "loud" if i % 2 else "soft", "melody") for i in range(65)]
    rows += [("large", "quiet", "melody"), ("small", "soft", "melody"), ("small", "loud", "melody")]
    plans = plan_rows(ref_session, presets, rows, "natural", True, True)
    bank = ref_session.bank()
    device_jobs, device, (device_bytes, device_spill, device_wait) = gpu_render(plans, bank, True, config, 2)
    host_jobs, host, (host_bytes, host_spill, host_wait) = gpu_render(plans, bank, True, config, 2, waiting=0)
    wide_jobs, wide, (wide_bytes, wide_spill, wide_wait) = gpu_render(plans, bank, True, config, 2, batch_jobs=128)
    assert device_bytes == host_bytes == wide_bytes > device_wait > 0
    assert (device_spill, host_wait, host_spill) == (0, 0, device_wait)
    assert (wide_spill, wide_wait) == (0, 0)
    assert status(device, 66) == "quietPerformance"
    for name, jobs, results in (("host", host_jobs, host), ("wide", wide_jobs, wide)):
        for field in ("frames", "dataFrames", "peak", "first", "last", "status"):
            np.testing.assert_array_equal(results[field], device[field], err_msg=f"{name} {field}")
        np.testing.assert_array_equal(results["audio"]["gain"], device["audio"]["gain"], err_msg=name)
        for a, b in zip(jobs, device_jobs):
            assert np.array_equal(a, b), name


for _name in ("test_gpu_assessment_matches_oracle", "test_gpu_assessment_real_music",
              "test_gpu_group_split_across_batches"):
    for _mark in gpu:
        globals()[_name] = _mark(globals()[_name])
