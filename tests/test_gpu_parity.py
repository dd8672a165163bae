"""GPU parity: the sm_100a render path against the reference's own render
(oracle/_ref: the reference planner, and src/cuda/render.cu run as the reference
runs it on this GPU, or compiled for the CPU where no GPU build exists) and the
plain-C restatement of its finishing stages (oracle/).

Tolerances (the contract for this path): float bus max |error| <= 1e-5 of full
scale; PCM16 within 1 LSB with >= 99.9 % of samples identical; tail frame indices,
output lengths and statuses bit-exact.
"""
import numpy as np
import pytest

from conftest import gpu_available, reference_mix

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not gpu_available(), reason="needs a CUDA GPU")]

BUS_TOLERANCE = 1e-5
PCM_IDENTICAL = 0.999


def render(plans, bank, natural=True, scratch_limit=0):
    from claysampler_b200.renderer import Renderer
    renderer = Renderer(natural=natural)
    renderer.upload_samples(bank)
    if scratch_limit:
        renderer.set_scratch_limit(scratch_limit)
    prepared = renderer.prepare(plans)
    prepared.run()
    pcm, results = prepared.collect()
    mix = prepared.mix()
    segments = prepared.segments
    prepared.close()
    renderer.close()
    return mix, pcm, results, segments


def compare_pcm(pcm, expected):
    assert pcm.shape == expected.shape
    diff = np.abs(pcm.astype(np.int32) - expected.astype(np.int32))
    identical = float(np.mean(diff == 0)) if diff.size else 1.0
    assert diff.max(initial=0) <= 1, f"PCM16 differs by {diff.max()} LSB"
    assert identical >= PCM_IDENTICAL, f"only {identical:.5f} of PCM16 samples identical"
    return identical


def compare_results(results, expected):
    for field in ("status", "frames", "dataFrames", "fade", "offset"):
        np.testing.assert_array_equal(results[field], expected[field], err_msg=field)


def plan_jobs(session, jobs, tail="natural"):
    return [session.plan(j.sfz, j.midi, tail=tail) for j in jobs]


@pytest.mark.parametrize("tail", ["natural", "orig"])
def test_plain_small_matches_reference(plain_small, ref_session, tail):
    from oracle import oracle, reference
    plans = plan_jobs(ref_session, plain_small, tail)
    bank = ref_session.bank()
    natural = tail == "natural"
    mix, pcm, results, _ = render(plans, bank, natural)
    ref_mix = reference_mix(plans, bank, natural)
    if natural:
        err = float(np.max(np.abs(mix - ref_mix)))
        assert err <= BUS_TOLERANCE, err
    else:
        assert np.max(np.abs(mix.astype(np.int32) - ref_mix.astype(np.int32))) <= 1
    ref_pcm, ref_results = oracle.finish(ref_mix, plans, natural)
    compare_results(results, ref_results)
    compare_pcm(pcm, ref_pcm)


@pytest.mark.parametrize("tail", ["natural", "orig"])
def test_filtered_batch_matches_reference(batch_mini, ref_session, tail):
    from oracle import oracle, reference
    plans = plan_jobs(ref_session, batch_mini, tail)
    assert all(p.filter_tracks > 0 for p in plans)
    bank = ref_session.bank()
    natural = tail == "natural"
    mix, pcm, results, _ = render(plans, bank, natural)
    ref_mix = reference_mix(plans, bank, natural)
    if natural:
        err = float(np.max(np.abs(mix - ref_mix)))
        assert err <= BUS_TOLERANCE, err
    else:
        assert np.max(np.abs(mix.astype(np.int32) - ref_mix.astype(np.int32))) <= 1
    ref_pcm, ref_results = oracle.finish(ref_mix, plans, natural)
    compare_results(results, ref_results)
    compare_pcm(pcm, ref_pcm)


def test_segmented_synthesis_is_byte_identical(batch_mini, ref_session):
    """Chain state (filter history, smoothing, loop phase) carries across segments."""
    plans = plan_jobs(ref_session, batch_mini)
    bank = ref_session.bank()
    mix, pcm, results, segments = render(plans, bank)
    mix2, pcm2, results2, segments2 = render(plans, bank, scratch_limit=64 * 1024)
    assert segments == 1 and segments2 > 4
    assert np.array_equal(mix.view(np.uint32), mix2.view(np.uint32))
    assert np.array_equal(pcm, pcm2)
    assert results.tobytes() == results2.tobytes()


@pytest.mark.parametrize("fixture", ["plain_small", "batch_mini"])
def test_host_planned_batch_matches_oracle(request, fixture):
    """Self-contained on any GPU box: this package's planner feeds both the GPU
    path and the oracle's restatement of the reference render (no reference build
    needed)."""
    from claysampler_b200.host import Host
    from oracle import oracle
    jobs = request.getfixturevalue(fixture)
    host = Host()
    plans = [host.plan(j.sfz, j.midi) for j in jobs]
    bank = host.bank()
    mix, pcm, results, _ = render(plans, bank, True)
    expected_mix = oracle.synthesize(plans, bank, True)
    assert float(np.max(np.abs(mix - expected_mix))) <= BUS_TOLERANCE
    expected_pcm, expected = oracle.finish(expected_mix, plans, True)
    compare_results(results, expected)
    compare_pcm(pcm, expected_pcm)


def test_page_locked_plans_render_identically(batch_mini, ref_session):
    """Control points uploaded straight from page-locked plan arrays give the same
    render as points passed through the staging buffer."""
    from claysampler_b200.renderer import Renderer
    plans = plan_jobs(ref_session, batch_mini)
    bank = ref_session.bank()
    outputs = []
    for pinned in (False, True):
        if pinned:
            for plan in plans[::2]:     # a mix of page-locked and pageable plans
                plan.pin()
        renderer = Renderer(natural=True)
        renderer.upload_samples(bank)
        batches = []
        renderer.render_window(plans, lambda batch, first: batches.append((first, batch.pcm, batch.results)))
        renderer.close()
        outputs.append(batches)
    (a,), (b,) = outputs
    assert a[0] == b[0] and np.array_equal(a[1], b[1]) and a[2].tobytes() == b[2].tobytes()


def test_zero_copy_publish_matches_copied(plain_small, ref_session):
    """render_window(copy=False) hands publish a view of the download buffer; read
    during the callback it holds the same PCM as the copying default."""
    from claysampler_b200.renderer import Renderer
    plans = plan_jobs(ref_session, plain_small)
    renderer = Renderer(natural=True)
    renderer.upload_samples(ref_session.bank())
    copied, viewed = [], []
    renderer.render_window(plans, lambda batch, first: copied.append(batch.pcm))
    renderer.render_window(plans, lambda batch, first: viewed.append(batch.pcm.copy()), copy=False)
    renderer.close()
    assert len(copied) == len(viewed) == 1 and np.array_equal(copied[0], viewed[0])


def test_transposed_stereo_matches_reference(ref_session, tmp_path):
    """Every resampler load path with transposed voices: mono and stereo, inline and
    filtered (lpf_2p), a loop with its crossfade, and a stereo sample that starts at
    an odd float offset in the bank (after an odd-length mono sample)."""
    from claysampler_b200 import workload as wl
    from oracle import oracle, reference
    rng = np.random.default_rng(21)
    samples = tmp_path / "s"
    samples.mkdir()

    def sample(name, seconds, channels, extra=0):
        frames = int(seconds * wl.RATE) + extra
        t = np.arange(frames) / wl.RATE
        data = np.stack([np.sin(2 * np.pi * f * t + rng.uniform(0, 6)) * np.exp(-t / 1.2)
                         for f in rng.uniform(150, 900, channels)], axis=1)
        data += rng.standard_normal(data.shape) * 0.01
        wl.write_wav(samples / name, 0.5 * data / np.max(np.abs(data)), bits=24)
        return f"s/{name}"

    regions = [
        (sample("mono_odd.wav", 1.0, 1, extra=1), 40, 47, 44, ""),
        (sample("stereo_a.wav", 1.5, 2), 48, 55, 50, ""),
        (sample("mono_odd2.wav", 0.7, 1, extra=1), 56, 59, 57, ""),
        (sample("stereo_b.wav", 1.5, 2), 60, 67, 62, "fil_type=lpf_2p cutoff=3000 resonance=3"),
        (sample("stereo_c.wav", 2.0, 2), 68, 75, 70,
         "fil_type=lpf_2p cutoff=1500 loop_mode=loop_continuous loop_start=20000 loop_end=70000 "
         "loop_crossfade=0.01"),
    ]
    lines = ["<group> ampeg_attack=0.004 ampeg_decay=0.3 ampeg_sustain=70 ampeg_release=0.25\n"]
    for path, lo, hi, center, extra in regions:
        lines.append(f"<region> sample={path} lokey={lo} hikey={hi} pitch_keycenter={center} {extra}\n")
    sfz = tmp_path / "stereo.sfz"
    sfz.write_text("".join(lines), encoding="ascii")
    notes = [(0.05, 0.6, 41, 100), (0.3, 0.8, 53, 90), (0.5, 0.4, 58, 80)]
    notes += [(0.8 + 0.35 * i, float(rng.uniform(0.2, 1.5)), int(rng.integers(40, 76)), int(rng.integers(40, 127)))
              for i in range(24)]
    midi = tmp_path / "stereo.mid"
    wl._note_midi(notes, [], 11.0, midi)
    plans = [ref_session.plan(sfz, midi, tail="natural")]
    spans = plans[0].spans
    assert (spans["channels"] == 2).any() and (spans["channels"] == 1).any()
    assert (spans["step"] != 1).mean() > 0.5 and (spans["filterTrack"] >= 0).any()
    odd = (spans["channels"] == 2) & (spans["sample"] % 2 == 1)
    assert odd.any(), "no stereo sample at an odd float offset"
    bank = ref_session.bank()
    mix, pcm, results, _ = render(plans, bank, True)
    ref_mix = reference_mix(plans, bank, True)
    err = float(np.max(np.abs(mix - ref_mix)))
    assert err <= BUS_TOLERANCE, err
    ref_pcm, ref_results = oracle.finish(ref_mix, plans, True)
    compare_results(results, ref_results)
    compare_pcm(pcm, ref_pcm)
