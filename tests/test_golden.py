"""Golden fixtures (tests/golden/*.npz, made by tests/golden/make_golden.py from the
reference's own planner and render.cu built for the host).

* The reference's own test expectations (tests/check_tail.py) hold on them —
  this pins the oracle's restatement of the finishing stages.
* The oracle's restatement and the C++ planner reproduce them exactly.
* The GPU path reproduces them within the render tolerance (gpu-marked).
"""
import importlib.util
import math
from pathlib import Path

import numpy as np
import pytest

from claysampler_b200.plans import TAIL_RESULT, Plan
from conftest import gpu_available

GOLDEN = Path(__file__).resolve().parent / "golden"
RATE = 44100


def load(case):
    data = np.load(GOLDEN / f"{case}.npz")
    plan = Plan.from_blob(data["plan"].tobytes())
    results = np.frombuffer(data["results"].tobytes(), TAIL_RESULT)
    return plan, data["bank"], data["pcm"], results, bool(data["natural"])


def written(case):
    """The WAV the reference CLI would write: channels, frames and samples with the
    logical zero padding (src/io/audio.cpp:264-285)."""
    plan, _, pcm, results, natural = load(case)
    channels = 1 if natural else 2
    r = results[0]
    samples = np.zeros(int(r["frames"]) * channels, np.int16)
    samples[:int(r["dataFrames"]) * channels] = pcm[:int(r["dataFrames"]) * channels]
    return channels, int(r["frames"]), samples, r


def test_reference_tail_expectations_hold():
    # tests/check_tail.py:52-61
    channels, frames, samples, r = written("natural")
    assert (channels, frames) == (1, round(.65 * RATE))
    assert samples[frames - 5000] > 3 and samples[-1] == 0
    peaks = np.abs(samples.astype(np.int32))
    audible = np.nonzero(peaks > 3)[0]
    assert [int(r["frames"]), int(r["peak"]), int(r["first"]), int(r["last"])] == \
        [frames, int(peaks.max()), int(audible[0]), int(audible[-1])]
    # :63-64
    assert written("orig")[:2] == (2, round(5.1 * RATE))
    # :66-72
    channels, frames, custom, _ = written("custom")
    _, _, dry, _ = written("custom_dry")
    assert (channels, frames) == (2, round(1.1 * RATE) + 1)
    assert np.array_equal(custom[:-4410 * 2], dry[:-4410 * 2])
    assert not custom[-2:].any() and dry[-2:].any()
    # :74-77
    channels, frames, uncut, _ = written("custom_uncut")
    assert (channels, frames) == (2, round(3.4 * RATE))
    assert np.array_equal(uncut, written("orig")[2][:frames * 2])
    # :79-81
    assert load("limited")[3]["status"][0] == 1           # duration: tail or audio duration limit
    # :92-95
    held, regular = written("pedal_held"), written("pedal_regular")
    later, sostenuto = written("pedal_later"), written("pedal_sostenuto")
    assert held[1] == regular[1] and np.array_equal(held[2], regular[2])
    assert later[1] == sostenuto[1] and np.array_equal(later[2], sostenuto[2])
    assert later[1] > held[1] + RATE // 4 and held[1] % 1024 == 0
    # :97-101
    filtered = written("filtered_regular")
    assert filtered[1] != regular[1] or not np.array_equal(filtered[2], regular[2])
    # :103-112
    _, _, repaired, _ = written("repaired")
    assert abs(int(np.abs(repaired.astype(np.int32)).max()) - round(32768 * 10 ** (-1 / 20))) <= 1
    assert load("too_hot")[3]["status"][0] == 3           # peak: more than 5 dB attenuation
    # :114-125
    channels, frames, padded, _ = written("padded")
    assert (channels, frames) == (1, 65 * 1024)
    assert not padded[RATE * 2 // 5:].any()


CASES = sorted(p.stem for p in GOLDEN.glob("*.npz"))


@pytest.mark.parametrize("case", CASES)
def test_oracle_reproduces_golden(case):
    from oracle import oracle
    plan, bank, pcm, results, natural = load(case)
    mix = oracle.synthesize([plan], bank, natural)
    mine_pcm, mine = oracle.finish(mix, [plan], natural)
    assert np.array_equal(mine_pcm, pcm)
    assert mine.tobytes() == results.tobytes()


def test_host_planner_reproduces_golden_plans(tmp_path):
    from claysampler_b200.host import Host
    spec = importlib.util.spec_from_file_location("make_golden", GOLDEN / "make_golden.py")
    make = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(make)
    make.write_inputs(tmp_path)
    for case, (preset, midi, tail, options) in make.CASES.items():
        host = Host()
        mine = host.plan(tmp_path / f"{preset}.sfz", tmp_path / f"{midi}.mid", tail=tail, **options)
        plan, bank, _, _, _ = load(case)
        assert mine.to_blob() == plan.to_blob(), case
        assert np.array_equal(host.bank(), bank), case
        host.close()


@pytest.mark.gpu
@pytest.mark.skipif(not gpu_available(), reason="needs a CUDA GPU")
@pytest.mark.parametrize("case", CASES)
def test_gpu_reproduces_golden(case):
    from claysampler_b200.renderer import Renderer
    plan, bank, pcm, results, natural = load(case)
    renderer = Renderer(natural=natural)
    renderer.upload_samples(bank)
    prepared = renderer.prepare([plan])
    prepared.run()
    mine_pcm, mine = prepared.collect()
    prepared.close()
    renderer.close()
    for field in ("status", "frames", "dataFrames", "fade", "offset"):
        assert np.array_equal(mine[field], results[field]), field
    assert mine_pcm.shape == pcm.shape
    diff = np.abs(mine_pcm.astype(np.int32) - pcm.astype(np.int32))
    assert diff.max(initial=0) <= 1
    assert (np.mean(diff == 0) if diff.size else 1.0) >= 0.999
