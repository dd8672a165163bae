"""Note-lifetime predictor: the oracle pinned by finite differences and by torch's
bfloat16 rounding (CPU), the training set's note isolation (CPU, the project's
planner), and the CUDA kernels against the oracle plus the trained network's gain
over the estimate made without it (GPU)."""
import math

import numpy as np
import pytest

from conftest import gpu_available
from oracle import lifetime as ref

F, O, P = ref.F, ref.O, ref.PARAMS


def random_problem(n, seed):
    rng = np.random.default_rng(seed)
    params = np.zeros(P, np.float32)
    at = 0
    for fan_in, fan_out in ((F, ref.H), (ref.H, ref.H), (ref.H, O)):
        bound = math.sqrt(6.0 / fan_in)
        params[at:at + fan_in * fan_out] = rng.uniform(-bound, bound, fan_in * fan_out)
        params[at + fan_in * fan_out:at + fan_in * fan_out + fan_out] = rng.uniform(-0.1, 0.1, fan_out)
        at += fan_in * fan_out + fan_out
    features = rng.normal(size=(n, F)).astype(np.float32) * rng.uniform(0.5, 3, F).astype(np.float32) + 2
    targets = np.stack([rng.normal(10, 1.5, n), rng.normal(-20, 6, n)], axis=1).astype(np.float32)
    f64 = features.astype(np.float64)
    norm = np.concatenate([f64.mean(0), 1 / f64.std(0), targets.mean(0), targets.std(0)]).astype(np.float32)
    return params, norm, features, targets


# ---- CPU: the oracle ---------------------------------------------------------------

def test_oracle_gradient_matches_finite_differences():
    params, norm, features, targets = random_problem(48, 1)
    p64 = params.astype(np.float64)
    grad, loss = ref.gradient(p64, norm, features, targets, rounding=False)
    assert loss == pytest.approx(ref.loss(p64, norm, features, targets, rounding=False), rel=1e-12)
    rng = np.random.default_rng(2)
    picks = np.concatenate([rng.choice(np.arange(a, b), 6, replace=False) for a, b in
                            ((ref.W1_AT, ref.B1_AT), (ref.B1_AT, ref.W2_AT), (ref.W2_AT, ref.B2_AT),
                             (ref.B2_AT, ref.W3_AT), (ref.W3_AT, ref.B3_AT))] + [np.arange(ref.B3_AT, P)])
    h = 1e-6
    for i in picks:
        up, down = p64.copy(), p64.copy()
        up[i] += h
        down[i] -= h
        numeric = (ref.loss(up, norm, features, targets, False) - ref.loss(down, norm, features, targets, False)) / (2 * h)
        assert numeric == pytest.approx(grad[i], rel=1e-5, abs=1e-9), i


def test_oracle_bf16_rounding_matches_torch():
    import torch
    rng = np.random.default_rng(3)
    values = np.concatenate([rng.normal(0, 1, 4000), rng.normal(0, 1e-3, 4000)]).astype(np.float32)
    # exact ties: the low 16 bits 0x8000, with both parities of bit 16
    ties = (values.view(np.uint32) & 0xFFFF0000) | 0x8000
    values = np.concatenate([values, ties.view(np.float32)])
    expected = torch.tensor(values).to(torch.bfloat16).to(torch.float64).numpy()
    np.testing.assert_array_equal(ref.bf16(values), expected)


def test_oracle_label_rule():
    rng = np.random.default_rng(4)
    mix = (rng.normal(0, 1e-3, (5000, 2)) * np.exp(-np.arange(5000) / 1200.0)[:, None]).astype(np.float32)
    windows = np.array([[0, 2000], [2000, 5000], [5000, 5000]], np.int64)
    peaks, lasts = ref.labels(mix, windows, 10 ** (-90 / 20))
    m = np.max(np.abs(mix), axis=1)
    assert peaks[0] == m[:2000].max() and peaks[1] == m[2000:].max() and peaks[2] == 0
    loud = np.nonzero(m[2000:] >= np.float32(10 ** (-4.5)))[0]
    assert 0 < loud[-1] < 2999 and lasts[1] == loud[-1] and lasts[2] == -1


def test_training_jobs_isolate_notes(tmp_path):
    """Each training job's spans merge into exactly one run per note, and the plain
    estimate bounds every run's length from above (it is the planner's own bound)."""
    from claysampler_b200 import lifetime
    from claysampler_b200.host import Host
    specs = lifetime.write_training_jobs(tmp_path, seed=5, jobs=3, notes=24, instruments=1)
    host = Host()
    try:
        for spec in specs:
            plan = host.plan(spec.sfz, spec.midi, tail="natural")
            runs = lifetime.note_windows(plan, len(spec.notes))
            assert runs is not None
            features = np.array([lifetime.features_of(n) for n in spec.notes])
            bound = np.exp(lifetime.envelope_estimate(features)[:, 0])
            # MIDI ticks (480 per beat at 120 bpm) quantise the held time to 46 frames
            assert np.all(runs[:, 1] - runs[:, 0] <= bound + 64)
            onsets = np.array([n.onset for n in spec.notes]) * lifetime.RATE
            assert np.all(np.abs(runs[:, 0] - onsets) < 0.01 * lifetime.RATE)
    finally:
        host.close()


# ---- GPU: the kernels against the oracle -------------------------------------------

@pytest.mark.gpu
@pytest.mark.skipif(not gpu_available(), reason="needs a CUDA GPU")
def test_gpu_forward_matches_oracle():
    from claysampler_b200.lifetime import LifetimeNet
    params, norm, features, _ = random_problem(1000, 6)
    net = LifetimeNet()
    net.load(params, norm)
    got = net.predict(features).cpu().numpy().astype(np.float64)
    want = ref.forward(params, norm, features)
    np.testing.assert_allclose(got, want, rtol=0, atol=2e-3)


@pytest.mark.gpu
@pytest.mark.skipif(not gpu_available(), reason="needs a CUDA GPU")
def test_gpu_gradient_matches_oracle():
    """Fused forward + backward over 1000 samples (7 full CTAs and a ragged one)."""
    from claysampler_b200.lifetime import LifetimeNet
    params, norm, features, targets = random_problem(1000, 7)
    net = LifetimeNet()
    net.load(params, norm)
    got = net.gradient(features, targets).astype(np.float64)
    want, loss = ref.gradient(params, norm, features, targets)
    assert got[P] == pytest.approx(loss, rel=1e-5)
    scale = np.abs(want).max()
    assert np.max(np.abs(got[:P] - want)) <= 2e-4 * scale
    for a, b in ((ref.W1_AT, ref.B1_AT), (ref.W2_AT, ref.B2_AT), (ref.W3_AT, ref.B3_AT)):
        layer = want[a:b]
        assert np.max(np.abs(got[a:b] - layer)) <= 1e-3 * np.abs(layer).max()
    # the same call twice gives the same bits (fixed summation order)
    np.testing.assert_array_equal(net.gradient(features, targets), got.astype(np.float32))


@pytest.mark.gpu
@pytest.mark.skipif(not gpu_available(), reason="needs a CUDA GPU")
def test_gpu_adam_step_matches_oracle():
    from claysampler_b200.lifetime import LifetimeNet
    params, norm, features, targets = random_problem(512, 8)
    net = LifetimeNet()
    net.load(params, norm)
    rate = 1e-3
    net.train(features, targets, epochs=1, batch=512, rate=rate, decay=1.0)
    got = net.state()[0].astype(np.float64)
    grad, _ = ref.gradient(params, norm, features, targets)
    want, _, _ = ref.adam(params.astype(np.float64), np.zeros(P), np.zeros(P), grad, 1, rate)
    clear = np.abs(grad) > 1e-3 * np.abs(grad).max()
    assert np.max(np.abs(got - want)[clear]) <= 1e-3 * rate + 1e-6
    assert np.max(np.abs(got - want)) <= 2 * rate + 1e-6


@pytest.mark.gpu
@pytest.mark.skipif(not gpu_available(), reason="needs a CUDA GPU")
def test_gpu_labels_match_oracle():
    import torch
    from claysampler_b200 import lifetime
    rng = np.random.default_rng(9)
    frames = 300_000
    mix = (rng.normal(0, 1e-2, (frames, 2)) * np.exp(-np.arange(frames) / 30000.0)[:, None]).astype(np.float32)
    cuts = np.sort(rng.choice(np.arange(1, frames), 40, replace=False))
    edges = np.concatenate([[0], cuts, [frames]])
    windows = np.stack([edges[:-1], edges[1:]], axis=1)
    windows = np.concatenate([windows, [[frames, frames]]])
    device_mix = torch.tensor(mix, device="cuda:0")
    peak, last = lifetime.note_labels(device_mix.data_ptr(), windows)
    want_peak, want_last = ref.labels(mix, windows, lifetime.AUDIBLE)
    np.testing.assert_array_equal(peak, want_peak)
    np.testing.assert_array_equal(last, want_last)


@pytest.mark.gpu
@pytest.mark.skipif(not gpu_available(), reason="needs a CUDA GPU")
def test_gpu_trained_network_beats_the_plain_estimate(tmp_path):
    """Single-note renders by the renderer label a training set; the network trained on
    the GPU predicts held-out notes' audible lifetime and peak better than the estimate
    made without it, and its lifetime reservation cuts reserved frames."""
    from claysampler_b200 import lifetime
    features, targets, spans, job = lifetime.render_training_set(tmp_path, seed=13, jobs=60, notes=40,
                                                                 batch_jobs=30, instruments=1)
    assert len(features) == 60 * 40 and np.all(np.isfinite(targets))
    # the labels never exceed the rendered runs
    assert np.all(np.exp(targets[:, 0]) <= spans + 1)
    train, test = job < 48, job >= 48
    net = lifetime.LifetimeNet(seed=1)
    net.set_normalisation(lifetime.normalisation(features[train], targets[train]))
    history = net.train(features[train], targets[train], epochs=150, batch=256, rate=3e-3, decay=0.98)
    assert history[-1] < 0.5 * history[0]
    predicted = net.predict(features[test]).cpu().numpy()
    plain = lifetime.envelope_estimate(features[test])
    err_net = np.abs(predicted - targets[test]).mean(0)
    err_plain = np.abs(plain - targets[test]).mean(0)
    assert err_net[0] < err_plain[0] and err_net[1] < err_plain[1], (err_net, err_plain)
    # the same predictions from the oracle
    np.testing.assert_allclose(predicted, ref.forward(*net.state(), features[test]), atol=2e-3)


def test_preset_regions_and_reservation_rules(tmp_path):
    """A generated batch preset's regions parse with its <global> defaults, and a
    lifetime reservation never exceeds the plain bound and grows with the margin."""
    from claysampler_b200 import lifetime, workload
    sfz = workload.write_plain_batch_preset(tmp_path, seed=4, keys=range(60, 64), layers=2)
    regions = lifetime.preset_regions(sfz, 4.0)
    assert len(regions) == 8
    assert all(r.attack == 0.005 and r.decay == 1.5 and r.sustain == 0.5 and r.release == 0.5 for r in regions)
    assert all(200 <= r.cutoff <= 8000 and abs(r.fileg_depth) == 2400 for r in regions)
    assert {r.loop for r in regions} == {True, False}
    rng = np.random.default_rng(5)
    truth = rng.normal(10, 1, 1000)
    predicted = truth + rng.normal(0, 0.2, 1000)
    margin = lifetime.calibrate_margin(predicted, truth, 0.01)
    assert np.mean(truth - predicted > margin) <= 0.011
    plain = truth + 0.5
    reserved = lifetime.admission_reservation(predicted, plain, margin)
    assert np.all(reserved <= np.ceil(np.exp(plain))) and np.all(reserved >= 1)
    assert np.all(lifetime.admission_reservation(predicted, plain, margin + 0.1) >= reserved)
