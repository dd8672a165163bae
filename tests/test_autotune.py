"""The end-to-end autotuner: it picks a GPU batch size, a lane count and the
shared-source mode, caches the choice per workload, and what it picks changes no
job's audio."""
import numpy as np
import pytest

from conftest import gpu_available


def test_signature_depends_on_the_workload(ref_session, batch_mini, plain_small):
    from claysampler_b200 import autotune
    plans = [ref_session.plan(j.sfz, j.midi) for j in list(batch_mini) + list(plain_small)]
    assert autotune.signature(plans) == autotune.signature(list(plans))
    assert autotune.signature(plans) != autotune.signature(plans[:-1])


@pytest.mark.gpu
@pytest.mark.skipif(not gpu_available(), reason="needs a CUDA GPU")
def test_tuned_batching_keeps_every_job_identical(ref_session, batch_mini, plain_small, tmp_path):
    from claysampler_b200 import autotune
    from claysampler_b200.renderer import Renderer
    plans = [ref_session.plan(j.sfz, j.midi) for j in list(batch_mini) + list(plain_small)] * 2
    bank = ref_session.bank()
    cache = tmp_path / "autotune.json"
    tuned = autotune.tune(plans, bank, candidates=(1, 2, 8), repeats=1, cache=cache)
    assert tuned["batch_jobs"] in (1, 2, 8) and tuned["lanes"] in (2, 4)
    assert {"1/2/shared", "2/2/shared", "8/2/shared"} <= set(tuned["sweep"])
    best = tuned["batch_jobs"]
    assert {f"{best}/2/shared", f"{best}/2/plain", f"{best}/4/shared", f"{best}/4/plain"} <= set(tuned["sweep"])
    assert any(name.endswith("/side") for name in tuned["sweep"]) and isinstance(tuned["ordered_compute"], bool)
    assert all(v > 0 for v in tuned["sweep"].values())
    assert autotune.tune(plans, bank, candidates=(1, 2, 8), cache=cache) == tuned   # cached

    def render(batch_jobs, lanes=2, shared=True, ordered=True):
        renderer = Renderer(natural=True, batch_jobs=batch_jobs)
        renderer.set_lanes(lanes)
        renderer.set_shared_sources(shared)
        renderer.set_ordered_compute(ordered)
        renderer.upload_samples(bank)
        jobs = {}

        def publish(batch, first):
            for k, r in enumerate(batch.results):
                start = int(r["offset"])
                jobs[first + k] = (batch.pcm[start:start + int(r["dataFrames"])].copy(), r.copy())

        renderer.render_window(plans, publish)
        renderer.close()
        return jobs

    one = render(1, 1, False)
    tuned_jobs = render(tuned["batch_jobs"], tuned["lanes"], tuned["shared_sources"], tuned["ordered_compute"])
    side_jobs = render(2, 4, True, False)
    assert sorted(side_jobs) == sorted(one)
    for j in one:
        np.testing.assert_array_equal(one[j][0], side_jobs[j][0])
    assert sorted(one) == sorted(tuned_jobs) == list(range(len(plans)))
    for j in one:
        np.testing.assert_array_equal(one[j][0], tuned_jobs[j][0])
        for field in ("frames", "dataFrames", "fade", "peak", "first", "last", "status", "scale"):
            assert one[j][1][field] == tuned_jobs[j][1][field], (j, field)    # offsets differ by batch
