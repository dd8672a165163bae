"""The out-of-memory ladder of cs_render_window (src/cuda/renderer.cpp:947-992),
driven by host-side fault injection: cs_renderer_fail_allocations makes the next
batch-arena allocations report cudaErrorMemoryAllocation without calling the
allocator, so no device allocation actually fails.

Rungs: publish the batches in flight and free the other lanes' arenas, halve the
batch, halve a lone job's scratch budget (more segments), and finally reject the
job with a MEMORY line.  Every job that renders must come out byte-identical to
the render without injected failures."""
import numpy as np
import pytest

from conftest import gpu_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not gpu_available(), reason="needs a CUDA GPU")]


def render_all(plans, bank, fail=0, batch_jobs=4):
    from claysampler_b200.renderer import Renderer
    renderer = Renderer(natural=True, batch_jobs=batch_jobs)
    renderer.upload_samples(bank)
    renderer.fail_allocations(fail)
    batches = []
    renderer.render_window(plans, lambda batch, first: batches.append((first, batch)))
    renderer.close()
    return batches


def per_job(batches):
    jobs = {}
    for first, batch in batches:
        for k, r in enumerate(batch.results):
            start = int(r["offset"])
            jobs[first + k] = (batch.pcm[start:start + int(r["dataFrames"])].copy(), r.copy())
    return jobs


def same_jobs(a, b):
    assert sorted(a) == sorted(b)
    for ticket in a:
        assert np.array_equal(a[ticket][0], b[ticket][0]), ticket
        for field in ("status", "frames", "dataFrames", "fade", "peak", "first", "last"):
            assert a[ticket][1][field] == b[ticket][1][field], (ticket, field)


def test_batch_halves_when_its_arena_does_not_fit(ref_session, batch_mini, plain_small):
    plans = [ref_session.plan(j.sfz, j.midi) for j in list(batch_mini) + list(plain_small)]
    bank = ref_session.bank()
    clean = render_all(plans, bank)
    assert [len(b.results) for _, b in clean] == [4]
    halved = render_all(plans, bank, fail=1)
    assert [len(b.results) for _, b in halved] == [2, 2]
    same_jobs(per_job(clean), per_job(halved))


def test_lone_job_renders_in_more_segments(ref_session, batch_mini, capfd):
    plan = ref_session.plan(batch_mini[0].sfz, batch_mini[0].midi)
    bank = ref_session.bank()
    clean = render_all([plan], bank)
    capfd.readouterr()
    segmented = render_all([plan], bank, fail=1)
    err = capfd.readouterr().err
    assert "SEGMENT\tfirst=0\tjobs=1" in err, err
    assert "MEMORY" not in err
    same_jobs(per_job(clean), per_job(segmented))


def test_job_is_rejected_when_nothing_fits(ref_session, batch_mini, plain_small, capfd):
    from claysampler_b200.renderer import Renderer
    filtered = ref_session.plan(batch_mini[0].sfz, batch_mini[0].midi)
    other = ref_session.plan(plain_small[0].sfz, plain_small[0].midi)
    bank = ref_session.bank()
    clean = per_job(render_all([other], bank))
    capfd.readouterr()
    renderer = Renderer(natural=True)
    renderer.upload_samples(bank)
    renderer.fail_allocations(64)           # more than every rung takes
    batches = []
    renderer.render_window([filtered], lambda batch, first: batches.append((first, batch)))
    err = capfd.readouterr().err
    assert "MEMORY\tjob=0\t" in err, err
    assert len(batches) == 1 and batches[0][1].failed_scratch_bytes > 0 and len(batches[0][1].results) == 0
    # The renderer stays usable once allocations succeed again.
    renderer.fail_allocations(0)
    after = []
    renderer.render_window([other], lambda batch, first: after.append((first, batch)))
    renderer.close()
    same_jobs(clean, per_job(after))
