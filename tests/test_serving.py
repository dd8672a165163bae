"""Serving: non-blocking submission with continuous batching (cs_submit /
cs_poll).  Jobs submitted while others are on the GPU are admitted as stream lanes
free up (and device memory allows), each batch is published as it finishes under
its jobs' tickets, and each job's audio and results are the same as when it is
rendered alone."""
import numpy as np
import pytest

from conftest import gpu_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not gpu_available(), reason="needs a CUDA GPU")]


def split_batch(batch, natural=True):
    """Per-job (pcm, result) pairs of one published batch."""
    channels = 1 if natural else 2
    out = []
    for r in batch.results:
        first = int(r["offset"]) * channels
        out.append((batch.pcm[first:first + int(r["dataFrames"]) * channels].copy(), r.copy()))
    return out


def alone(renderer, plan):
    got = []
    renderer.render_window([plan], lambda batch, first: got.extend(split_batch(batch)))
    return got[0]


def test_submissions_while_rendering_match_jobs_alone(ref_session, batch_mini, plain_small):
    from claysampler_b200.renderer import Renderer
    plans = [ref_session.plan(j.sfz, j.midi) for j in list(batch_mini) + list(plain_small)]
    plans += [ref_session.plan(j.sfz, j.midi) for j in batch_mini]          # repeats in other batches
    bank = ref_session.bank()
    renderer = Renderer(natural=True, batch_jobs=2)
    renderer.set_lanes(3)
    renderer.upload_samples(bank)
    published = {}
    order = []

    def publish(batch, first):
        order.append(first)
        for k, job in enumerate(split_batch(batch)):
            published[first + k] = job

    tickets = [renderer.submit(plans[:3])]
    assert renderer.pending_jobs == 3
    renderer.poll(publish)                           # whatever has finished, without waiting
    tickets.append(renderer.submit(plans[3:5]))      # arrives while the first jobs render
    renderer.poll(publish, wait=True)
    tickets.append(renderer.submit(plans[5:]))
    while renderer.pending_jobs:
        renderer.poll(publish, wait=True)
    assert tickets == [0, 3, 5]
    # Every ticket once; batches may finish (and publish) out of ticket order.
    assert sorted(published) == list(range(len(plans))) and len(order) == len(set(order))
    for ticket, plan in enumerate(plans):
        pcm, result = alone(renderer, plan)
        got_pcm, got_result = published[ticket]
        assert np.array_equal(pcm, got_pcm), ticket
        for field in ("frames", "dataFrames", "fade", "peak", "first", "last", "status"):
            assert result[field] == got_result[field], (ticket, field)
    renderer.close()


def test_render_window_waits_for_submitted_jobs(ref_session, plain_small):
    from claysampler_b200.renderer import Renderer
    plans = [ref_session.plan(j.sfz, j.midi) for j in plain_small]
    renderer = Renderer(natural=True)
    renderer.upload_samples(ref_session.bank())
    renderer.submit(plans)
    with pytest.raises(RuntimeError, match="poll them first"):
        renderer.render_window(plans, lambda batch, first: None)
    while renderer.pending_jobs:
        renderer.poll(lambda batch, first: None, wait=True)
    renderer.render_window(plans, lambda batch, first: None)
    renderer.close()
