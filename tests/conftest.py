import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 GPU (B200); run with -m gpu")


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def plain_small(tmp_path_factory):
    """The 12-region mono preset and one 30 s / 64-note MIDI file."""
    from claysampler_b200 import workload
    root = tmp_path_factory.mktemp("plain_small")
    return workload.write_plain_small(root)


@pytest.fixture(scope="session")
def batch_mini(tmp_path_factory):
    """A reduced plain-batch preset (13 keys x 2 layers, stereo 24-bit, loops,
    lpf_2p + filter envelope + LFO) and three MIDI files of 8-20 s with pedal."""
    from claysampler_b200 import workload
    root = tmp_path_factory.mktemp("batch_mini")
    return workload.write_plain_batch(root, seed=5, jobs=3, min_seconds=8, max_seconds=20,
                                      keys=range(48, 61), layers=2)


@pytest.fixture(scope="session")
def ref_session():
    from oracle import reference
    if not reference.available():
        reference.build()
    if not reference.available():
        pytest.skip("oracle/_ref (the reference built for the host) is not available")
    session = reference.RefSession()
    yield session
    session.close()


def reference_mix(plans, bank, natural=True):
    """The reference's float mix of `plans`: its own render.cu kernels on the GPU
    (the contract's oracle, built with its NVRTC defaults) where that build exists,
    else its render.cu built for the host.  Orig/custom (PCM16) mixes come from the
    host build."""
    from oracle import reference
    if natural and reference.gpu_available() and gpu_available():
        return reference.synthesize_gpu(plans, bank)
    return reference.synthesize(plans, bank, natural)
