"""The C ABI libraries load without a GPU and export every function that
include/*.h declares (no compute calls are made)."""
import ctypes
import re
from pathlib import Path

import pytest

from claysampler_b200 import build

ROOT = Path(__file__).resolve().parents[1]


def declared(header):
    text = re.sub(r"/\*.*?\*/", "", (ROOT / "include" / header).read_text(), flags=re.S)
    names = set(re.findall(r"\b(cs_\w+)\s*\(", text))
    typedefs = set(re.findall(r"\(\s*\*\s*(cs_\w+)\s*\)", text))
    return sorted(names - typedefs)


@pytest.mark.parametrize("header,library", [("claysampler_b200.h", "LIBRARY"), ("claysampler_lifetime.h", "LIBRARY"),
                                            ("claysampler_host.h", "HOST_LIBRARY")])
def test_library_exports_declared_symbols(header, library):
    path = getattr(build, library)
    if not path.exists():
        build.build_all()
    lib = ctypes.CDLL(str(path))
    missing = [name for name in declared(header) if not hasattr(lib, name)]
    assert not missing, missing
    assert len(declared(header)) >= 5


def test_plan_records_match_reference_layout():
    from claysampler_b200.plans import AUDIO_CONFIG, CONTROL_POINT, TAIL_RESULT, VOICE_MODULATION, VOICE_SPAN
    assert VOICE_SPAN.itemsize == 472 and VOICE_SPAN.fields["filteredOffset"][1] == 104
    assert VOICE_SPAN.fields["filters"][1] == 148 and VOICE_SPAN.fields["extraEnvelope"][1] == 248
    assert CONTROL_POINT.itemsize == 12 and VOICE_MODULATION.itemsize == 24
    assert TAIL_RESULT.itemsize == 112 and TAIL_RESULT.fields["audio"][1] == 40 and AUDIO_CONFIG.itemsize == 72
