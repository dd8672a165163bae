"""Offline builds of the native parts (no JIT, no torch extension cache).

* ``libclaysampler_b200.so`` - the sm_100a kernels and the C ABI of
  ``include/claysampler_b200.h``, built by nvcc in-tree next to this file.
* ``libclaysampler_host.so`` / ``claysampler`` - the C++17 host: SFZ and MIDI
  loading, the planner, WAV output and the command line (built by g++).
"""
from __future__ import annotations

import os
import shutil
import subprocess
from pathlib import Path

PACKAGE = Path(__file__).resolve().parent
ROOT = PACKAGE.parent
CSRC = PACKAGE / "csrc"
HOST = PACKAGE / "host"
LIBRARY = PACKAGE / "libclaysampler_b200.so"
HOST_LIBRARY = PACKAGE / "libclaysampler_host.so"
CLI = PACKAGE / "claysampler"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    found = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(found).exists():
        raise RuntimeError("nvcc not found")
    return found


def _stale(target: Path, sources: list[Path]) -> bool:
    if not target.exists():
        return True
    mtime = target.stat().st_mtime
    return any(src.stat().st_mtime > mtime for src in sources)


def _run(cmd: list[str]) -> None:
    result = subprocess.run(cmd, capture_output=True, text=True)
    if result.returncode:
        raise RuntimeError("build failed:\n" + " ".join(cmd) + "\n" + result.stdout + result.stderr)


def build_library(force: bool = False, verbose: bool = False) -> Path:
    sources = sorted(CSRC.glob("*.cu"))
    deps = (sources + sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.hpp"))
            + [ROOT / "include" / "claysampler_b200.h", ROOT / "include" / "claysampler_lifetime.h"])
    if force or _stale(LIBRARY, deps):
        tmp = LIBRARY.with_suffix(f".so.tmp{os.getpid()}")
        cmd = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O2",
               "-Xptxas", "-v" if verbose else "-O3", "-shared", "-o", str(tmp), *map(str, sources)]
        _run(cmd)
        os.replace(tmp, LIBRARY)
    return LIBRARY


def build_host(force: bool = False) -> Path | None:
    """The C++ host (planner, SFZ/MIDI/WAV, CLI); skipped while its sources are absent."""
    sources = sorted(HOST.glob("*.cpp"))
    if not sources:
        return None
    deps = sources + sorted(HOST.glob("*.hpp")) + [ROOT / "include" / "claysampler_b200.h",
                                                   ROOT / "include" / "claysampler_host.h"]
    deps = [d for d in deps if d.exists()]
    library_sources = [s for s in sources if s.name != "cli.cpp"]
    if force or _stale(HOST_LIBRARY, deps):
        tmp = HOST_LIBRARY.with_suffix(f".so.tmp{os.getpid()}")
        _run(["g++", "-std=c++17", "-O2", "-fPIC", "-ffp-contract=off", "-shared", "-o", str(tmp),
              *map(str, library_sources)])
        os.replace(tmp, HOST_LIBRARY)
    cli = HOST / "cli.cpp"
    if cli.exists() and (force or _stale(CLI, deps + [HOST_LIBRARY, LIBRARY])):
        tmp = CLI.with_suffix(f".tmp{os.getpid()}")
        _run(["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-o", str(tmp), str(cli),
              f"-L{PACKAGE}", "-lclaysampler_host", "-lclaysampler_b200", f"-Wl,-rpath,$ORIGIN", "-lpthread"])
        os.replace(tmp, CLI)
    return HOST_LIBRARY


def build_all(force: bool = False) -> None:
    build_library(force)
    build_host(force)
