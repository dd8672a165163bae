"""Learned note lifetime and peak (include/claysampler_lifetime.h).

An MLP (16 -> 64 -> 64 -> 2, BF16 weights, FP32 accumulation) predicts from a
note's region parameters, velocity, key and held time two things: the log of the
number of frames the note stays audible (its render's last frame at or above
-90 dBFS, counted from the note-on) and its peak level in dBFS.  It is trained
on the GPU by the library's own fused forward/backward and Adam kernels, on labels
measured from single-note renders made by the renderer itself
(:func:`render_training_set`).

The predictor never touches audio: no render path reads it, and every job is still
finished by the plain tail detection, so PCM is identical with or without it.
:func:`admission_reservation` turns a prediction into a per-note frame
reservation (raised by a margin calibrated on the training notes, capped by the
planner's own bound), and ``bench.py --learned`` reports how much less that
reserves than the plain bound and how often a note outlives its reservation.  The
renderer itself keeps reserving exactly what the plan needs: it renders every span
in full (that is what keeps PCM bit-identical), so a shorter predicted lifetime
cannot shrink its scratch without changing what is rendered.

Everything device-side goes through the C ABI with plain device pointers; torch is
only the allocator for those buffers.
"""
from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

from . import workload
from .renderer import library as _renderer_library

FEATURES = (
    "log_attack_s", "log_hold_s", "log_decay_s", "sustain", "log_release_s", "velocity", "key",
    "log2_cutoff_hz", "fileg_depth", "log_sample_s", "loop", "lfo_depth", "log_held_s", "transpose",
    "log_fileg_decay_s", "fileg_sustain",
)
OUTPUTS = ("log_audible_frames", "peak_dbfs")
F, H, O = 16, 64, 2
PARAMS = H * F + H + H * H + H + O * H + O
NORM = 2 * F + 2 * O
BLOCK_SAMPLES = 128
AUDIBLE_DBFS = -90.0
AUDIBLE = 10.0 ** (AUDIBLE_DBFS / 20.0)
RATE = workload.RATE
NO_FILTER_HZ = 22050.0
assert len(FEATURES) == F


def library() -> ctypes.CDLL:
    lib = _renderer_library()
    if not getattr(lib, "_lifetime_bound", False):
        c = ctypes
        vp, i32, f32 = c.c_void_p, c.c_int, c.c_float
        lib.cs_lifetime_forward.argtypes = [vp, vp, vp, i32, vp, vp]
        lib.cs_lifetime_partial_floats.argtypes = [i32]
        lib.cs_lifetime_partial_floats.restype = c.c_size_t
        lib.cs_lifetime_gradient.argtypes = [vp, vp, vp, vp, i32, vp, vp, vp]
        lib.cs_lifetime_train_step.argtypes = [vp, vp, vp, vp, vp, vp, i32, vp, i32, f32, vp, vp]
        lib.cs_note_labels.argtypes = [vp, vp, i32, f32, vp, vp, vp]
        lib.cs_lifetime_last_error.restype = c.c_char_p
        lib.cs_prepared_mix_device.argtypes = [vp, c.POINTER(vp), c.POINTER(c.c_size_t)]
        lib._lifetime_bound = True
    return lib


def _check(status: int) -> None:
    if status:
        raise RuntimeError(library().cs_lifetime_last_error().decode())


def _stream() -> int:
    import torch
    return torch.cuda.current_stream().cuda_stream


def initial_params(seed: int) -> np.ndarray:
    """He-uniform weights, zero biases, in the layout of the header."""
    rng = np.random.default_rng(seed)
    p = np.zeros(PARAMS, np.float32)
    at = 0
    for fan_in, fan_out in ((F, H), (H, H), (H, O)):
        bound = math.sqrt(6.0 / fan_in)
        p[at:at + fan_in * fan_out] = rng.uniform(-bound, bound, fan_in * fan_out)
        at += fan_in * fan_out + fan_out
    return p


def normalisation(features: np.ndarray, targets: np.ndarray) -> np.ndarray:
    f = np.asarray(features, np.float64)
    t = np.asarray(targets, np.float64)
    std = np.maximum(f.std(0), 1e-6)
    tstd = np.maximum(t.std(0), 1e-6)
    return np.concatenate([f.mean(0), 1.0 / std, t.mean(0), tstd]).astype(np.float32)


class LifetimeNet:
    """Parameters, Adam moments and normalisation resident on one device."""

    def __init__(self, device: str = "cuda:0", seed: int = 0):
        import torch
        self.torch = torch
        self.device = torch.device(device)
        self.params = torch.tensor(initial_params(seed), device=self.device)
        self.moment1 = torch.zeros(PARAMS, device=self.device)
        self.moment2 = torch.zeros(PARAMS, device=self.device)
        self.norm = torch.zeros(NORM, device=self.device)
        self.norm[F:2 * F] = 1
        self.norm[2 * F + O:] = 1
        self.steps = 0

    def _tensor(self, array) -> "torch.Tensor":
        t = self.torch.as_tensor(np.asarray(array, np.float32) if isinstance(array, np.ndarray) else array)
        return t.to(self.device, self.torch.float32).contiguous()

    def set_normalisation(self, norm: np.ndarray) -> None:
        self.norm.copy_(self._tensor(norm))

    def load(self, params: np.ndarray, norm: np.ndarray) -> None:
        self.params.copy_(self._tensor(params))
        self.set_normalisation(norm)

    def predict(self, features) -> "torch.Tensor":
        x = self._tensor(features)
        out = self.torch.empty((x.shape[0], O), device=self.device)
        _check(library().cs_lifetime_forward(self.params.data_ptr(), self.norm.data_ptr(), x.data_ptr(),
                                             x.shape[0], out.data_ptr(), _stream()))
        return out

    def gradient(self, features, targets) -> np.ndarray:
        """dL/dparams followed by L (PARAMS + 1 floats)."""
        x, t = self._tensor(features), self._tensor(targets)
        n = x.shape[0]
        partials = self.torch.empty(library().cs_lifetime_partial_floats(n), device=self.device)
        out = self.torch.empty(PARAMS + 1, device=self.device)
        _check(library().cs_lifetime_gradient(self.params.data_ptr(), self.norm.data_ptr(), x.data_ptr(),
                                              t.data_ptr(), n, partials.data_ptr(), out.data_ptr(), _stream()))
        return out.cpu().numpy()

    def train(self, features, targets, epochs: int = 20, batch: int = 4096, rate: float = 2e-3,
              seed: int = 0, decay: float = 0.85) -> list[float]:
        """Adam over shuffled minibatches; returns the mean minibatch loss of each epoch."""
        torch = self.torch
        x, t = self._tensor(features), self._tensor(targets)
        n = x.shape[0]
        steps = (n + batch - 1) // batch
        partials = torch.empty(library().cs_lifetime_partial_floats(min(batch, n)), device=self.device)
        losses = torch.zeros(steps, device=self.device)
        generator = torch.Generator(device=self.device)
        generator.manual_seed(seed)
        history = []
        lib = library()
        for epoch in range(epochs):
            order = torch.randperm(n, device=self.device, generator=generator)
            xs, ts = x[order].contiguous(), t[order].contiguous()
            lr = rate * decay ** epoch
            for s in range(steps):
                lo, hi = s * batch, min(n, (s + 1) * batch)
                self.steps += 1
                _check(lib.cs_lifetime_train_step(
                    self.params.data_ptr(), self.moment1.data_ptr(), self.moment2.data_ptr(),
                    self.norm.data_ptr(), xs[lo:hi].data_ptr(), ts[lo:hi].data_ptr(), hi - lo,
                    partials.data_ptr(), self.steps, lr, losses[s:s + 1].data_ptr(), _stream()))
            history.append(float(losses.mean().item()))
        return history

    def state(self) -> tuple[np.ndarray, np.ndarray]:
        return self.params.cpu().numpy(), self.norm.cpu().numpy()


def note_labels(mix_pointer: int, windows: np.ndarray, device: str = "cuda:0") -> tuple[np.ndarray, np.ndarray]:
    """Peak and last audible frame offset per frame window of a device float2 mix."""
    import torch
    w = torch.as_tensor(np.ascontiguousarray(windows, np.int64).reshape(-1, 2), device=device)
    n = w.shape[0]
    peak = torch.empty(n, device=device)
    last = torch.empty(n, dtype=torch.int32, device=device)
    _check(library().cs_note_labels(mix_pointer, w.data_ptr(), n, AUDIBLE, peak.data_ptr(), last.data_ptr(),
                                    _stream()))
    return peak.cpu().numpy(), last.cpu().numpy()


def targets_from_labels(peak: np.ndarray, last: np.ndarray) -> np.ndarray:
    frames = np.maximum(np.asarray(last, np.int64) + 1, 1)
    return np.stack([np.log(frames), 20 * np.log10(np.maximum(np.asarray(peak, np.float64), 1e-7))],
                    axis=1).astype(np.float32)


# ---- training instruments and single-note jobs ---------------------------------------

@dataclass
class Region:
    lokey: int
    hikey: int
    lovel: int
    hivel: int
    center: int
    attack: float
    hold: float
    decay: float
    sustain: float         # 0..1
    release: float
    cutoff: float          # NO_FILTER_HZ when unfiltered
    fileg_depth: float
    fileg_decay: float
    fileg_sustain: float   # 0..1
    lfo_depth: float
    loop: bool
    sample_seconds: float


@dataclass
class Note:
    onset: float
    held: float
    key: int
    velocity: int
    region: Region


@dataclass
class TrainingJob:
    sfz: Path
    midi: Path
    notes: list[Note] = field(default_factory=list)


def _log_uniform(rng, low, high):
    return float(math.exp(rng.uniform(math.log(low), math.log(high))))


def write_training_instrument(root: Path, seed: int, name: str, samples: int = 12) -> tuple[Path, list[Region]]:
    """One SFZ of 22 key zones x 4 velocity layers, every region with random envelope, filter,
    filter envelope, LFO depth, loop mode and one of `samples` decaying harmonic samples."""
    rng = np.random.default_rng(seed)
    folder = root / f"{name}_samples"
    folder.mkdir(parents=True, exist_ok=True)
    lengths = []
    for s in range(samples):
        seconds = float(rng.uniform(0.3, 4.0))
        frames = int(seconds * RATE)
        t = np.arange(frames) / RATE
        f0 = float(rng.uniform(60, 900))
        tau = _log_uniform(rng, 0.15, 4.0)
        channels = 2 if s % 2 else 1
        data = np.zeros((frames, channels))
        for k in range(1, 9):
            if k * f0 >= RATE / 2:
                break
            amp = float(rng.uniform(0.3, 1.0)) / k
            for c in range(channels):
                data[:, c] += amp * np.sin(2 * np.pi * k * f0 * t + rng.uniform(0, 2 * np.pi))
        data *= np.exp(-t / tau)[:, None]
        data += rng.standard_normal(data.shape) * 0.01 * np.exp(-t / 0.03)[:, None]
        data *= float(rng.uniform(0.1, 0.9)) / max(1e-9, float(np.max(np.abs(data))))
        workload.write_wav(folder / f"s{s:02d}.wav", data, bits=24)
        lengths.append(frames)
    regions = []
    lines = ["<global> fileg_attack=0.01 fileg_release=0.4 lfo1_freq=5\n"]
    for zone in range(22):
        lokey = 21 + 4 * zone
        for layer in range(4):
            s = int(rng.integers(0, samples))
            frames = lengths[s]
            region = Region(
                lokey=lokey, hikey=lokey + 3, lovel=max(1, 32 * layer), hivel=32 * layer + 31,
                center=int(rng.integers(lokey - 6, lokey + 10)),
                attack=_log_uniform(rng, 0.001, 0.3), hold=float(rng.choice([0.0, rng.uniform(0.0, 0.2)])),
                decay=_log_uniform(rng, 0.05, 3.0), sustain=float(rng.uniform(0, 1)),
                release=_log_uniform(rng, 0.02, 2.5),
                cutoff=_log_uniform(rng, 150, 12000) if rng.uniform() < 0.75 else NO_FILTER_HZ,
                fileg_depth=0.0, fileg_decay=0.0, fileg_sustain=0.0, lfo_depth=0.0,
                loop=bool(rng.uniform() < 0.4), sample_seconds=frames / RATE)
            opcodes = [f"sample={folder.name}/s{s:02d}.wav", f"lokey={region.lokey}", f"hikey={region.hikey}",
                       f"pitch_keycenter={region.center}", f"lovel={region.lovel}", f"hivel={region.hivel}",
                       f"ampeg_attack={region.attack:.4f}", f"ampeg_hold={region.hold:.4f}",
                       f"ampeg_decay={region.decay:.4f}", f"ampeg_sustain={100 * region.sustain:.2f}",
                       f"ampeg_release={region.release:.4f}"]
            if region.cutoff != NO_FILTER_HZ:
                region.fileg_depth = float(rng.uniform(-2400, 2400))
                region.fileg_decay = _log_uniform(rng, 0.05, 2.0)
                region.fileg_sustain = float(rng.uniform(0, 1))
                region.lfo_depth = float(rng.uniform(0, 1200)) if rng.uniform() < 0.5 else 0.0
                opcodes += ["fil_type=lpf_2p", f"cutoff={region.cutoff:.1f}",
                            f"fileg_depth={int(region.fileg_depth)}", f"fileg_decay={region.fileg_decay:.4f}",
                            f"fileg_sustain={100 * region.fileg_sustain:.2f}",
                            f"lfo1_cutoff={int(region.lfo_depth)}"]
                region.fileg_depth = float(int(region.fileg_depth))
                region.lfo_depth = float(int(region.lfo_depth))
            if region.loop:
                first = int(rng.integers(frames // 4, frames // 2))
                opcodes += ["loop_mode=loop_continuous", f"loop_start={first}",
                            f"loop_end={frames - 1 - int(rng.integers(0, frames // 8))}"]
            else:
                opcodes.append("loop_mode=no_loop")
            regions.append(region)
            lines.append("<region> " + " ".join(opcodes) + "\n")
    sfz = root / f"{name}.sfz"
    sfz.write_text("".join(lines), encoding="ascii")
    return sfz, regions


def _region_for(regions: list[Region], key: int, velocity: int) -> Region:
    for r in regions:
        if r.lokey <= key <= r.hikey and r.lovel <= velocity <= r.hivel:
            return r
    raise ValueError(f"no region for key {key} velocity {velocity}")


def preset_regions(sfz: Path, sample_seconds: float) -> list[Region]:
    """Regions of a generated plain-batch preset (workload.write_plain_batch_preset): its
    <global> envelope and filter opcodes, each region's key, velocity range, cutoff,
    filter-envelope depth, LFO depth and loop mode."""
    glob, regions = {}, []
    for line in Path(sfz).read_text().splitlines():
        fields = dict(tok.split("=", 1) for tok in line.split()[1:] if "=" in tok)
        if line.startswith("<global>"):
            glob = fields
        elif line.startswith("<region>"):
            o = {**glob, **fields}
            key = int(o["key"])
            regions.append(Region(
                lokey=key, hikey=key, lovel=int(o["lovel"]), hivel=int(o["hivel"]), center=key,
                attack=float(o.get("ampeg_attack", 0)), hold=float(o.get("ampeg_hold", 0)),
                decay=float(o.get("ampeg_decay", 0)), sustain=float(o.get("ampeg_sustain", 100)) / 100,
                release=float(o.get("ampeg_release", 0)),
                cutoff=float(o["cutoff"]) if "cutoff" in o else NO_FILTER_HZ,
                fileg_depth=float(o.get("fileg_depth", 0)), fileg_decay=float(o.get("fileg_decay", 0)),
                fileg_sustain=float(o.get("fileg_sustain", 100)) / 100,
                lfo_depth=float(o.get("lfo1_cutoff", 0)), loop=o.get("loop_mode") == "loop_continuous",
                sample_seconds=sample_seconds))
    return regions


def write_training_jobs(root: Path, seed: int, jobs: int, notes: int, instruments: int = 4,
                        kits: list[tuple[Path, list[Region]]] | None = None, velocities: tuple[int, int] = (1, 127),
                        name: str = "train") -> list[TrainingJob]:
    """`jobs` MIDI files of `notes` isolated notes each: every note starts after the previous
    one's release has ended, so each stretch of a job's render is one single-note render.
    The instruments are `kits` ((sfz, regions) pairs), else `instruments` random ones."""
    rng = np.random.default_rng(seed)
    if kits is None:
        kits = [write_training_instrument(root, seed * 1000 + i, f"train{i}") for i in range(instruments)]
    out = []
    for j in range(jobs):
        sfz, regions = kits[j % len(kits)]
        job = TrainingJob(sfz=sfz, midi=root / f"{name}_{j:05d}.mid")
        onset = 0.05
        keys = sorted({k for r in regions for k in range(r.lokey, r.hikey + 1)})
        for _ in range(notes):
            key = int(rng.choice(keys))
            velocity = int(rng.integers(velocities[0], velocities[1] + 1))
            held = _log_uniform(rng, 0.05, 3.0)
            region = _region_for(regions, key, velocity)
            job.notes.append(Note(onset, held, key, velocity, region))
            onset += held + 1.1 * region.release + 0.15
        workload._note_midi([(n.onset, n.held, n.key, n.velocity) for n in job.notes], [], onset, job.midi)
        out.append(job)
    return out


def features_of(note: Note) -> np.ndarray:
    r = note.region
    lg = lambda s: math.log(max(s, 1e-3))  # noqa: E731
    return np.array([lg(r.attack), lg(r.hold), lg(r.decay), r.sustain, lg(r.release), note.velocity / 127.0,
                     note.key / 127.0, math.log2(r.cutoff), r.fileg_depth / 2400.0, lg(r.sample_seconds),
                     float(r.loop), r.lfo_depth / 1200.0, lg(note.held), (note.key - r.center) / 12.0,
                     lg(r.fileg_decay), r.fileg_sustain], np.float32)


def note_windows(plan, count: int) -> np.ndarray | None:
    """Frame windows of a training job's notes: its spans merged into disjoint runs.
    None when the runs do not come out one per note."""
    spans = np.sort(plan.spans[["begin", "end"]], order="begin")
    runs = []
    for begin, end in zip(spans["begin"].astype(np.int64), spans["end"].astype(np.int64)):
        if runs and begin <= runs[-1][1]:
            runs[-1][1] = max(runs[-1][1], end)
        else:
            runs.append([begin, end])
    return np.array(runs, np.int64) if len(runs) == count else None


def render_training_set(root: Path, seed: int = 11, jobs: int = 512, notes: int = 64, batch_jobs: int = 128,
                        device: str = "cuda:0", host=None, renderer=None, instruments: int = 4, kits=None,
                        velocities: tuple[int, int] = (1, 127), name: str = "train"):
    """Features and targets of single-note renders made by the renderer (natural mode).

    Returns (features (n, 16), targets (n, 2), planned frames of each note's spans,
    index of each note's job)."""
    from .host import Host
    from .renderer import Renderer
    own_host, own_renderer = host is None, renderer is None
    host = host or Host()
    specs = write_training_jobs(root, seed, jobs, notes, instruments, kits, velocities, name)
    plans, kept, job_of = [], [], []
    for index, spec in enumerate(specs):
        plan = host.plan(spec.sfz, spec.midi, tail="natural")
        windows = note_windows(plan, len(spec.notes))
        if windows is not None:
            plans.append(plan)
            kept.append((spec, windows))
            job_of.extend([index] * len(spec.notes))
    renderer = renderer or Renderer(device=int(str(device).split(":")[-1]), natural=True)
    renderer.upload_samples(host.bank())
    feats, targets, span_frames = [], [], []
    lib = library()
    for lo in range(0, len(plans), batch_jobs):
        chunk = plans[lo:lo + batch_jobs]
        prepared = renderer.prepare(chunk)
        prepared.run()
        pointer, nbytes = ctypes.c_void_p(), ctypes.c_size_t()
        _check(lib.cs_prepared_mix_device(prepared.handle, ctypes.byref(pointer), ctypes.byref(nbytes)))
        import torch
        torch.cuda.synchronize(device)
        base, windows = 0, []
        for plan, (spec, runs) in zip(chunk, kept[lo:lo + batch_jobs]):
            windows.append(runs + base)
            base += plan.frames
            feats.extend(features_of(n) for n in spec.notes)
            span_frames.extend((runs[:, 1] - runs[:, 0]).tolist())
        peak, last = note_labels(pointer.value, np.concatenate(windows), device)
        targets.append(targets_from_labels(peak, last))
        prepared.close()
    if own_renderer:
        renderer.close()
    if own_host:
        host.close()
    return (np.array(feats, np.float32), np.concatenate(targets), np.array(span_frames, np.int64),
            np.array(job_of, np.int64))


# ---- the plain estimate and admission --------------------------------------------------

def envelope_estimate(features: np.ndarray) -> np.ndarray:
    """The method without the network: the planner's own bound on a note's render length
    (held time plus the release to -80 dB and its 50 ms fade, cut at the end of an
    unlooped sample), as log frames; the peak estimate is the velocity gain in dBFS."""
    f = np.asarray(features, np.float64)
    held = np.exp(f[:, 12])
    release = np.exp(f[:, 4])
    sample = np.exp(f[:, 9]) / np.exp2(f[:, 13])     # source length in output seconds
    length = held + release * math.log(1e4) / 9 + 0.05
    length = np.where(f[:, 10] > 0.5, length, np.minimum(length, sample))
    velocity = np.maximum(f[:, 5], 1 / 127)
    return np.stack([np.log(np.maximum(length * RATE, 1)), 40 * np.log10(velocity)], axis=1)


def calibrate_margin(predicted_log: np.ndarray, true_log: np.ndarray, mispredict_rate: float = 0.01) -> float:
    """Log-frame margin above the prediction that covers all but `mispredict_rate` of the
    calibration notes (a quantile of their residuals)."""
    residual = np.asarray(true_log, np.float64) - np.asarray(predicted_log, np.float64)
    return float(np.quantile(residual, 1.0 - mispredict_rate))


def admission_reservation(predicted_log: np.ndarray, plain_log: np.ndarray, margin_log: float) -> np.ndarray:
    """Frames reserved per note: the prediction raised by the calibrated margin, never more
    than the plain estimate (the planner's bound on the note's render length)."""
    predicted = np.exp(np.asarray(predicted_log, np.float64) + margin_log)
    return np.ceil(np.minimum(predicted, np.exp(np.asarray(plain_log, np.float64)))).astype(np.int64)
