"""Throughput of the batch voice-render path: audio-seconds rendered per second.

Workload (default, `--workload uneven`): the batching configuration — 1024 jobs
over four presets of 12 mono 16-bit regions (keys up to four semitones from each
keycenter, so most voices run the 48-tap sinc resampler), no filter, Pareto(1.5)
lengths from 2 to 600 s — generated from a seed (the reference's sample libraries
and MIDI corpora are not redistributable) and planned by this package's C++ host.
`--workload plain_batch` renders instead the 64-job filtered batch: one preset of
88 keys x 4 velocity layers of stereo 24-bit samples (half looping), lpf_2p with a
+-2400 cent filter envelope and a 5 Hz LFO on the cutoff, MIDI lengths
log-uniform 10-180 s at Poisson 4 notes/s with sustain-pedal toggles.

A step renders the whole batch: synthesis (sources, filter recurrences, mix) and
natural-tail finishing to packed mono PCM16.  `value` times steps on inputs that
are already resident in device memory (each step writes a float mix of gigabytes,
well above the 126 MB L2, which evicts it between steps, so no flush is needed);
`e2e` times the public render_window call with the plans in host memory,
including the plan upload and the PCM download, in GPU batches (the CLI's
--gpu-batch-jobs) whose size the autotuner (claysampler_b200/autotune.py)
measured fastest for the workload.  Under torchrun every rank renders its own
batch (no collective), so scaling is weak.

`cpu_baseline` and `parity` (one rank): the first jobs of the workload planned by
the reference's own planner and rendered by the reference's render.cu built for
the host (oracle/_ref, all cores) with the oracle's tail.cu restatement; the GPU
renders the same reference plans, and `parity` compares that render with the
reference's own render.cu kernels run on the same GPU (oracle/ref/ref_gpu.cu) and
with the host build.

`--learned` trains and scores the note-lifetime predictor.  `--serve` measures
the submit-to-publish latency of requests that arrive one at a time (Poisson)
through the non-blocking submit / poll pair.

`--impl reference` times the reference's own CPU implementation of the path
(its planner and src/cuda/render.cu built for the host, see oracle/ref) on a
bounded sample of the same workload, with the same `config`.
"""
from __future__ import annotations

import argparse
import contextlib
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

RATE = 44100
METRIC = "audio-sec/sec on 1 B200 (batched+learned vs plain, ≤1 LSB); HBM GB/s; p99"
WORKLOAD = "plain batch: {jobs} jobs, 88 keys x 4 layers stereo 24-bit, lpf_2p + fileg + 5 Hz LFO, loops, pedal"
WORKLOADS = {
    "plain_batch": WORKLOAD,
    "uneven": "uneven batch: {jobs} jobs over 4 presets of 12 mono 16-bit regions (48-tap sinc resampling, "
              "no filter), Pareto(1.5) lengths 2-600 s",
    "uneven_hbm": "uneven batch with an HBM-resident bank: {jobs} jobs over 4 presets of 22 keycenters x 8 "
                  "velocity layers x 48 s mono (about 6 GB of float samples), Pareto(1.5) lengths 2-600 s",
}
# Jobs of the bounded CPU sample (the reference arm's step and the cpu_baseline /
# parity leg): about 1-6 s of the reference's host render on 16 cores.
CPU_SAMPLE_JOBS = {"plain_batch": 16, "uneven": 128, "uneven_hbm": 64}


def parse():
    p = argparse.ArgumentParser(description=__doc__)
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["b200", "reference"], default="b200")
    p.add_argument("--workload", choices=sorted(WORKLOADS), default="uneven",
                   help="uneven: 1024 Pareto-length jobs (the batching configuration); plain_batch: the 64-job "
                        "filtered batch")
    p.add_argument("--jobs", type=int, default=None, help="jobs per rank (default 64, or 1024 for uneven)")
    p.add_argument("--seed", type=int, default=2)
    p.add_argument("--cpu-sample-jobs", type=int, default=None,
                   help="jobs of the bounded CPU sample (default: 128 for uneven, 16 for plain_batch)")
    p.add_argument("--workdir", type=Path, default=Path(tempfile.gettempdir()) / "claysampler_bench")
    p.add_argument("--e2e-batch-jobs", type=int, default=32,
                   help="GPU batch size of the end-to-end pass (the CLI's --gpu-batch-jobs): two batches in "
                        "flight overlap one's upload and download with the other's kernels")
    p.add_argument("--no-autotune", action="store_true",
                   help="skip the GPU batch-size sweep and use --e2e-batch-jobs for the end-to-end pass")
    p.add_argument("--device-only", action="store_true",
                   help="time only the device step of the batched form (no plain comparison, end-to-end pass or "
                        "CPU baseline): the command the committed ncu launch lists run")
    p.add_argument("--serve", action="store_true",
                   help="serving run instead: Poisson arrivals through cs_submit / cs_poll, job latency")
    p.add_argument("--learned", action="store_true",
                   help="train the note-lifetime predictor on single-note renders and report it")
    p.add_argument("--learned-jobs", type=int, default=2048, help="training jobs of 64 isolated notes each")
    p.add_argument("--learned-epochs", type=int, default=30)
    p.add_argument("--learned-preset-jobs", type=int, default=320,
                   help="jobs of 64 isolated notes of the 64-job batch's preset (80 % train, 20 % held out)")
    p.add_argument("--learned-mispredict", type=float, default=0.01,
                   help="mispredict rate the reservation margin is calibrated to on the training notes")
    p.add_argument("--serve-jobs", type=int, default=3000, help="requests (3000 at 50/s: a minute of arrivals)")
    p.add_argument("--serve-rate", type=float, default=50.0)
    p.add_argument("--serve-lanes", type=int, default=4, help="batches in flight (cs_renderer_set_lanes)")
    p.add_argument("--serve-batch", type=int, default=32, help="jobs per batch at most")
    p.add_argument("--serve-bank", choices=("small", "large"), default="small",
                   help="presets of the small kind, or of the HBM-bank kind (8 presets: about 12 GB of samples)")
    return p.parse_args()


def dist_info():
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    return rank, world, local


def workload(args, rank):
    from claysampler_b200 import workload as wl
    kind = getattr(args, "workload", "plain_batch")
    if args.jobs is None:
        args.jobs = 1024 if kind.startswith("uneven") else 64
    root = args.workdir / f"{kind}_s{args.seed + rank}_j{args.jobs}"
    marker = root / "ready"
    if not marker.exists():
        if kind == "uneven":
            jobs = wl.write_uneven_batch(root, seed=args.seed + rank, jobs=args.jobs)
        elif kind == "uneven_hbm":
            jobs = wl.write_uneven_hbm_batch(root, seed=args.seed + rank, jobs=args.jobs)
        else:
            jobs = wl.write_plain_batch(root, seed=args.seed + rank, jobs=args.jobs)
        marker.write_text("\n".join(f"{j.sfz}\t{j.midi}" for j in jobs))
    return [tuple(map(Path, line.split("\t"))) for line in marker.read_text().splitlines()]


def pin_plans(plans):
    """Moves the plans' span, point and binding arrays into one page-locked block
    (the end-to-end inputs come from pinned host memory); returns the block."""
    import torch
    fields = ("spans", "points", "modulation")
    total = sum((getattr(p, f).nbytes + 63) // 64 * 64 for p in plans for f in fields)
    block = torch.empty(max(total, 64), dtype=torch.uint8, pin_memory=True).numpy()
    at = 0
    for plan in plans:
        for f in fields:
            array = getattr(plan, f)
            view = block[at:at + array.nbytes].view(array.dtype).reshape(array.shape)
            view[...] = array
            setattr(plan, f, view)
            at += (array.nbytes + 63) // 64 * 64
    return block


def plan_jobs(jobs):
    from claysampler_b200.host import Host
    host = Host()
    plans = [host.plan(sfz, midi, tail="natural") for sfz, midi in jobs]
    bank = host.bank()
    host.close()
    return plans, bank


class ClockSampler:
    """SM clocks and clock-event (throttle) reasons sampled during the timed region:
    NVML read every 2 ms from a thread (read-only queries), else nvidia-smi."""
    FIELDS = ("clocks.sm,clocks.max.sm,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")
    NAMES = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.nvml = None
        self.lines = []
        self.samples = []               # (sm MHz, max MHz, reasons) from NVML
        self.stop = threading.Event()

    def _nvml_handle(self):
        import pynvml
        import torch
        pynvml.nvmlInit()
        try:
            uuid = str(torch.cuda.get_device_properties(self.index).uuid)
            return pynvml, pynvml.nvmlDeviceGetHandleByUUID(uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.index)

    def _nvml_sample(self):
        pynvml, handle = self.nvml
        sm = pynvml.nvmlDeviceGetClockInfo(handle, pynvml.NVML_CLOCK_SM)
        top = pynvml.nvmlDeviceGetMaxClockInfo(handle, pynvml.NVML_CLOCK_SM)
        bits = pynvml.nvmlDeviceGetCurrentClocksEventReasons(handle)
        flags = (pynvml.nvmlClocksEventReasonHwSlowdown, pynvml.nvmlClocksEventReasonHwThermalSlowdown,
                 pynvml.nvmlClocksEventReasonSwThermalSlowdown, pynvml.nvmlClocksEventReasonSwPowerCap)
        self.samples.append((float(sm), float(top), {n for n, f in zip(self.NAMES, flags) if bits & f}))

    def _nvml_loop(self):
        while not self.stop.is_set():
            try:
                self._nvml_sample()
            except Exception:
                return
            time.sleep(0.002)

    def __enter__(self):
        try:
            self.nvml = self._nvml_handle()
            self._nvml_sample()
            self.samples.clear()
            self.thread = threading.Thread(target=self._nvml_loop, daemon=True)
            self.thread.start()
            return self
        except Exception:
            self.nvml = None
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "50", "-i", str(self.index)],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            # nvidia-smi takes a moment to start: wait for its first sample, then keep
            # only the samples taken from here on (the timed region follows).
            deadline = time.time() + 5
            while not self.lines and time.time() < deadline and self.proc.poll() is None:
                time.sleep(0.01)
            self.lines.clear()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.nvml:
            self.stop.set()
            self.thread.join(timeout=1)
            if not self.samples:        # a region shorter than one period: read once at its end
                try:
                    self._nvml_sample()
                except Exception:
                    pass
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, top, reasons = [], 0.0, set()
        for clock, peak, active in self.samples:
            sm.append(clock)
            top = max(top, peak)
            reasons |= active
        for line in self.lines:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                top = max(top, float(parts[1]))
            except ValueError:
                continue
            for name, flag in zip(self.NAMES, parts[3:7]):
                if flag.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": top or None,
                "reasons": sorted(reasons), "samples": len(sm),
                "source": "nvml" if self.nvml else "nvidia-smi"}


def gather_rows(totals, world):
    """Every rank's row of per-rank figures (a 1-D tensor on the process group's
    device), as a (world, fields) array on every rank."""
    import torch
    if world == 1:
        return totals.cpu().numpy()[None]
    gathered = [torch.zeros_like(totals) for _ in range(world)]
    torch.distributed.all_gather(gathered, totals)
    return torch.stack(gathered).cpu().numpy()


def combine(rows):
    """Whole-job figures from per-rank rows (audio-s, device ms per step, e2e s per
    step, e2e audio-s): audio summed over ranks, times the max over ranks."""
    return float(rows[:, 0].sum()), float(rows[:, 1].max()), float(rows[:, 2].max()), float(rows[:, 3].sum())


def algorithmic_bytes(plans):
    """Bytes each stage must move per launch (source samples read once at the voice's
    step, scratch written/read once, mix written once), from the plans."""
    src = rec = mix = 0.0
    for p in plans:
        s = p.spans
        frames = (s["end"].astype(np.int64) - s["begin"]).astype(np.float64)
        ch = s["channels"].astype(np.float64)
        step = np.maximum(1.0, np.abs(s["step"]))
        chain = s["filterTrack"] >= 0
        filtered = (s["filters"]["type"] != 0).any(axis=1)
        moving = (s["activeEnvelope"][:, 0] != 0) if len(s) else np.zeros(0, bool)
        bank = frames * ch * 4 * step
        src += float(np.sum((bank + frames * ch * 4 + np.where(filtered & moving, frames * 12, 0))[chain]))
        rec += float(np.sum((frames * ch * 8 + np.where(moving, frames * 12, 0))[chain & filtered]))
        mix += float(np.sum(np.where(chain, frames * ch * 4, bank))) + p.frames * 8
    return {"source": src, "recurrence": rec, "mix": mix}


def sinc_flops(plans):
    """FP32 flops of the 48-tap sinc MACs per launch of each stage: 2 * 48 * channels per
    voice-frame of a span whose step is not 1 (at step 1 every position is a whole
    frame and the MAC loop does not run), counted where the span is rendered (chains
    in the source stage, the rest inline in the mix)."""
    src = mix = 0.0
    for p in plans:
        s = p.spans
        frames = (s["end"].astype(np.int64) - s["begin"]).astype(np.float64)
        ch = s["channels"].astype(np.float64)
        sinc = (s["step"] != 1.0) | (s["pitchSlope"] != 0) | (s["variablePitch"] != 0)
        chain = s["filterTrack"] >= 0
        flops = np.where(sinc, frames * ch * 96.0, 0.0)
        src += float(np.sum(flops[chain]))
        mix += float(np.sum(flops[~chain]))
    return {"source": src, "mix": mix}


def simt_fp32_tflops(sm_mhz):
    """FP32 FMA peak of the 148 SMs (128 lanes each, 2 flops per FMA) at `sm_mhz`."""
    return 2 * 128 * 148 * sm_mhz * 1e6 / 1e12


def measured_peaks():
    path = ROOT / "MEASURED_PEAKS.json"
    if path.exists():
        peaks = json.loads(path.read_text())
        return float(peaks["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def traffic_per_unit(workload_name: str) -> dict:
    """DRAM bytes per voice-frame per kernel for `workload_name` from the committed
    ncu summary (rows: workload, kernel, bytes per voice-frame, algorithmic bytes)."""
    path = ROOT / "profiles" / "dram_traffic.txt"
    table = {}
    if path.exists():
        for line in path.read_text().splitlines():
            parts = line.split()
            if len(parts) >= 3 and not line.startswith("#") and parts[0] == workload_name:
                try:
                    table[parts[1]] = float(parts[2])
                except ValueError:
                    pass
    return table


def sample_jobs(args):
    """The bounded CPU sample: the first jobs of the workload (jobs are drawn
    independently, so a prefix is an unbiased sample of the lengths)."""
    if args.cpu_sample_jobs is None:
        args.cpu_sample_jobs = CPU_SAMPLE_JOBS.get(args.workload, 32)
    return args.cpu_sample_jobs


def bench_config(args, jobs, ranks):
    """The `config` object of the bench line, identical in both arms."""
    return {"workload": WORKLOADS[args.workload].format(jobs=len(jobs)), "jobs_per_gpu": len(jobs), "seed": args.seed, "tail": "natural",
            "taps": 48, "l2": "each step writes a float mix above the 126 MB L2, evicting it (no flush)",
            "parallelism": f"jobs sharded by rank, {ranks} rank(s)"}


def reference_render(jobs, threads):
    """The reference end to end on the host: its own planner (oracle/_ref, the
    reference's plan.cpp / instrument.cpp / midi.cpp / audio.cpp) plans `jobs`, its
    render.cu built for the host renders them on `threads` cores and the oracle's
    restatement of tail.cu finishes them.  Returns (plans, bank, render) where
    render() times one pass and returns (seconds, pcm, results, mix)."""
    from oracle import oracle, reference
    if not reference.available():
        reference.build()
    if not reference.available():
        raise RuntimeError("the reference is not built for the host (oracle/_ref)")
    session = reference.RefSession()
    plans = [session.plan(sfz, midi, tail="natural") for sfz, midi in jobs]
    bank = session.bank()
    session.close()

    def render():
        start = time.perf_counter()
        mix = reference.synthesize(plans, bank, True, threads)
        pcm, results = oracle.finish(mix, plans)
        return time.perf_counter() - start, pcm, results, mix
    return plans, bank, render


def cpu_baseline(jobs, sample_jobs, host_plans, host_bank, renderer):
    """The reference on the host cores (its planner and its render.cu built for the
    host, all cores) over the first `sample_jobs` jobs, and the parity of this
    package on the same jobs: its planner's plans byte for byte against the
    reference planner's, and the GPU render of the reference's plans against the
    reference's own render.cu kernels on this GPU (the oracle the contract names)
    and against its host build (float bus error in full scale, PCM16 LSBs,
    statuses and frames)."""
    threads = os.cpu_count() or 1
    sample = jobs[:sample_jobs]
    plans, bank, render = reference_render(sample, threads)
    seconds, pcm, results, mix = render()
    audio = float(results["frames"].sum()) / RATE
    baseline = {"value": audio / seconds, "unit": "audio-s/s", "cores": threads, "kind": "reference",
                "sample": f"first {len(sample)} of {len(jobs)} jobs ({audio:.1f} output audio-s), natural tail, "
                          "planned by the reference planner"}
    prepared = renderer.prepare(plans)
    try:
        prepared.run()
        gpu_pcm, gpu_results = prepared.collect()
        gpu_mix = prepared.mix()
    finally:
        prepared.close()
    same_plans = all(a.to_blob() == b.to_blob() for a, b in zip(host_plans[:len(plans)], plans))
    # The renderer holds this package's bank; the reference plans index the
    # reference's, which must be the same floats.
    same_plans = same_plans and bank.size <= host_bank.size and np.array_equal(bank, host_bank[:bank.size])

    def agreement(ref_mix, ref_pcm, ref_results):
        diff = np.abs(gpu_pcm.astype(np.int32) - ref_pcm.astype(np.int32)) if gpu_pcm.shape == ref_pcm.shape else None
        out = {"max_bus_error_fs": float(np.max(np.abs(gpu_mix - ref_mix))) if gpu_mix.shape == ref_mix.shape else None,
               "bus_bit_identical": bool(gpu_mix.shape == ref_mix.shape
                                         and np.array_equal(gpu_mix.view(np.uint32), ref_mix.view(np.uint32))),
               "max_lsb": int(diff.max(initial=0)) if diff is not None else None,
               "identical_fraction": float(np.mean(diff == 0)) if diff is not None and diff.size else None,
               "statuses_equal": bool(np.array_equal(gpu_results["status"], ref_results["status"])),
               "frames_equal": bool(np.array_equal(gpu_results["frames"], ref_results["frames"]))}
        out["ok"] = bool(out["statuses_equal"] and out["frames_equal"] and out["max_bus_error_fs"] is not None
                         and out["max_bus_error_fs"] <= 1e-5 and out["max_lsb"] is not None and out["max_lsb"] <= 1
                         and (out["identical_fraction"] or 1.0) >= 0.999)
        return out

    host = agreement(mix, pcm, results)
    host["against"] = "the reference's render.cu built for the host (host libm, no FMA contraction)"
    parity = {"jobs": len(plans), "plans_identical": bool(same_plans),  # plans and sample bank
              "bounds": "bus <= 1e-5 FS, PCM16 <= 1 LSB with >= 99.9 % identical, statuses and frames exact",
              "host_reference": host}
    from oracle import oracle, reference
    if reference.gpu_available():
        ref_mix = reference.synthesize_gpu(plans, bank)
        ref_pcm, ref_results = oracle.finish(ref_mix, plans)
        device = agreement(ref_mix, ref_pcm, ref_results)
        device["against"] = "the reference's own render.cu kernels on this GPU (NVRTC defaults: FMA contraction)"
        parity["gpu_reference"] = device
        parity["ok"] = bool(same_plans and device["ok"])
    else:
        parity["ok"] = bool(same_plans and host["ok"])
    parity["finishing"] = "the oracle's restatement of tail.cu on the reference's mix"
    return baseline, parity


def reference_gpu(jobs, stage_ms, audio):
    """The reference's own synthesis kernels (its render.cu built for this GPU with
    the NVRTC defaults, launched as its renderer launches them for one segment) on
    every job of the workload, planned by the reference planner: device time of the
    synthesis launches against this package's synthesis stages on the same jobs
    (finishing excluded on both sides)."""
    from oracle import reference
    if not reference.gpu_available():
        raise RuntimeError("oracle/_ref/libclayref_gpu.so is not built")
    session = reference.RefSession()
    plans = [session.plan(sfz, midi, tail="natural") for sfz, midi in jobs]
    bank = session.bank()
    session.close()
    ms = reference.time_gpu(plans, bank, repeats=3)
    ours = sum(v for k, v in stage_ms.items() if k not in ("finish", "assess"))
    return {"synthesis_ms": ms, "ours_synthesis_ms": ours, "speedup": ms / ours if ours else None,
            "reference_audio_s_per_s": audio / (ms * 1e-3), "jobs": len(plans),
            "what": "src/cuda/render.cu kernels (pitch, filter sources, filters, tiles) on this GPU, "
                    "device time, one segment; ours: the shared-source, source, recurrence and mix stages"}


def run_reference(args):
    rank, world, _ = dist_info()
    if rank != 0:
        return
    jobs = workload(args, 0)
    sample = jobs[:sample_jobs(args)]
    threads = os.cpu_count() or 1
    try:
        plans, bank, render = reference_render(sample, threads)
    except Exception as error:  # no host build of the reference
        print(json.dumps({"impl": "reference", "unavailable": f"reference CPU path unavailable: {error}"}))
        return
    times, audio = [], 0.0
    for i in range(args.warmup + args.steps):
        elapsed, _, results, _ = render()
        audio = float(results["frames"].sum()) / RATE
        if i >= args.warmup:
            times.append(elapsed)
    mean = sum(times) / len(times)
    value = audio / mean
    out = {"metric": METRIC, "value": value, "unit": "audio-s/s", "n_gpus": args.gpus, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": mean * 1e3, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded SFZ/WAV/MIDI)", "impl": "reference",
           "config": bench_config(args, jobs, args.gpus),
           "cpu_baseline": {"value": value, "unit": "audio-s/s", "cores": threads, "kind": "reference",
                            "sample": f"first {len(sample)} of {len(jobs)} jobs per step ({audio:.1f} output "
                                      "audio-s), planned by the reference planner"},
           "e2e": {"value": value, "unit": "audio-s/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out))


def run_b200(args):
    import torch
    rank, world, local = dist_info()
    distributed = world > 1
    if distributed:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    torch.cuda.set_device(local)
    from claysampler_b200.plans import PlanSet
    from claysampler_b200.renderer import Renderer

    jobs = workload(args, rank)
    plans, bank = plan_jobs(jobs)
    for plan in plans:                  # inputs in page-locked host memory
        plan.pin()
    renderer = Renderer(device=local, natural=True, batch_jobs=len(plans))
    renderer.upload_samples(bank)
    stream = torch.cuda.Stream()          # a real stream: handle 0 would mean the renderer's own

    def barrier():
        if distributed:
            torch.distributed.barrier()

    def timed(prepared, clocks=None):
        """Warm-up steps, then `steps` steps each bracketed by CUDA events on the
        launching stream; per-stage device times summed over the steps."""
        for _ in range(args.warmup):
            prepared.run(stream.cuda_stream)
        torch.cuda.synchronize()
        totals, step_ms = {}, []
        with (clocks or contextlib.nullcontext()):
            barrier()
            torch.cuda.synchronize()
            for _ in range(args.steps):
                start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                start.record(stream)
                prepared.run(stream.cuda_stream)
                end.record(stream)
                end.synchronize()
                step_ms.append(start.elapsed_time(end))
                for name, stage in prepared.stage_ms().items():
                    totals[name] = totals.get(name, 0.0) + stage
            barrier()
            torch.cuda.synchronize()
        return sum(step_ms) / len(step_ms), totals

    # The plain path first: every voice frame resampled inline.
    plain_ms, plain_totals = float("nan"), {}
    if not args.device_only:
        renderer.set_shared_sources(False)
        plain = renderer.prepare(plans)
        plain.set_profile(True)
        plain_ms, plain_totals = timed(plain)
        plain.close()
    # The batched form: each voice source shared by several voices of the batch
    # rendered once (bit-identical audio).
    renderer.set_shared_sources(True)
    prepared = renderer.prepare(plans)
    prepared.set_profile(True)
    shared_info = prepared.shared
    clocks = ClockSampler(local)
    ms, stage_totals = timed(prepared, clocks)
    _, results = prepared.collect()
    audio = float(results["frames"].sum()) / RATE
    statuses = np.bincount(results["status"], minlength=12).tolist()
    launches = prepared.launches * args.steps
    if args.device_only:
        if rank == 0:
            print(json.dumps({"metric": METRIC, "device_only": True, "value": audio / (ms * 1e-3), "unit": "audio-s/s",
                              "ms_per_step": ms, "steps": args.steps, "warmup": args.warmup,
                              "stage_ms": {k: v / args.steps for k, v in stage_totals.items()},
                              "config": bench_config(args, jobs, world), "gpu_launches": launches}))
        prepared.close()
        renderer.close()
        if distributed:
            torch.distributed.destroy_process_group()
        return

    # End to end through the public API: plans in host memory, PCM back to host, in
    # GPU batches of the size the autotuner measured fastest for this workload.
    # The caller's plans sit in page-locked memory and its plan array is built
    # once, as a C caller holds its cs_plan array.
    pinned_block = pin_plans(plans)
    plan_set = PlanSet(plans)
    e2e_batch = min(args.e2e_batch_jobs, len(plans)) if args.e2e_batch_jobs > 0 else len(plans)
    tuned = None
    if not getattr(args, "no_autotune", False):
        from claysampler_b200 import autotune
        tuned = autotune.tune(plan_set, bank, device=local, cache=args.workdir / "autotune.json")
        e2e_batch = tuned["batch_jobs"]
    e2e_renderer = Renderer(device=local, natural=True, batch_jobs=e2e_batch)
    if tuned:
        e2e_renderer.set_lanes(tuned["lanes"])
        e2e_renderer.set_shared_sources(tuned["shared_sources"])
        e2e_renderer.set_ordered_compute(tuned["ordered_compute"])
    e2e_renderer.upload_samples(bank)
    h2d = sum(p.spans.nbytes + p.points.nbytes + p.modulation.nbytes + p.track_offsets.nbytes for p in plans)
    box = {}

    def publish(batch, first):
        # The PCM arrives in the renderer's page-locked buffer (the device-to-host
        # read of the step's result); the callback reads it in place.
        box["pcm"] += batch.pcm.nbytes + batch.results.nbytes
        box["audio"] += float(batch.results["frames"].sum()) / RATE
        box["checksum"] += int(batch.pcm[::4096].astype(np.int64).sum())

    e2e_times, pass_phases = [], []
    for i in range(args.warmup + args.steps):
        barrier()
        torch.cuda.synchronize()
        box.update(pcm=0, audio=0.0, checksum=0)
        before = e2e_renderer.host_ms()
        start = time.perf_counter()
        e2e_renderer.render_window(plan_set, publish, copy=False)
        elapsed = time.perf_counter() - start
        after = e2e_renderer.host_ms()
        if i >= args.warmup:
            e2e_times.append(elapsed)
            pass_phases.append({k: round(after[k] - before[k], 2) for k in after})
    e2e_s = sum(e2e_times) / len(e2e_times)
    host_ms = {k: v / (args.warmup + args.steps) for k, v in e2e_renderer.host_ms().items()}

    totals = torch.tensor([audio, ms, e2e_s, box.get("audio", 0.0)], dtype=torch.float64, device="cuda")
    total_audio, max_ms, max_e2e, total_e2e_audio = combine(gather_rows(totals, world))

    if rank == 0:
        peak, peak_kind = measured_peaks()
        algorithmic = algorithmic_bytes(plans)
        flops = sinc_flops(plans)
        # Shared voice sources: their sinc MACs move from the mix to the shared
        # stage, which reads each source's samples once and writes it once.
        flops["mix"] -= 96.0 * shared_info["voice_sinc_floats"]
        flops["shared"] = 96.0 * shared_info["sinc_floats"]
        algorithmic["shared"] = 8.0 * shared_info["floats"]
        stage_ms = {k: v / args.steps for k, v in stage_totals.items()}
        candidates = {k: stage_ms.get(k, 0.0) for k in ("source", "recurrence", "mix", "shared")}
        dominant = max(candidates, key=candidates.get)
        achieved = algorithmic[dominant] / (stage_ms[dominant] * 1e-3) / 1e9
        per_unit = traffic_per_unit(args.workload)
        voice_frames = sum(p.voice_frames() for p in plans)
        traffic = per_unit[dominant] * voice_frames if dominant in per_unit else None
        clock = clocks.summary().get("sm_mhz") or 1965.0
        fp32_peak = simt_fp32_tflops(clock)
        fp32 = None
        if flops.get(dominant, 0.0) > 0 and stage_ms.get(dominant):
            rate = flops[dominant] / (stage_ms[dominant] * 1e-3) / 1e12
            fp32 = {"kernel": dominant, "achieved": rate, "peak": fp32_peak, "unit": "TFLOP/s",
                    "frac": rate / fp32_peak, "flops": flops[dominant],
                    "peak_kind": f"SIMT FP32 FMA peak at the sampled {clock:.0f} MHz"}
        roofline = {"bound": "hbm", "kernel": dominant, "achieved": achieved, "peak": peak, "peak_kind": peak_kind,
                    "unit": "GB/s", "frac": achieved / peak, "algorithmic_bytes": algorithmic[dominant],
                    "traffic": traffic, "fp32_sinc": fp32}
        # The binding roof of the dominant kernel is the one it is closest to.
        roofline["binding"] = "fp32" if fp32 and fp32["frac"] > roofline["frac"] else "hbm"
        # Every synthesis stage against both roofs.
        roofline["stages"] = {
            k: {"ms": stage_ms[k], "gbs": algorithmic.get(k, 0.0) / (stage_ms[k] * 1e-3) / 1e9,
                "hbm_frac": algorithmic.get(k, 0.0) / (stage_ms[k] * 1e-3) / 1e9 / peak,
                "sinc_tflops": flops.get(k, 0.0) / (stage_ms[k] * 1e-3) / 1e12,
                "fp32_frac": flops.get(k, 0.0) / (stage_ms[k] * 1e-3) / 1e12 / fp32_peak}
            for k in ("source", "recurrence", "mix", "shared") if stage_ms.get(k, 0.0) > 0.01}
        bank_mb = float(bank.nbytes) / 1e6
        out = {"metric": METRIC, "value": total_audio / (max_ms * 1e-3), "unit": "audio-s/s", "n_gpus": world,
               "steps": args.steps, "warmup": args.warmup, "ms_per_step": max_ms, "higher_is_better": True,
               "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded SFZ/WAV/MIDI)",
               "config": bench_config(args, jobs, world),
               "workload_stats": {"output_audio_s_per_gpu": audio, "voice_frames_per_gpu": voice_frames,
                                  "bank_mb": bank_mb, "statuses": statuses},
               "stage_ms": stage_ms, "roofline": roofline,
               "plain": {"value": audio / (plain_ms * 1e-3), "ms_per_step": plain_ms,
                         "stage_ms": {k: v / args.steps for k, v in plain_totals.items()},
                         "what": "every voice frame resampled inline (shared voice sources off)"},
               "batched_vs_plain": plain_ms / ms,
               "shared_sources": shared_info,
               "e2e": {"value": total_e2e_audio / max_e2e, "unit": "audio-s/s", "h2d_bytes_per_step": int(h2d),
                       "d2h_bytes_per_step": int(box.get("pcm", 0)), "ms_per_step": max_e2e * 1e3,
                       "batch_jobs": e2e_batch, "autotune": tuned, "host_staging_ms_per_step": host_ms,
                       "pass_ms": [round(t * 1e3, 2) for t in e2e_times],
                       "median_ms": round(statistics.median(e2e_times) * 1e3, 2),
                       "slowest_pass_host_ms": pass_phases[int(np.argmax(e2e_times))] if pass_phases else None},
               "gpu_launches": launches, "clocks": clocks.summary()}
        if world == 1:
            try:
                out["cpu_baseline"], out["parity"] = cpu_baseline(jobs, sample_jobs(args), plans, bank, renderer)
            except Exception as error:
                out["cpu_baseline"] = {"value": None, "unavailable": str(error)}
            try:
                out["reference_gpu"] = reference_gpu(jobs, stage_ms, audio)
            except Exception as error:
                out["reference_gpu"] = {"unavailable": str(error)}
        print(json.dumps(out))
    prepared.close()
    renderer.close()
    e2e_renderer.close()
    if distributed:
        torch.distributed.destroy_process_group()


def serving_requests(args, rank):
    """The serving workload's plans (planned on the host), arrival times in seconds
    and sample bank."""
    from claysampler_b200 import workload as wl
    from claysampler_b200.host import Host
    large = getattr(args, "serve_bank", "small") == "large"
    root = args.workdir / f"serving_s{args.seed + rank}_j{args.serve_jobs}_r{args.serve_rate:g}{'_large' if large else ''}"
    marker = root / "ready"
    if not marker.exists():
        jobs, arrivals = wl.write_serving_jobs(root, seed=args.seed + rank, jobs=args.serve_jobs, rate=args.serve_rate,
                                               large=large)
        marker.write_text("\n".join(f"{j.sfz}\t{j.midi}\t{float(t)!r}" for j, t in zip(jobs, arrivals)))
    rows = [line.split("\t") for line in marker.read_text().splitlines()]
    host = Host()
    plans = [host.plan(Path(sfz), Path(midi), tail="natural") for sfz, midi, _ in rows]
    arrivals = np.array([float(t) for _, _, t in rows])
    bank = host.bank()
    host.close()
    return plans, arrivals, bank


def run_serve(args):
    """Render requests of the small kind (log-uniform 5-300 s over 8 presets)
    arriving by a Poisson process, submitted one by one to a running renderer
    (cs_submit) and published by cs_poll: continuous batching.  Reports the
    submit-to-publish latency percentiles and the rendered audio-seconds per second;
    each request is planned beforehand (CPU work outside the GPU path)."""
    import torch
    from claysampler_b200.renderer import Renderer
    rank, world, local = dist_info()
    torch.cuda.set_device(local)
    plans, arrivals, bank = serving_requests(args, rank)
    plans = [p.pin() for p in plans]
    renderer = Renderer(device=local, natural=True, batch_jobs=args.serve_batch)
    renderer.set_lanes(args.serve_lanes)
    renderer.upload_samples(bank)
    done = {}

    def publish(batch, first):
        now = time.perf_counter()
        for k, r in enumerate(batch.results):
            done[first + k] = (now, float(r["frames"]) / RATE)

    warm = min(8, len(plans))                  # warm-up: kernels, arenas, page-locked buffers
    renderer.submit(plans[:warm])
    while renderer.pending_jobs:
        renderer.poll(publish, wait=True)
    done.clear()
    submitted = {}
    start = time.perf_counter()
    i = 0
    while i < len(plans) or renderer.pending_jobs:
        now = time.perf_counter() - start
        while i < len(plans) and arrivals[i] <= now:
            submitted[renderer.submit([plans[i]])] = time.perf_counter()
            i += 1
        if renderer.poll(publish, wait=i == len(plans)) == 0 and i < len(plans):
            time.sleep(max(0.0, min(0.001, arrivals[i] - (time.perf_counter() - start))))
    wall = time.perf_counter() - start
    latency = np.array([1e3 * (done[t][0] - submitted[t]) for t in submitted])
    audio = sum(done[t][1] for t in submitted)
    offered = float(np.sum([p.frames for p in plans]) / RATE / arrivals[-1])
    out = {"metric": "serving: submit-to-publish job latency, Poisson arrivals (continuous batching)",
           "value": float(np.percentile(latency, 99)), "unit": "ms", "higher_is_better": False,
           "p50_ms": float(np.percentile(latency, 50)), "p95_ms": float(np.percentile(latency, 95)),
           "p99_ms": float(np.percentile(latency, 99)), "throughput_audio_s_per_s": audio / wall,
           "offered_audio_s_per_s": offered, "jobs": len(submitted), "rate_jobs_per_s": args.serve_rate,
           "wall_s": wall, "n_gpus": 1, "dtype": "f32", "data": "synthetic (seeded SFZ/WAV/MIDI)",
           "deferred_launches": renderer.deferred_launches,
           "bank_gb": float(bank.nbytes) / 1e9,
           "config": {"workload": ("requests over 8 presets of the HBM-bank kind"
                                   if getattr(args, "serve_bank", "small") == "large" else
                                   "requests of the small kind over 8 presets") + ", lengths log-uniform 5-300 s",
                      "batch_jobs": args.serve_batch, "lanes": args.serve_lanes,
                      "publication": "as batches finish (cs_poll)",
                      "admission": "a batch launches while others run only if its estimated footprint fits in "
                                   "half of the free device memory"}}
    if rank == 0:
        print(json.dumps(out))
    renderer.close()


def run_learned(args):
    """The learned part end to end on one GPU: single-note renders by the renderer label
    a training set (audible frames at -90 dBFS and peak), the MLP is trained by the
    library's fused forward/backward + Adam kernels, and held-out notes compare its
    predictions and its lifetime reservation with the plain estimate (the planner's
    release bound, velocity gain).  The training notes are random regions of four
    instruments plus notes of the 64-job batch's preset; the held-out notes are the
    last 10 % of the random-region jobs and the last 20 % of the preset's jobs."""
    import torch
    from claysampler_b200 import lifetime
    from claysampler_b200 import workload as wl
    rank, world, local = dist_info()
    torch.cuda.set_device(local)
    device = f"cuda:{local}"
    root = args.workdir / f"learned_s{args.seed + rank}_j{args.learned_jobs}"
    root.mkdir(parents=True, exist_ok=True)
    t0 = time.perf_counter()
    features, targets, spans, job = lifetime.render_training_set(root, seed=args.seed + rank,
                                                                 jobs=args.learned_jobs, notes=64,
                                                                 batch_jobs=128, device=device)
    # Notes of the 64-job batch's preset (88 keys x 4 layers, stereo, loops, lpf_2p +
    # filter envelope + LFO), rendered alone in the same way.
    kit_root = root / "batch_preset"
    kit_root.mkdir(parents=True, exist_ok=True)
    kit_sfz = wl.write_plain_batch_preset(kit_root, seed=args.seed)
    kit = (kit_sfz, lifetime.preset_regions(kit_sfz, 4.0))
    bf, bt, bspans, bjob = lifetime.render_training_set(kit_root, seed=args.seed + 7, jobs=args.learned_preset_jobs,
                                                        notes=64, batch_jobs=64, device=device, kits=[kit],
                                                        velocities=(40, 120), name="batch")
    label_s = time.perf_counter() - t0
    cut = int(round(0.9 * args.learned_jobs))
    train, test = job < cut, job >= cut
    pcut = int(round(0.8 * args.learned_preset_jobs))
    ptrain, ptest = bjob < pcut, bjob >= pcut
    tf = np.concatenate([features[train], bf[ptrain]])
    tt = np.concatenate([targets[train], bt[ptrain]])
    net = lifetime.LifetimeNet(device=device, seed=args.seed)
    net.set_normalisation(lifetime.normalisation(tf, tt))
    net.train(tf[:4096], tt[:4096], epochs=1, batch=4096)   # warm-up
    net = lifetime.LifetimeNet(device=device, seed=args.seed)
    net.set_normalisation(lifetime.normalisation(tf, tt))
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    start.record()
    history = net.train(tf, tt, epochs=args.learned_epochs, batch=4096, rate=3e-3, decay=0.9)
    end.record()
    torch.cuda.synchronize()
    train_ms = start.elapsed_time(end)
    margin = lifetime.calibrate_margin(net.predict(tf).cpu().numpy()[:, 0], tt[:, 0], args.learned_mispredict)

    def score(feats, truth, rendered):
        predicted = net.predict(feats).cpu().numpy()
        plain = lifetime.envelope_estimate(feats)
        audible = np.exp(truth[:, 0]).round().astype(np.int64)
        reserve_net = lifetime.admission_reservation(predicted[:, 0], plain[:, 0], margin)
        reserve_plain = np.ceil(np.exp(plain[:, 0])).astype(np.int64)
        return {"notes": int(len(feats)),
                "mae_log_frames": {"network": float(np.abs(predicted[:, 0] - truth[:, 0]).mean()),
                                   "plain": float(np.abs(plain[:, 0] - truth[:, 0]).mean())},
                "mae_peak_db": {"network": float(np.abs(predicted[:, 1] - truth[:, 1]).mean()),
                                "plain": float(np.abs(plain[:, 1] - truth[:, 1]).mean())},
                "reserved_frames": {"network": int(reserve_net.sum()), "plain": int(reserve_plain.sum()),
                                    "audible": int(audible.sum()), "rendered_spans": int(rendered.sum())},
                "reservation_cut": float(1 - reserve_net.sum() / reserve_plain.sum()),
                "mispredict_rate": {"network": float(np.mean(audible > reserve_net)),
                                    "plain": float(np.mean(audible > reserve_plain))}}

    random_regions = score(features[test], targets[test], spans[test])
    batch_preset = score(bf[ptest], bt[ptest], bspans[ptest])
    out = {"metric": "learned note lifetime / peak: held-out mean absolute error and lifetime reservation",
           "value": random_regions["mae_log_frames"]["network"], "unit": "|log audible frames| error",
           "higher_is_better": False,
           "random_regions": random_regions, "batch_preset": batch_preset,
           "train_notes": int(len(tf)), "epochs": args.learned_epochs,
           "loss_first_last": [history[0], history[-1]],
           "train_ms": train_ms, "train_samples_per_s": 1e3 * args.learned_epochs * int(len(tf)) / train_ms,
           "label_render_s": label_s, "n_gpus": 1, "dtype": "bf16 weights, f32 accumulate",
           "data": "synthetic (seeded random regions and the batch preset, single-note MIDI)",
           "config": {"workload": "MLP 16-64-64-2 on single-note renders: 4 instruments x 88 random regions "
                                  "+ the 64-job batch's preset", "batch": 4096, "margin_log_frames": margin,
                      "calibrated_mispredict_rate": args.learned_mispredict,
                      "threshold_dbfs": lifetime.AUDIBLE_DBFS}}
    if rank == 0:
        print(json.dumps(out))


def main():
    args = parse()
    if args.learned:
        run_learned(args)
        return
    if args.serve:
        run_serve(args)
        return
    if args.impl == "reference":
        run_reference(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
