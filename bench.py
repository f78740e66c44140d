#!/usr/bin/env python
"""Benchmark: Lenia Mpixel-steps/s on one 1920x1080 world, 3 kernels R=24.

A step is one Lenia substep (multi-kernel FFT convolution, growth, Euler
step, clip) of the ``fft3_1080p`` workload (life_simulation_b200/workloads.py:
seeded uniform patches, exponential kernel core, growth mode 0). Units are
pixels x steps; ``value`` is whole-job Mpixel-steps/s.

* value: state resident in HBM; K steps, each bracketed by CUDA events on
  the launching stream, with a 256 MiB write between steps to flush the
  126 MB L2 (outside the events); time = sum of the step intervals, max over
  ranks. Under torchrun every rank steps its own world (replicas, no
  collective on the data path; weak scaling). Before the warm-up the launch
  shapes of the two passes are chosen under these same conditions
  (lenia_set_tuning; --keep-tuning keeps the setup autotuner's).
* e2e: the same metric through the C ABI with host buffers: every step
  copies its whole input field in from pinned host memory and its whole
  result out to pinned host memory. The copies run on their own streams
  through device staging buffers (lenia_upload_device / lenia_step /
  lenia_download_device on the step's stream), so a step overlaps the next
  input's copy and the previous result's copy; CUDA events from the first
  copy in to the last copy out. e2e.serial: lenia_upload, lenia_step,
  lenia_download in turn.
* roofline: the dominant kernel's algorithmic bytes per launch (HBM-bound
  figures of the spectral path, per pixel: column pass 4 + 2K + 4K, row
  growth pass 4K + 4 + 4 + 4) over its mean launch duration, timed by CUDA
  events around every launch over further flushed steps (events between
  launches serialise them, so the durations are upper bounds; the value
  region has none), against the measured copy bandwidth in
  MEASURED_PEAKS.json.
* cpu_baseline: the reference's own Lenia module and kernels compiled for
  the CPU (oracle/_ref), on a bounded row band of the same workload.
* accuracy_vs_fp64 (with the CPU leg): max and RMS |A_gpu - A_fp64| of 5
  steps of the workload, each from the GPU's field, against the FP64 oracle.
* adjoint: the gradient form on 32 worlds of 512x512 (K=2, R=16, growth
  mode 1, T=64, checkpoints every 8): device time of the forward rollout and of the
  backward (recomputation included), CUDA events on the launching stream
  with an L2 flush before each; ratio = backward / forward.
* sweep (one GPU): the 512-world sweep (128 each of 128^2, 256^2, 384x216,
  512^2; R 8..32), batched against the plain one-context-per-world loop;
  Mpixel-steps/s of both, the speed-up and the per-readback activity.
* tc (one GPU): 4096x4096, 3 kernels R=32, 64 steps per arithmetic of the
  column DFT stages (fp32 CUDA cores, fp16x3 / bf16x3 split-precision tensor
  cores); per-step device time, the column pass's HBM roofline and tensor
  FLOP rate (a radix-16 stage as a real 32x32 GEMM: 128 FLOP per point, x3
  hi/lo), and each one's max / RMS error against the FP64 oracle.
* cpu_baseline_fft_1024x512: the reference's own FFT path (85 passes per
  substep) compiled for the CPU, whole 1024x512 field, all host threads.
* library_fft_baseline: the same step from torch.fft (cuFFT) and torch ops
  in one CUDA graph, same flush protocol: a library comparator.
* published_config / published_direct_config: 1024x512, 3 kernels R=24 (FFT)
  and 1280x720, 1 kernel R=32 (direct) -- the two Lenia configurations the
  reference publishes times for (Apple M5 Max, README.md:47-48) -- timed the
  same way, beside those published figures.
* --impl reference: that CPU reference alone, as the reference arm.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Lenia Mpixel-steps/s (FFT, 3 kernels, 1080p)"
UNIT = "Mpixel-steps/s"
WORKLOAD = "fft3_1080p"
FALLBACK_HBM_GBS = 6650.0
# DRAM traffic per launch (dram__bytes_read.sum + dram__bytes_write.sum) of
# the step's kernels, as one ncu capture of this workload measured it, with
# the capture's command: written beside the ncu summaries when a capture is
# taken. Without it, roofline.traffic is null.
TRAFFIC_FILE = os.path.join(ROOT, "profiles", "ncu_dram_traffic.json")


def captured_traffic(kernel: str, workload: str):
    """(bytes per launch, source) from the capture file, or (None, None)."""
    try:
        d = json.load(open(TRAFFIC_FILE))
    except (OSError, ValueError):
        return None, None
    k = d.get("kernels", {}).get(kernel)
    if not k or d.get("workload") != workload:
        return None, None
    return int(k["dram_bytes_per_launch"]), f"ncu capture: {d.get('command')} ({d.get('note', '')})"


def parse_args():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--workload", default=WORKLOAD)
    ap.add_argument("--e2e-steps", type=int, default=None)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--mode", choices=["step", "sweep", "adjoint", "tc"], default="step",
                    help="step: the 1080p headline; sweep: the 512-world batched sweep; "
                         "adjoint: the gradient form alone; tc: 4096^2 with the column DFT stages "
                         "on FP32 CUDA cores vs split-precision tensor cores")
    ap.add_argument("--adjoint-reps", type=int, default=5)
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--no-library-baseline", action="store_true")
    ap.add_argument("--no-sweep", action="store_true", help="skip the 512-world sweep in the step line")
    ap.add_argument("--no-tc", action="store_true", help="skip the 4096^2 tensor-core comparison in the step line")
    ap.add_argument("--tc-variants", default=None,
                    help="--mode tc: comma-separated subset of fp32, fp16x3, bf16x3, fp16x3_tcgen05, bf16x3_tcgen05, "
                         "fp16x3_tcgen05_pipelined, bf16x3_tcgen05_pipelined")
    ap.add_argument("--tc-steps", type=int, default=64, help="--mode tc: timed steps per variant")
    ap.add_argument("--no-tc-error", action="store_true", help="--mode tc: skip the FP64 error check")
    ap.add_argument("--launch-shape", default=None,
                    help="columns,rows per CTA of the two passes, e.g. 4,4p (p: pipelined rows; "
                         "h after the columns: half-thread column pass); "
                         "skips the shape search")
    ap.add_argument("--keep-tuning", action="store_true",
                    help="keep the setup autotuner's launch shapes instead of choosing them under the "
                         "bench's own conditions (flushed L2) before the timed region")
    ap.add_argument("--plain-steps", type=int, default=10)
    return ap.parse_args()


def dist_env():
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled every 200 ms."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (OSError, FileNotFoundError):
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                self.rows.append(parts)

    def stop(self):
        if not self.proc:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.thread.join(timeout=2)
        if not self.rows:
            return None
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "", 1).isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "", 1).isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if r[5 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons, "samples": len(self.rows)}


def cpu_baseline_reference(params, w, h, init, seconds, band=64):
    """The compiled reference on a bounded row band; Mpixel-steps/s."""
    from oracle.lenia_oracle import RefLenia
    r = RefLenia(params, w, h)
    r.reset(2)
    r.set_initial_field(init)
    r.set_row_window(0, band)
    r.encode(0, 1)  # init + one sample step (warm-up)
    steps, t0 = 0, time.perf_counter()
    while True:
        r.encode(1 + steps, 1)
        steps += 1
        el = time.perf_counter() - t0
        if el >= seconds or steps >= 1000:
            break
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    conv = "direct convolution with kernels[0] (the reference falls back from convMode fft at a " \
           "non-power-of-two size, Lenia.cpp:245-269)"
    return {"value": w * band * steps / el / 1e6, "unit": UNIT, "cores": cores, "kind": "reference",
            "sample": f"rows 0..{band} of the {w}x{h} field, {steps} substeps in {el:.1f} s; {conv}"}


def cpu_baseline_port(params, w, h, init, seconds):
    """The oracle port (FP64, FFT convolution) when oracle/_ref is absent."""
    from oracle.lenia_oracle import OracleLenia
    o = OracleLenia(params, w, h, "f64")
    o.reset(2)
    o.set_initial_field(init)
    o.encode(0, 1)
    steps, t0 = 0, time.perf_counter()
    while True:
        o.encode(1 + steps, 1)
        steps += 1
        el = time.perf_counter() - t0
        if el >= seconds or steps >= 100:
            break
    return {"value": w * h * steps / el / 1e6, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"full {w}x{h} field, {steps} substeps in {el:.1f} s (FP64 oracle)"}


_FP32_PEAK = None


def fp32_peak_measured() -> dict:
    """The device's FP32 FMA peak measured by lenia_fp32_peak (scalar FFMA,
    the instruction the direct kernel issues; packed FFMA2 beside it)."""
    global _FP32_PEAK
    if _FP32_PEAK is None:
        import life_simulation_b200 as lb
        r = lb.fp32_peak(5)
        r["source"] = "measured (lenia_fp32_peak: 8 FMA chains per thread, 8 x 256 threads per SM)"
        _FP32_PEAK = r
    return _FP32_PEAK


def published_direct_bench(steps: int = 50, warmup: int = 5) -> dict:
    """The reference's published direct configuration: one kernel, R=32,
    1280x720 (README.md:47-48, 19.4 ms per frame on an Apple M5 Max, one
    substep per frame); the module's default kernel shell, seeded patches.
    Timed like the value region."""
    import torch

    import life_simulation_b200 as lb
    from life_simulation_b200 import workloads as wl

    w, h = 1280, 720
    m = lb.LeniaModule({"radius": 32, "convMode": "direct"}, w, h)
    m.reset(2)
    m.upload(wl.patches(w, h, 12, 96, seed=2))
    stream = torch.cuda.Stream()
    sh = stream.cuda_stream
    fp = m.frame_params(0)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    evs = []
    with torch.cuda.stream(stream):
        for i in range(warmup + steps):
            flush.zero_()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            m.step(fp, 1, sh)
            b.record(stream)
            if i >= warmup:
                evs.append((a, b))
    torch.cuda.synchronize()
    ms = float(np.mean([a.elapsed_time(b) for a, b in evs]))
    info = m.info()
    m.close()
    ref_ms = 19.4
    # FP32 roofline: 2 FLOP per nonzero tap + 12 for the growth map, per pixel.
    flops = (2 * info["direct_taps"] + 12) * w * h
    peak = fp32_peak_measured()
    tflops = flops / (ms / 1e3) / 1e12
    return {"workload": "direct, 1 kernel R=32, 1280x720 (the reference's published direct configuration)",
            "ms_per_step": ms, "value": w * h / (ms / 1e3) / 1e6, "unit": UNIT,
            "direct_tma": info["direct_tma"], "direct_split": info["direct_split"],
            "direct_outputs_per_thread": info["direct_outputs_per_thread"],
            "direct_rows_per_thread": info["direct_rows_per_thread"],
            "fp32": {"achieved_tflops": tflops, "peak_tflops": peak["ffma_tflops"],
                     "frac": tflops / peak["ffma_tflops"], "peak_source": peak["source"],
                     "algorithmic_flops_per_step": flops},
            "reference_published": {"ms_per_frame": ref_ms, "value": w * h / (ref_ms / 1e3) / 1e6,
                                    "hardware": "Apple M5 Max (Metal), README.md:47-48; not reproducible here"}}


def published_config_bench(steps: int = 100, warmup: int = 5) -> dict:
    """The one FFT configuration the reference publishes a number for:
    1024x512, 3 kernels, R=24 (README.md:47-48, 1.13 ms per frame on an Apple
    M5 Max through Metal, one substep per frame). Same timing as the value
    region (L2 flushed before each step, CUDA events, launch shapes as the
    setup autotuner picked them)."""
    import torch

    import life_simulation_b200 as lb
    from life_simulation_b200 import workloads as wl

    params, w, h, init = wl.workload("fft3_1024x512")
    m = lb.LeniaModule(params, w, h)
    m.reset(2)
    m.upload(init)
    stream = torch.cuda.Stream()
    sh = stream.cuda_stream
    fp = m.frame_params(0)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    evs = []
    with torch.cuda.stream(stream):
        for i in range(warmup + steps):
            flush.zero_()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            m.step(fp, 1, sh)
            b.record(stream)
            if i >= warmup:
                evs.append((a, b))
    torch.cuda.synchronize()
    ms = float(np.mean([a.elapsed_time(b) for a, b in evs]))
    m.close()
    ref_ms = 1.13
    return {"workload": "fft3_1024x512: 1024x512, 3 kernels R=24 (the reference's published FFT configuration)",
            "ms_per_step": ms, "value": w * h / (ms / 1e3) / 1e6, "unit": UNIT,
            "reference_published": {"ms_per_frame": ref_ms, "value": w * h / (ref_ms / 1e3) / 1e6,
                                    "hardware": "Apple M5 Max (Metal), README.md:47-48; not reproducible here"}}


def library_fft_baseline(params, w, h, init, steps: int = 50, warmup: int = 5) -> dict:
    """The same step written with library FFTs: torch.fft (cuFFT) rfft2 of
    the field, per kernel a product with its real spectrum and irfft2, the
    growth sum, Euler step and clip in torch ops; the whole step captured
    in one CUDA graph. Timed like the value region (L2 flushed before each
    step, CUDA events around the graph replay). A comparator only: the
    library's own kernels, none of this package's."""
    import torch

    K = len(params["kernels"])
    r = float(params["radius"])
    yy, xx = np.meshgrid(np.fft.fftfreq(h) * h, np.fft.fftfreq(w) * w, indexing="ij")
    khat = []
    for k in params["kernels"]:
        # Ring image: exponential core exp(4 - 1/(s(1-s))) on each of the
        # kernel's len(betas) shells of the normalised radius, peak beta_i.
        d = np.sqrt(xx * xx + yy * yy) / (r * k.get("radiusScale", 1.0))
        nb = len(k["betas"])
        u = d * nb
        i = np.minimum(np.floor(u), nb - 1).astype(int)
        f = np.clip(u - i, 1e-6, 1 - 1e-6)
        img = np.where(d < 1.0, np.array(k["betas"])[i] * np.exp(4.0 - 1.0 / (f * (1.0 - f))), 0.0)
        img /= img.sum()
        khat.append(torch.from_numpy(np.fft.rfft2(img).real.astype(np.float32)).cuda())
    mu = [float(k["mu"]) for k in params["kernels"]]
    sigma = [float(k["sigma"]) for k in params["kernels"]]
    hw = [float(k["weight"]) for k in params["kernels"]]
    dt = float(params["dt"])
    state = torch.from_numpy(np.ascontiguousarray(init, dtype=np.float32)).cuda()
    stream = torch.cuda.Stream()

    def step():
        fa = torch.fft.rfft2(state)
        g = torch.zeros_like(state)
        for q in range(K):
            u = torch.fft.irfft2(fa * khat[q], s=state.shape)
            g += hw[q] * (2.0 * torch.exp(-0.5 * ((u - mu[q]) / sigma[q]) ** 2) - 1.0)
        state.copy_(torch.clamp(state + dt * g, 0.0, 1.0))

    with torch.cuda.stream(stream):
        for _ in range(3):
            step()  # cuFFT plans made outside the capture
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=stream):
        step()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    times = []
    with torch.cuda.stream(stream):
        for i in range(warmup + steps):
            flush.zero_()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            graph.replay()
            b.record(stream)
            if i >= warmup:
                times.append((a, b))
    torch.cuda.synchronize()
    ms = float(np.mean([a.elapsed_time(b) for a, b in times]))
    del graph
    return {"what": "torch.fft (cuFFT) rfft2 + per kernel product and irfft2 + growth/Euler/clip in torch "
                    "ops, one CUDA graph per step, L2 flushed before each step",
            "ms_per_step": ms, "value": w * h / (ms / 1e3) / 1e6, "unit": UNIT, "steps": steps}


def cpu_baseline_fft_1024x512(seconds: float = 8.0) -> dict:
    """The reference's own FFT path (radix-2 Stockham passes, 85 per substep
    at K=3: Modules/FieldModules/Lenia.cpp:576-643, Shaders/Common/
    FFT.metal:65-177) compiled for the CPU, on the whole 1024x512 field of
    the multi-kernel workload (3 kernels R=24, the reference's Gaussian-shell
    core), all host threads: the like-for-like CPU figure for the spectral
    path, where 1080p makes the reference fall back to direct convolution."""
    from life_simulation_b200 import workloads as wl
    from oracle.lenia_oracle import RefLenia

    if not RefLenia.available():
        return {"value": None, "error": "oracle/_ref (compiled reference) not built"}
    p = wl.fft3_params(1024, 512)
    p.pop("kernelCore")
    p.pop("fftAnySize")
    r = RefLenia(p, 1024, 512)
    r.reset(2)
    r.set_initial_field(wl.patches(1024, 512, 20, 96, seed=2))
    r.encode(0, 1)  # init pass + kernel spectra + one substep (warm-up)
    p0 = r.pass_count()
    steps, t0 = 0, time.perf_counter()
    while True:
        r.encode(1 + steps, 1)
        steps += 1
        el = time.perf_counter() - t0
        if el >= seconds or steps >= 200:
            break
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    return {"value": 1024 * 512 * steps / el / 1e6, "unit": UNIT, "cores": cores, "kind": "reference",
            "passes_per_substep": (r.pass_count() - p0) / steps,
            "sample": f"whole 1024x512 field, 3 kernels R=24 (Gaussian shell), convMode fft: {steps} "
                      f"substeps in {el:.1f} s"}


def cpu_baseline(params, w, h, init, seconds):
    from oracle.lenia_oracle import RefLenia
    if RefLenia.available():
        return cpu_baseline_reference(params, w, h, init, seconds)
    return cpu_baseline_port(params, w, h, init, seconds)


def accuracy_vs_fp64(params, w, h, init, steps: int = 5) -> dict:
    """Max and RMS |A_gpu - A_fp64| per step of the workload: every step,
    the GPU module (through the C ABI) and the FP64 oracle both start from
    the GPU's current field, so each figure is one step's error, not an
    accumulated drift. Part of the CPU leg: the oracle only checks."""
    import life_simulation_b200 as lb
    from oracle import lenia_oracle as lo

    m = lb.LeniaModule(params, w, h)
    o = lo.OracleLenia(params, w, h, "f64")
    m.reset(3)
    o.reset(3)
    m.upload(init)
    o.set_initial_field(init)
    o.encode(0)  # builds the oracle's kernels; its state is replaced below
    fp = m.frame_params(0)
    a = np.asarray(init, np.float32)
    mx, rms = [], []
    for s in range(steps):
        fp.frame_index = fp.audio_frame = s
        m.upload(a)
        m.step(fp, 1)
        g = m.field()
        o.state = a.astype(np.float64)
        o.step_once(o.frame_params(), lo.pcg_hash(o.seed_ ^ (s * 197)), s, s)
        d = g.astype(np.float64) - o.state
        mx.append(float(np.abs(d).max()))
        rms.append(float(np.sqrt(np.mean(d * d))))
        a = g
    m.close()
    return {"steps": steps, "max_abs": mx, "rms": rms, "bound": 1e-5,
            "what": "per step from the GPU's field, FP32 GPU vs the FP64 oracle"}


def base_line(args, n, steps, warmup, w, h, params):
    return {
        "metric": METRIC, "unit": UNIT, "n_gpus": n, "steps": steps, "warmup": warmup,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded uniform patches, SplitMix64 seed 2)",
        "config": {"workload": args.workload, "width": w, "height": h,
                   "kernels": len(params.get("kernels", [])) or 1, "radius": params.get("radius"),
                   "kernel_core": params.get("kernelCore", "gaussShell"),
                   "growth_mode": params.get("growthMode"),
                   "l2": "flushed between timed steps (256 MiB write)",
                   "parallelism": f"replicas x{n}" if n > 1 else "single world"},
    }


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    from life_simulation_b200 import workloads as wl
    from oracle.lenia_oracle import RefLenia
    params, w, h, init = wl.workload(args.workload)
    line = base_line(args, args.gpus, args.steps, args.warmup, w, h, params)
    line["impl"] = "reference"
    if not RefLenia.available():
        # The compiled reference is missing; the oracle port stands in.
        cb = cpu_baseline_port(params, w, h, init, 10.0)
        line.update(value=cb["value"], ms_per_step=w * h / cb["value"] / 1e3, cpu_baseline=cb)
        line["e2e"] = {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
        print(json.dumps(line))
        return 0
    band = 32
    r = RefLenia(params, w, h)
    r.reset(2)
    r.set_initial_field(init)
    r.set_row_window(0, band)
    r.encode(0, 1)
    for i in range(args.warmup):
        r.encode(1 + i, 1)
    t0 = time.perf_counter()
    for i in range(args.steps):
        r.encode(1 + args.warmup + i, 1)
    el = time.perf_counter() - t0
    value = w * band * args.steps / el / 1e6
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    line.update(value=value, ms_per_step=el * 1e3 / args.steps)
    line["cpu_baseline"] = {
        "value": value, "unit": UNIT, "cores": cores, "kind": "reference",
        "sample": f"each step: rows 0..{band} of the {w}x{h} field (one substep); the reference "
                  "falls back from convMode fft to direct convolution with kernels[0] at this "
                  "non-power-of-two size (Lenia.cpp:245-269)"}
    line["e2e"] = {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    print(json.dumps(line))
    return 0


def run_b200(args):
    import torch

    rank, world, local = dist_env()
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    torch.cuda.set_device(local)
    import life_simulation_b200 as lb
    from life_simulation_b200 import workloads as wl

    params, w, h, init = wl.workload(args.workload)
    m = lb.LeniaModule(params, w, h)
    m.reset(2 + rank)
    m.upload(init)
    # A dedicated stream: handle 0 (the legacy default stream) would mean
    # "the context's own stream" to the C ABI.
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    sh = stream.cuda_stream
    fp = m.frame_params(0)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
            torch.cuda.synchronize()

    def run_steps(n, first):
        """n steps, the L2 flushed before each; per-step CUDA-event times (ms)
        on the bench stream."""
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(n)]
        for i in range(n):
            flush.zero_()
            fp.frame_index = fp.audio_frame = first + i
            evs[i][0].record(stream)
            m.step(fp, 1, sh)
            evs[i][1].record(stream)
        barrier()
        return [a.elapsed_time(b) for a, b in evs]

    # Launch shapes (columns / rows per CTA of the two passes) chosen under
    # this run's own conditions -- the L2 flushed before every step -- by
    # timing each supported shape outside the timed region; then the state
    # is reset so the timed steps start from the same field as without it.
    shape, chosen_by = m.tuning(), "setup autotuner"
    if shape != (0, 0) and args.launch_shape:
        c, r = args.launch_shape.split(",")
        shape = (int(c.rstrip("h")) | (lb.COLS_HALF_THREADS if c.endswith("h") else 0),
                 int(r.rstrip("p")) | (lb.ROWS_PIPELINED if r.endswith("p") else 0))
        m.set_tuning(*shape)
        chosen_by = "--launch-shape"
    elif shape != (0, 0) and not args.keep_tuning:
        best = None
        for c in (8, 4, 2, 4 | lb.COLS_HALF_THREADS):
            for r in (4, 2, 1, 4 | lb.ROWS_PIPELINED, 2 | lb.ROWS_PIPELINED, 1 | lb.ROWS_PIPELINED):
                try:
                    m.set_tuning(c, r)
                except lb.LeniaError:
                    continue  # over the thread or shared-memory limit at this size
                run_steps(3, 0)
                t = statistics.median(run_steps(30, 0))
                if best is None or t < best[0]:
                    best = (t, (c, r))
        shape, chosen_by = best[1], "bench: median of 30 flushed steps per shape"
        m.set_tuning(*shape)
        m.reset(2 + rank)
        m.upload(init)
    for i in range(max(3, args.warmup)):
        fp.frame_index = fp.audio_frame = i
        m.step(fp, 1, sh)
    barrier()
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    m.profile(False)  # resets the launch counter; no per-launch events
    step_ms = run_steps(args.steps, args.warmup)
    launches = m.profile_read()["launches"]
    cl = clocks.stop()
    total_ms = float(sum(step_ms))
    # Per-kernel durations for the roofline: the same steps again with CUDA
    # events around every launch (events between the two passes serialise
    # them, so these durations are an upper bound; the step value above is
    # timed without them).
    prof_steps = min(args.steps, 100)
    m.profile(True)
    run_steps(prof_steps, args.warmup + args.steps)
    prof = m.profile_read()
    m.profile(False)
    if world > 1:
        t = torch.tensor([total_ms], device="cuda", dtype=torch.float64)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        total_ms = float(t.item())
    value = world * w * h * args.steps / (total_ms / 1e3) / 1e6

    # A frame with its colour layer (RGBA16F at the sim size): lenia_step +
    # lenia_render_rgba16f against lenia_step_render, which writes the texels
    # from the last substep's row pass. Flushed, CUDA events, same stream.
    rgba = torch.empty((h, w, 4), dtype=torch.float16, device="cuda")
    frame_ms = {}
    for mode in ("separate", "fused", "separate", "fused"):
        evs = []
        for i in range(40):
            flush.zero_()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            if mode == "fused":
                m.step_render(fp, 1, rgba.data_ptr(), w, h, sh)
            else:
                m.step(fp, 1, sh)
                m.render_device(rgba.data_ptr(), w, h, sh)
            b.record(stream)
            if i >= 5:
                evs.append((a, b))
        barrier()
        frame_ms[mode] = statistics.median(x.elapsed_time(y) for x, y in evs)
    render_line = {"what": "one substep + the RGBA16F colour layer at the sim size per frame, L2 flushed",
                   "separate_ms": frame_ms["separate"], "fused_ms": frame_ms["fused"]}

    # End to end through the C ABI with pinned host buffers, two ways.
    # serial: per step lenia_upload (pinned host -> field), lenia_step,
    # lenia_download (field -> pinned host), each call waiting for the last.
    # pipelined (the e2e figure): every step still copies its whole input in
    # from pinned host memory and its whole result out, but the copies run on
    # their own streams into / out of device staging buffers, so step i's
    # host->device copy overlaps step i-1's compute and step i-2's
    # device->host copy (PCIe moves both directions at once); the staged
    # field enters and leaves the context by lenia_upload_device /
    # lenia_download_device on the step's stream. Timed by CUDA events from
    # the first copy in to the last copy out.
    e2e_steps = args.e2e_steps or max(10, args.steps // 4)
    host_in = [torch.empty((h, w), dtype=torch.float32, pin_memory=True) for _ in range(2)]
    host_out = [torch.empty((h, w), dtype=torch.float32, pin_memory=True) for _ in range(2)]
    start_field = torch.from_numpy(m.field())
    for x in host_in:
        x.copy_(start_field)
    ctx_stream = torch.cuda.ExternalStream(m.stream())
    barrier()
    serial_ms = 0.0
    for i in range(e2e_steps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        fp.frame_index = fp.audio_frame = 100000 + i
        a.record(ctx_stream)
        m.upload(host_in[0].numpy())
        m.step(fp, 1, None)
        m.download_into(host_out[0].numpy())
        b.record(ctx_stream)
        b.synchronize()
        serial_ms += a.elapsed_time(b)
    d_in = [torch.empty((h, w), dtype=torch.float32, device="cuda") for _ in range(2)]
    d_out = [torch.empty((h, w), dtype=torch.float32, device="cuda") for _ in range(2)]
    s_in, s_out = torch.cuda.Stream(), torch.cuda.Stream()
    ev_in = [torch.cuda.Event() for _ in range(e2e_steps)]
    ev_step = [torch.cuda.Event() for _ in range(e2e_steps)]
    ev_out = [torch.cuda.Event() for _ in range(e2e_steps)]

    def pipelined(frame0):
        """e2e_steps pipelined steps; device milliseconds from the first copy
        in to the last copy out."""
        t_a, t_b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        barrier()
        t_a.record(s_in)
        for i in range(e2e_steps):
            k = i % 2
            with torch.cuda.stream(s_in):
                if i >= 2:
                    s_in.wait_event(ev_step[i - 2])  # staging buffer k consumed by step i-2
                d_in[k].copy_(host_in[k], non_blocking=True)
                ev_in[i].record(s_in)
            stream.wait_event(ev_in[i])
            if i >= 2:
                stream.wait_event(ev_out[i - 2])  # result buffer k copied out
            fp.frame_index = fp.audio_frame = frame0 + i
            m.upload_device(d_in[k].data_ptr(), sh)
            m.step(fp, 1, sh)
            m.download_device(d_out[k].data_ptr(), sh)
            ev_step[i].record(stream)
            with torch.cuda.stream(s_out):
                s_out.wait_event(ev_step[i])
                host_out[k].copy_(d_out[k], non_blocking=True)
                ev_out[i].record(s_out)
        s_out.wait_event(ev_out[-1])
        t_b.record(s_out)
        barrier()
        return t_a.elapsed_time(t_b)

    pipelined(200000)  # warm-up (first use of the staging buffers and streams)
    runs = [pipelined(300000 + 1000 * r) for r in range(3)]
    e2e_ms = statistics.median(runs)
    # The pipelined results are the real steps: the last one equals the
    # context's field.
    e2e_ok = bool(np.array_equal(host_out[(e2e_steps - 1) % 2].numpy(), m.field()))
    if world > 1:
        t = torch.tensor([e2e_ms, serial_ms], device="cuda", dtype=torch.float64)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        e2e_ms, serial_ms = float(t[0].item()), float(t[1].item())
    e2e_value = world * w * h * e2e_steps / (e2e_ms / 1e3) / 1e6
    e2e_serial = world * w * h * e2e_steps / (serial_ms / 1e3) / 1e6

    # Roofline of the dominant kernel (HBM bound).
    K = len(params.get("kernels", [])) or 1
    bytes_px = {"column": 4 + 2 * K + 4 * K, "row_growth": 4 * K + 4 + 4 + 4, "row_fft": 4 + 4,
                "direct": 8}
    phases = {k: v for k, v in prof.items() if isinstance(v, dict) and v["count"] > 0}
    dom = max(phases, key=lambda k: phases[k]["ms"])
    launch_ms = phases[dom]["ms"] / phases[dom]["count"]
    peak, peak_kind = measured_peaks()
    achieved = bytes_px[dom] * w * h / (launch_ms / 1e3) / 1e9
    direct_flops = None
    if dom == "direct":
        # The direct convolution is FP32-FMA bound: 2 FLOP per nonzero tap
        # plus ~12 for the growth map, per pixel and kernel.
        info = m.info()
        direct_flops = (2 * info["direct_taps"] + 12 * info["num_kernels"]) * w * h
    step_bytes = (20 + 10 * K) * w * h  # canonical three-sweep bytes per pixel-step
    mean_step_ms = total_ms / args.steps
    line = base_line(args, world, args.steps, args.warmup, w, h, params)
    if shape != (0, 0):
        line["config"]["launch_shape"] = {"cols_per_cta": shape[0] & 0xF,
                                          "cols_half_threads": bool(shape[0] & lb.COLS_HALF_THREADS),
                                          "rows_per_cta": shape[1] & 0xFF,
                                          "rows_pipelined": bool(shape[1] & lb.ROWS_PIPELINED),
                                          "chosen_by": chosen_by}
    if direct_flops is not None:
        pk = fp32_peak_measured()
        fp32_peak = pk["ffma_tflops"]
        tflops = direct_flops / (launch_ms / 1e3) / 1e12
        roofline = {"bound": "fp32", "kernel": dom, "achieved": tflops, "peak": fp32_peak,
                    "peak_source": pk["source"], "unit": "TFLOP/s",
                    "frac": tflops / fp32_peak, "traffic": None, "algorithmic_flops_per_launch": direct_flops,
                    "launch_ms": launch_ms}
    else:
        traffic, traffic_source = captured_traffic(dom, args.workload)
        roofline = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak,
                    "peak_source": peak_kind, "unit": "GB/s", "frac": achieved / peak,
                    "traffic": traffic, "traffic_source": traffic_source,
                    "algorithmic_bytes_per_launch": bytes_px[dom] * w * h,
                    "launch_ms": launch_ms,
                    "step": {"bytes": step_bytes, "achieved": step_bytes / (mean_step_ms / 1e3) / 1e9,
                             "frac": step_bytes / (mean_step_ms / 1e3) / 1e9 / peak}}
    line.update({
        "value": value, "ms_per_step": mean_step_ms,
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(w * h * 4),
                "d2h_bytes_per_step": int(w * h * 4), "steps": e2e_steps,
                "how": "pipelined: pinned host -> staging (copy stream), lenia_upload_device + lenia_step + "
                       "lenia_download_device (step stream), staging -> pinned host (copy stream)",
                "last_result_equals_field": e2e_ok,
                "timing": "median of 3 timed runs after one warm-up run",
                "serial": {"value": e2e_serial, "how": "lenia_upload, lenia_step, lenia_download in turn"}},
        "gpu_launches": int(launches),
        "roofline": roofline,
        "phases_ms_per_step": {k: v["ms"] / prof_steps for k, v in phases.items()},
        "kernel_timing": f"per-launch CUDA events over {prof_steps} further flushed steps",
        "frame_with_colour_layer": render_line,
        "clocks": cl,
    })
    if rank == 0 and world == 1 and not args.no_adjoint:
        line["adjoint"] = adjoint_bench(args.adjoint_reps)
    if rank == 0 and world == 1 and not args.no_library_baseline:
        line["library_fft_baseline"] = library_fft_baseline(params, w, h, init)
    if rank == 0 and world == 1 and args.workload == WORKLOAD:
        line["published_config"] = published_config_bench()
        line["published_direct_config"] = published_direct_bench()
    if rank == 0 and world == 1:
        line["fp32_peak"] = fp32_peak_measured()
    if rank == 0 and world == 1 and not args.no_sweep:
        line["sweep"] = sweep_bench(args.plain_steps)
    if rank == 0 and world == 1 and not args.no_tc:
        line["tc"] = tc_bench(error_check=not args.no_cpu_baseline)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            line["cpu_baseline"] = cpu_baseline(params, w, h, init, args.cpu_seconds)
        except Exception as e:  # the oracle is optional here; the GPU number stands
            line["cpu_baseline"] = {"value": None, "error": str(e)}
        try:
            line["cpu_baseline_fft_1024x512"] = cpu_baseline_fft_1024x512()
        except Exception as e:
            line["cpu_baseline_fft_1024x512"] = {"value": None, "error": str(e)}
        try:
            line["accuracy_vs_fp64"] = accuracy_vs_fp64(params, w, h, init)
        except Exception as e:
            line["accuracy_vs_fp64"] = {"error": str(e)}
    if rank == 0:
        print(json.dumps(line))
    m.close()
    if world > 1:
        torch.distributed.destroy_process_group()
    return 0


def adjoint_bench(reps: int = 5, warmup: int = 3) -> dict:
    """Forward rollout and backward of the gradient form on the adjoint_512
    workload (life_simulation_b200/workloads.py), device-timed."""
    import torch

    import life_simulation_b200 as lb
    from life_simulation_b200 import workloads as wl

    c = wl.ADJOINT_512
    B, W, H, T = c["batch"], c["width"], c["height"], c["steps"]
    eng = lb.LeniaAdjoint(W, H, B, wl.ADJOINT_KERNELS, c["radius"], T, c["checkpoint_every"], c["dt"],
                          c["growth_mode"], lb.CORE_EXP)
    stream = torch.cuda.Stream()
    sh = stream.cuda_stream
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    with torch.cuda.stream(stream):
        a0 = torch.from_numpy(wl.adjoint_fields(4000, B, W, H)).cuda()
        t0 = torch.from_numpy(wl.adjoint_fields(5000, B, W, H)).cuda()
        target = torch.empty_like(t0)
        eng.forward(t0.data_ptr(), target.data_ptr(), sh)
        out = torch.empty_like(a0)
        ga0 = torch.empty_like(a0)
        gp = torch.empty(lb.ADJOINT_NUM_PARAMS, dtype=torch.float64, device="cuda")
        fwd, bwd = [], []
        for i in range(warmup + reps):
            e = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
            flush.zero_()
            e[0].record(stream)
            eng.forward(a0.data_ptr(), out.data_ptr(), sh)
            e[1].record(stream)
            g = 2.0 * (out - target) / out.numel()
            flush.zero_()
            e[2].record(stream)
            eng.backward(g.data_ptr(), ga0.data_ptr(), gp.data_ptr(), sh)
            e[3].record(stream)
            stream.synchronize()
            if i >= warmup:
                fwd.append(e[0].elapsed_time(e[1]))
                bwd.append(e[2].elapsed_time(e[3]))
        loss = float(torch.mean((out - target) ** 2))
        gnorm = float(ga0.abs().max())
    st = eng.stats()
    eng.close()
    f, b = statistics.median(fwd), statistics.median(bwd)
    px_steps = B * W * H * T
    return {"workload": "adjoint_512: 32 worlds 512x512, K=2 R=16 b=[1],[0.5,1], growth mode 1, T=64, checkpoints every 8",
            "forward_ms": f, "backward_ms": b, "ratio": b / f,
            "forward_mpx_steps_s": px_steps / (f / 1e3) / 1e6,
            "backward_mpx_steps_s": px_steps / (b / 1e3) / 1e6,
            "reps": reps, "loss": loss, "max_abs_grad_a0": gnorm,
            "device_bytes": st["device_bytes"],
            "timing": "median of reps; CUDA events on the launching stream; L2 flushed before each"}


def run_adjoint(args):
    import torch

    torch.cuda.set_device(0)
    r = adjoint_bench(args.adjoint_reps)
    line = {"metric": "Lenia adjoint/forward time ratio (32 x 512x512, K=2, R=16, growth mode 1, T=64, checkpoints every 8)",
            "value": r["ratio"], "unit": "x", "higher_is_better": False, "n_gpus": 1, "dtype": "f32",
            "data": "synthetic", "config": {"workload": r["workload"]}}
    line.update(r)
    print(json.dumps(line))
    return 0


def tc_bench(warmup: int = 3, steps: int = 64, error_check: bool = True, only=None) -> dict:
    """4096x4096, 3 kernels R=32: the column DFT stages on the CUDA cores (FP32)
    and on the tensor cores (FP16 / BF16 hi/lo, FP32 accumulation): per
    precision the device time per step, the column pass's HBM roofline and
    tensor FLOP rate, and (error_check) max / RMS |A - A_fp64| of one step
    from the same field against the FP64 oracle."""
    import torch

    import life_simulation_b200 as lb
    from life_simulation_b200 import workloads as wl

    w = h = 4096
    K = 3
    init = wl.patches(w, h, 40, 256, seed=2)
    stream = torch.cuda.Stream()
    sh = stream.cuda_stream
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    peak, peak_kind = measured_peaks()
    col_bytes = (4 + 2 * K + 4 * K) * w * h
    # Tensor FLOPs per column launch, (1 forward + K inverse) transforms per
    # column: mma.sync engine, 3 radix-16 stages x H points x 128 FLOP (real
    # 32x32 GEMM per 16 points) x 3 (hi/lo); tcgen05 engine, 2 radix-64
    # passes x H/64 items x 2 x 128 x 128 x 3 (real 128x128 GEMM per 64
    # points, hi/lo).
    tc05_flops = (1 + K) * 2 * (h // 64) * 2 * 128 * 128 * 3 * (w // 2)
    tc_flops = {"mma": (1 + K) * 3 * h * 128 * 3 * (w // 2), "tcgen05_serial": tc05_flops,
                "tcgen05_pipelined": tc05_flops}
    res = {}
    variants = (("fp32", "fp32", None), ("fp16x3", "fp16x3", "mma"), ("bf16x3", "bf16x3", "mma"),
                ("fp16x3_tcgen05", "fp16x3", "tcgen05_serial"), ("bf16x3_tcgen05", "bf16x3", "tcgen05_serial"),
                ("fp16x3_tcgen05_pipelined", "fp16x3", "tcgen05_pipelined"),
                ("bf16x3_tcgen05_pipelined", "bf16x3", "tcgen05_pipelined"))
    for name, prec, engine in variants:
        if only and name not in only:
            continue
        p = wl.fft3_params(w, h)
        p["radius"] = 32
        p["fftPrecision"] = prec
        # LENIA_TC_ENGINE at setup keeps one engine's candidates.
        old_engine = os.environ.pop("LENIA_TC_ENGINE", None)
        if engine:
            os.environ["LENIA_TC_ENGINE"] = engine
        try:
            m = lb.LeniaModule(p, w, h)
        finally:
            os.environ.pop("LENIA_TC_ENGINE", None)
            if old_engine is not None:
                os.environ["LENIA_TC_ENGINE"] = old_engine
        m.reset(2)
        m.upload(init)
        fp = m.frame_params(0)
        for i in range(max(3, warmup)):
            fp.frame_index = fp.audio_frame = i
            m.step(fp, 1, sh)
        torch.cuda.synchronize()
        m.profile(True)
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        for i in range(steps):
            with torch.cuda.stream(stream):
                flush.zero_()
            fp.frame_index = fp.audio_frame = 100 + i
            evs[i][0].record(stream)
            m.step(fp, 1, sh)
            evs[i][1].record(stream)
        torch.cuda.synchronize()
        prof = m.profile_read()
        m.profile(False)
        step_ms = sum(a.elapsed_time(b) for a, b in evs) / steps
        col = prof["column"]
        col_ms = col["ms"] / col["count"]
        r = {"ms_per_step": step_ms, "mpx_steps_s": w * h / (step_ms / 1e3) / 1e6,
             "column_ms": col_ms, "row_ms": prof["row_growth"]["ms"] / prof["row_growth"]["count"],
             "column_gbs": col_bytes / (col_ms / 1e3) / 1e9, "column_frac_hbm": col_bytes / (col_ms / 1e3) / 1e9 / peak,
             "fft_precision": m.info()["fft_precision"], "tc_engine": m.info()["tc_engine"]}
        if prec != "fp32":
            r["column_tensor_tflops"] = tc_flops[engine] / (col_ms / 1e3) / 1e12
        if error_check:
            # One step from the seeded field itself (alive; the timed steps
            # have let the patches decay by now).
            m.upload(init)
            fp.frame_index = fp.audio_frame = 0
            m.step(fp, 1, sh)
            torch.cuda.synchronize()
            r["_next"] = m.field()
        res[name] = r
        m.close()
    if error_check:
        from oracle import lenia_oracle as lo
        p = wl.fft3_params(w, h)
        p["radius"] = 32
        o = lo.OracleLenia(p, w, h, "f64")
        o.reset(2)
        o.set_initial_field(init)
        o.encode(0)  # builds the kernels; its state is replaced below
        o.state = init.astype(np.float64)
        o.step_once(o.frame_params(), lo.pcg_hash(o.seed_), 0, 0)
        for prec, r in res.items():
            d = r.pop("_next").astype(np.float64) - o.state
            r["max_err_vs_fp64"] = float(np.abs(d).max())
            r["rms_err_vs_fp64"] = float(np.sqrt(np.mean(d * d)))
    return {"workload": "4096x4096, 3 kernels R=32 (fft3 peaks/mu/sigma/h), 40 patches of 256x256 (seed 2)",
            "steps": steps, "l2": "256 MiB write between steps", "peak_hbm_gbs": peak, "peak_source": peak_kind,
            "column_bytes_per_launch": col_bytes, "column_tensor_flops_per_launch": tc_flops,
            "engines": "tc_engine 1: mma.sync radix-16 tiles; 2: tcgen05 radix-64 GEMMs, accumulators in tensor "
                       "memory, each pass waited for; 3: the same over two operand slots, one kernel's MMAs "
                       "overlapping the next kernel's operand build",
            "error": "one step from the seeded field vs one FP64 oracle step from it",
            "precisions": res}


def run_tc(args):
    import torch

    torch.cuda.set_device(0)
    only = set(args.tc_variants.split(",")) if args.tc_variants else None
    r = tc_bench(args.warmup, args.tc_steps, not args.no_tc_error, only)
    first = next(iter(r["precisions"].values()))
    line = {"metric": "Lenia Mpixel-steps/s, 4096x4096 K=3 R=32: column DFT stages FP32 CUDA cores vs "
                      "split-precision tensor cores",
            "unit": UNIT, "value": r["precisions"].get("fp32", first)["mpx_steps_s"], "higher_is_better": True,
            "n_gpus": 1,
            "dtype": "f32 / fp16x3 / bf16x3", "data": "synthetic", "config": {"workload": r["workload"]}}
    line.update(r)
    print(json.dumps(line))
    return 0


def sweep_batched(worlds, inits, form=None):
    """The 512-world sweep's batched form on this GPU: the batch's graphs
    replay 4 x 60 substeps with the activity readback after each (the lab's
    luma statistic per world). `form`: the launch form (None: the one the
    batch's autotuner picks). Returns (wall seconds, per-readback activity,
    path per world, launch form used)."""
    import torch

    import life_simulation_b200 as lb
    from life_simulation_b200.sweep import is_alive

    b = lb.LeniaBatch(worlds, lb.BATCH_AUTO)
    if form is not None:
        b.set_launch_form(form)
    used = b.launch_form()
    for i, a in enumerate(inits):
        b.upload(i, a)
    b.step(60)  # warm-up (also captures the graph)
    b.sync()
    for i, a in enumerate(inits):
        b.upload(i, a)
    b.step(0)
    b.sync()
    cm = lb.colormap_from_params({})
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    acts = []
    for _ in range(4):
        b.step(60)
        acts.append(b.activity(cm))  # synchronising readback
    seconds = time.perf_counter() - t0
    # Per readback: the worlds' mean luma and luma variance, averaged over
    # the worlds, and how many pass the lab's alive rule.
    activity = [{"step": 60 * (j + 1), "mean_luma": float(mean.mean()), "mean_var_luma": float((std * std).mean()),
                 "alive": sum(1 for x, y in zip(mean, std) if is_alive(float(x), float(y)))}
                for j, (mean, std) in enumerate(acts)]
    paths = [b.path(i) for i in range(len(worlds))]
    b.close()
    return seconds, activity, paths, used


def sweep_worlds(specs):
    import life_simulation_b200 as lb

    return [lb.make_world(s["width"], s["height"], s["radius"], s["mu"], s["sigma"], s["dt"], 0, seed=s["seed"])
            for s in specs]


def sweep_bench(plain_steps: int = 10) -> dict:
    """The 512-world sweep on one GPU: batched (graph replays, activity
    readback every 60 substeps, wall clock) against the plain form (one
    context per world, worlds stepped one after another on one stream, as
    the reference's variant loop steps one SceneRunner at a time:
    Apps/LifePresetLab/main.cpp:718-795)."""
    import torch

    import life_simulation_b200 as lb
    from life_simulation_b200 import workloads as wl

    specs, inits = wl.sweep512()
    worlds = sweep_worlds(specs)
    px = sum(w.width * w.height for w in worlds)
    batched_s, activity, paths, form = sweep_batched(worlds, inits)
    # The other launch form, timed the same way, for comparison.
    other = lb.BATCH_FORM_PER_SIZE if form == lb.BATCH_FORM_PERSISTENT else lb.BATCH_FORM_PERSISTENT
    try:
        other_s = sweep_batched(worlds, inits, other)[0]
    except lb.LeniaError:
        other_s = None
    names = {lb.BATCH_FORM_PERSISTENT: "persistent", lb.BATCH_FORM_PER_SIZE: "per_size"}
    forms = {names[form]: px * 240 / batched_s / 1e6}
    if other_s:
        forms[names[other]] = px * 240 / other_s / 1e6
    mods = []
    for i, w in enumerate(worlds):
        conv = "fft" if paths[i] == lb.CONV_FFT else "direct"
        m = lb.LeniaModule(lb.single_world_params(w, conv), w.width, w.height)
        m.reset(w.seed)
        m.upload(inits[i])
        mods.append(m)
    one = torch.cuda.Stream()
    sh = one.cuda_stream
    for m in mods:
        m.encode(0, 1, stream=sh)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for m in mods:
        for f in range(plain_steps):
            m.encode(1 + f, 1, stream=sh)
    torch.cuda.synchronize()
    plain_s = time.perf_counter() - t0
    for m in mods:
        m.close()
    batched = px * 240 / batched_s / 1e6
    plain = px * plain_steps / plain_s / 1e6
    return {"value": batched, "unit": UNIT, "plain": plain, "speedup": batched / plain,
            "worlds": len(worlds), "pixels_per_step": px, "steps": 240,
            "direct_worlds": paths.count(lb.CONV_DIRECT), "fft_worlds": paths.count(lb.CONV_FFT),
            "launch_form": names[form], "forms": forms,
            "launches_per_substep": {"persistent": 1,
                                     "per_size": 2 * len({(w.width, w.height) for w in worlds}) + 1},
            "activity": activity,
            "timing": "wall clock incl. 4 activity readbacks (batched); plain: "
                      f"{plain_steps} substeps per world, worlds in sequence on one stream"}


def run_sweep(args):
    """The 512-world sweep, batched against the plain form (one GPU), or
    sharded by world over the ranks under torchrun."""
    import torch

    import life_simulation_b200 as lb
    from life_simulation_b200 import workloads as wl
    from life_simulation_b200.shard import loads, partition, world_cost

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world == 1:
        line = {"metric": "Lenia Mpixel-steps/s, 512-world sweep (batched vs one world at a time)", "n_gpus": 1}
        line.update(sweep_bench(args.plain_steps))
        print(json.dumps(line))
        return 0
    import datetime

    torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    specs, inits = wl.sweep512()
    px_all = sum(s["width"] * s["height"] for s in specs)
    # Each rank steps its cost-balanced share of the worlds as one batch;
    # nothing crosses between GPUs until the final timing.
    costs = [world_cost(s["width"], s["height"], s["radius"]) for s in specs]
    shares = partition(costs, world)
    mine = shares[rank]
    torch.distributed.barrier()
    batched_s, _, paths, _ = sweep_batched(sweep_worlds([specs[i] for i in mine]), [inits[i] for i in mine])
    t = torch.tensor([batched_s], device="cuda", dtype=torch.float64)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    batched_s = float(t.item())
    n_direct = torch.tensor([paths.count(lb.CONV_DIRECT)], device="cuda")
    torch.distributed.all_reduce(n_direct)
    torch.cuda.synchronize()
    torch.distributed.barrier()
    torch.distributed.destroy_process_group()
    if rank == 0:
        print(json.dumps({
            "metric": "Lenia Mpixel-steps/s, 512-world sweep (batched, worlds sharded over GPUs)",
            "unit": UNIT, "value": px_all * 240 / batched_s / 1e6, "n_gpus": world, "scaling": "strong",
            "worlds": 512, "pixels_per_step": px_all, "steps": 240, "direct_worlds": int(n_direct.item()),
            "shares": [len(x) for x in shares],
            "estimated_load_ratio": max(loads(costs, shares)) / min(loads(costs, shares)),
            "timing": "wall clock incl. 4 activity readbacks, max over ranks; worlds assigned "
                      "largest estimated cost first to the least-loaded rank"}))
    return 0


def main():
    args = parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.mode == "sweep":
        return run_sweep(args)
    if args.mode == "adjoint":
        return run_adjoint(args)
    if args.mode == "tc":
        return run_tc(args)
    return run_b200(args)


if __name__ == "__main__":
    sys.exit(main())
