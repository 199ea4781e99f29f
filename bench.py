#!/usr/bin/env python
"""Benchmark of the equirectangular rasterizer: forward + backward of one 2048 x 1024 view over
1,000,000 Gaussians per step (the reference's headline single-view workload).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl omnigs|reference]

One process per GPU (torchrun for N > 1, NCCL).  Each rank renders and back-propagates its own
view of the shared Gaussian set (weak scaling); for N > 1 the per-Gaussian gradients are summed
across ranks every step with one NCCL all-reduce, as a data-parallel train step does.

* value: views/s of the whole job, device-timed with CUDA events on the launching stream over K
  steps (max over ranks), inputs resident in HBM.  Each step touches far more than the 126 MB L2
  (the SH coefficients alone are 192 MB), so no flush is needed between steps.
* e2e: the same metric through the reference-facing LibTorch API (RasterizeGaussiansCUDA +
  RasterizeGaussiansBackwardCUDA), with every step copying its per-view inputs (camera, upstream
  image gradient) from pinned host memory and its rendered image back to pinned host memory; the
  copies run on two copy streams, overlapped with the neighbouring steps' compute as a training
  loop would pipeline them.  The Gaussian parameters and their gradients stay on the device, as in
  the reference trainer.
* roofline: per-kernel device times from the library's event timing, against the algorithmic bytes
  of each stage; the dominant kernel is reported against MEASURED_PEAKS.json.  roofline_fp32 puts
  the blends against the FP32 issue peak (they are FP32/MUFU-issue-bound, not HBM-bound), and
  path_roofline sums every stage's lower-bound time (bytes at the HBM peak or FP32 work at the FP32
  peak) over the measured step time.
* cpu_baseline: the FP64 oracle (multithreaded C++ restatement of the reference algorithm) on the
  same view, on this host's cores.
* configs: the precision configuration (6M pole-heavy Gaussians, 4096x2048), peak memory at
  4096x2048 over 3M Gaussians (stored and recomputed transmittance), the headline view with
  transmittance checkpointing, and the differentiation configuration (500 Adam steps over 24
  views through the LibTorch autograd Function).
* --impl reference: the reference arm.  The reference's rasterizer is CUDA-only, so its CPU
  implementation of the path is the FP64 oracle port, timed here on all host cores.  The same line
  carries reference_gpu: the reference's own CUDA rasterizer rebuilt for sm_100a
  (oracle/ref/Makefile), timed on this workload on the same GPU, and its peak memory at the
  peak-memory workload -- the like-for-like GPU comparison.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "fwd+bwd ms/view & views/s, 1M Gaussians 2048x1024 ERP, batched vs plain"
UNIT = "views/s"
P_GAUSS, WIDTH, HEIGHT = 1_000_000, 2048, 1024
WORKLOAD = "plain single-view fwd+bwd, 1M Gaussians, 2048x1024 equirect, identity pose, SH deg 3"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="omnigs", choices=["omnigs", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched multi-view leg")
    ap.add_argument("--no-extra", action="store_true",
                    help="skip the precision, peak-memory and differentiation legs")
    ap.add_argument("--no-reference-gpu", action="store_true",
                    help="skip the rebuilt reference rasterizer's GPU timing and peak memory")
    # smaller cases for profiling captures only; bench lines use the defaults
    ap.add_argument("--gaussians", type=int, default=P_GAUSS)
    ap.add_argument("--width", type=int, default=WIDTH)
    ap.add_argument("--height", type=int, default=HEIGHT)
    return ap.parse_args()


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), \
        int(os.environ.get("LOCAL_RANK", 0))


# ---------------------------------------------------------------- clocks -----------------------
class NvmlClockSampler:
    """Samples SM clock and clock-event (throttle) reasons through NVML every 5 ms while running
    (read-only queries), so that even a timed region of a few tens of milliseconds gets samples."""

    REASONS = (("hw_slowdown", "nvmlClocksEventReasonHwSlowdown"),
               ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown"),
               ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown"),
               ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap"))

    def __init__(self, gpu_uuid: str):
        import pynvml

        self.nvml = pynvml
        pynvml.nvmlInit()
        self.handle = pynvml.nvmlDeviceGetHandleByUUID(gpu_uuid)
        self.max_mhz = float(pynvml.nvmlDeviceGetMaxClockInfo(self.handle, pynvml.NVML_CLOCK_SM))
        self.samples, self.stop = [], threading.Event()

    def _poll(self):
        n = self.nvml
        while not self.stop.is_set():
            try:
                mhz = float(n.nvmlDeviceGetClockInfo(self.handle, n.NVML_CLOCK_SM))
                bits = int(n.nvmlDeviceGetCurrentClocksEventReasons(self.handle))
                self.samples.append((mhz, bits))
            except n.NVMLError:
                pass
            self.stop.wait(0.005)

    def __enter__(self):
        self._poll_once()
        self.thread = threading.Thread(target=self._poll, daemon=True)
        self.thread.start()
        return self

    def _poll_once(self):
        n = self.nvml
        self.samples.append((float(n.nvmlDeviceGetClockInfo(self.handle, n.NVML_CLOCK_SM)),
                             int(n.nvmlDeviceGetCurrentClocksEventReasons(self.handle))))

    def __exit__(self, *exc):
        self.stop.set()
        self.thread.join(timeout=5)
        self._poll_once()

    def summary(self) -> dict:
        reasons = set()
        for _, bits in self.samples:
            for name, attr in self.REASONS:
                if bits & getattr(self.nvml, attr):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(m for m, _ in self.samples), "sm_max_mhz": self.max_mhz,
                "reasons": sorted(reasons), "samples": len(self.samples), "source": "nvml, 5 ms"}


def clock_sampler(gpu_uuid: str | None):
    """NVML sampler when NVML answers, else nvidia-smi at its 200 ms interval."""
    if gpu_uuid:
        try:
            return NvmlClockSampler(gpu_uuid)
        except Exception:
            pass
    return ClockSampler(gpu_uuid)


class ClockSampler:
    """Samples SM clock and throttle reasons with nvidia-smi while running."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id: str | None):
        self.gpu_id, self.proc, self.lines = gpu_id, None, []

    def __enter__(self):
        cmd = ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200"]
        if self.gpu_id:
            cmd += ["-i", self.gpu_id]
        try:
            self.proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
            except ValueError:
                continue
            for n, v in zip(names, parts[4:8]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm), "source": "nvidia-smi, 200 ms"}


# ---------------------------------------------------------------- roofline ---------------------
def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), float(d.get("sm_max_mhz", 1965.0)), "measured"
    return 6650.0, 1965.0, "fallback"


def traffic_from_profiles() -> dict:
    """Per-launch DRAM bytes per kernel from the committed ncu summary, if present."""
    path = os.path.join(ROOT, "profiles", "dram_traffic_per_launch.txt")
    out = {}
    if os.path.exists(path):
        for ln in open(path):
            parts = ln.split()
            if len(parts) >= 2 and not ln.startswith("#"):
                try:
                    out[parts[0]] = float(parts[1])
                except ValueError:
                    pass
    return out


def stage_bytes(P, V, R, N, Tl):
    """Algorithmic (compulsory) HBM bytes of each stage for one view."""
    return {
        "preprocess": 44 * P + 192 * V + 8 * P + 40 * V + 8 * P,  # + the fused scan of tiles_touched
        "duplicate": 20 * V + 12 * R,
        "sort": 24 * R,
        "ranges": 8 * R + 8 * Tl,
        "render_forward": 40 * R + 8 * Tl + 12 * N + 8 * N,
        "render_backward": 40 * R + 8 * Tl + 12 * N + 8 * N + 44 * V,
        "preprocess_backward": 264 * V + 232 * V,
    }


# ---------------------------------------------------------------- CPU baseline ------------------
def cpu_baseline(g, view, dpix_np, budget_s=30.0):
    import oracle
    nthreads = os.cpu_count() or 1
    t0 = time.perf_counter()
    oracle.forward_backward(g, view, dpix_np, nthreads=nthreads)
    t = time.perf_counter() - t0
    reps = 1
    if 2 * t < budget_s:
        t0 = time.perf_counter()
        reps = max(1, min(5, int(budget_s / max(t, 1e-3)) - 1))
        for _ in range(reps):
            oracle.forward_backward(g, view, dpix_np, nthreads=nthreads)
        t = (time.perf_counter() - t0) / reps
    return {"value": 1.0 / t, "unit": UNIT, "cores": nthreads, "kind": "port",
            "sample": f"{reps} full view(s) of the headline workload (1M Gaussians, 2048x1024, "
                      f"fwd+bwd) through the FP64 oracle; {t:.2f} s per view"}


# ---------------------------------------------------------------- reference arm ----------------
def run_reference(args, rank, world):
    if rank != 0:
        return
    from omnigs_b200 import scenes
    g = scenes.make_gaussians(P_GAUSS, seed=0)
    view = scenes.identity_view(WIDTH, HEIGHT)
    dpix = scenes.upstream_grad(WIDTH, HEIGHT)
    import oracle
    nthreads = os.cpu_count() or 1
    # the requested warm-up views (at most 10: each is a full 1M-Gaussian view on the CPU); the last
    # one's time bounds the number of timed steps to about 150 s of work
    warmup = min(max(args.warmup, 1), 10)
    t_est = 1e-3
    for _ in range(warmup):
        t0 = time.perf_counter()
        oracle.forward_backward(g, view, dpix, nthreads=nthreads)
        t_est = max(time.perf_counter() - t0, 1e-3)
    steps = max(1, min(args.steps, int(150.0 / t_est)))
    t0 = time.perf_counter()
    for _ in range(steps):
        oracle.forward_backward(g, view, dpix, nthreads=nthreads)
    dt = time.perf_counter() - t0
    value = steps / dt
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": steps,
            "warmup": warmup, "ms_per_step": 1000 * dt / steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded scene generators)",
            "config": {"workload": WORKLOAD, "gaussians": P_GAUSS, "width": WIDTH, "height": HEIGHT},
            "impl": "reference",
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": nthreads, "kind": "port",
                             "sample": f"{steps} full view(s); the reference rasterizer has no CPU "
                                       "path, so this is the FP64 oracle restating its algorithm"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if not args.no_reference_gpu:
        line["reference_gpu"] = run_reference_gpu(args)
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- batched views ----------------
BATCH_VIEWS = 16


def run_batched(args, g, gt, dev, plain_views_per_s):
    """Batched fwd+bwd of 16 uneven equirect views over the shared 1M-Gaussian set, one launch per
    stage for the whole batch, the step captured in a CUDA graph and replayed (poses and upstream
    gradients live at fixed device addresses; instance counts stay on the device).  Timed with SH
    stored as BF16 (the precision mode's storage) and, for comparison, as FP32."""
    import torch

    from omnigs_b200 import batch, capi, lonlat, scenes

    views = scenes.random_views(BATCH_VIEWS, scenes.BATCH_RESOLUTIONS, seed=1, cube=2.0, pitch_deg=30.0)
    cams = batch.BatchCameras.from_views(views, dev)
    dl = [torch.from_numpy(scenes.upstream_grad(v.width, v.height, seed=100 + i)).to(dev)
          for i, v in enumerate(views)]
    images = [torch.empty(3, v.height, v.width, device=dev) for v in views]
    pixels = sum(v.width * v.height for v in views)
    results = {}
    stream = torch.cuda.Stream(dev)
    for name, shs in (("bf16", gt.shs.to(torch.bfloat16)), ("fp32", gt.shs)):
        gg = lonlat.GaussianTensors(means3D=gt.means3D, opacities=gt.opacities, shs=shs,
                                    scales=gt.scales, rotations=gt.rotations)
        _, per_view, sizing = batch.render_batch(gg, cams)
        total = sum(per_view)
        del sizing
        state = batch.BatchState(gg.P, cams.sizes, total + total // 8 + 4096, dev)
        grads = batch.BatchGradients.empty(gg.P, gg.M, dev, stats=True)

        def step():
            state.forward(gg, cams, images)
            state.backward(gg, cams, dl, grads)

        if name == "bf16":  # choose the blend staging batch for this workload (kept for the rest)
            state.forward(gg, cams, images)
            results["autotune"] = state.autotune(gg, cams, images, dl, repeats=3)
        with torch.cuda.stream(stream):
            for _ in range(2):
                step()
        torch.cuda.synchronize()
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph, stream=stream):
            step()
        for _ in range(args.warmup):
            graph.replay()
        torch.cuda.synchronize()
        n, per2, st = state.status()
        assert st == 0 and per2 == per_view, (st, per2, per_view)
        cur = torch.cuda.current_stream(dev)
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(cur)
        for _ in range(args.steps):
            graph.replay()
        ev1.record(cur)
        torch.cuda.synchronize()
        ms = ev0.elapsed_time(ev1) / args.steps
        del graph
        # per-stage device times from eager (uncaptured) steps with the library's event timing
        k = max(1, args.steps // 4)
        capi.timing_enable(True)
        for _ in range(k):
            step()
        torch.cuda.synchronize()
        stages = capi.timing_read()
        capi.timing_enable(False)
        results[name] = {
            "views_per_s": round(BATCH_VIEWS / (ms / 1000.0), 3), "ms_per_view": round(ms / BATCH_VIEWS, 4),
            "ms_per_step": round(ms, 4),
            "speedup_vs_plain_fp32": round(BATCH_VIEWS / (ms / 1000.0) / plain_views_per_s, 3),
            "num_rendered": int(n), "gpu_launches_per_step": sum(v[1] for v in stages.values()) // k,
            "stages_ms_per_step": {s: round(v[0] / k, 4) for s, v in stages.items() if v[1]},
        }
        del state, grads
        torch.cuda.empty_cache()
    results["train_step"] = run_train_step(args, g, gt, cams, dev)
    return {"workload": f"{BATCH_VIEWS} equirect views, resolutions drawn from {scenes.BATCH_RESOLUTIONS}, "
                        "positions uniform in a 2 m cube, random yaw, pitch +-30 deg, 1M shared Gaussians, "
                        "fwd+bwd of the whole batch per step, CUDA graph replay",
            "views": BATCH_VIEWS, "pixels_per_step": pixels, "sizes": [list(s) for s in cams.sizes],
            "autotune": results["autotune"], "sh_bf16": results["bf16"], "sh_fp32": results["fp32"],
            "train_step": results["train_step"]}


def run_train_step(args, g, gt, cams, dev):
    """The whole training iteration over the 16-view batch (forward, L1 + 0.2 D-SSIM per view,
    backward with densification statistics, fused Adam; SH in BF16), captured in one CUDA graph."""
    import torch

    from omnigs_b200 import batch, capi, train

    targets, per_view, _ = batch.render_batch(gt, cams)
    total = sum(per_view)
    model = train.GaussianModelState.from_activated(g, device=dev, sh_bf16=True)
    stepper = train.BatchTrainStep(model, cams, targets, capacity=total + total // 4 + 4096)
    stepper.run()
    torch.cuda.synchronize()
    stepper.capture()
    for _ in range(args.warmup):
        stepper.replay()
    torch.cuda.synchronize()
    cur = torch.cuda.current_stream(dev)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(cur)
    for _ in range(args.steps):
        stepper.replay()
    ev1.record(cur)
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1) / args.steps
    n, _, st = stepper.status()
    assert st == 0, st
    # eager step with stage timing: loss and Adam run under the "other" stage
    capi.timing_enable(True)
    stepper.run()
    torch.cuda.synchronize()
    stages = capi.timing_read()
    capi.timing_enable(False)
    del stepper
    return {"ms_per_step": round(ms, 4), "views_per_s": round(BATCH_VIEWS / (ms / 1000.0), 3),
            "sh": "bf16", "graph": True,
            "stages_ms_one_step": {k: round(v[0], 4) for k, v in stages.items() if v[1]},
            "note": "loss + Adam appear under 'other'"}


def run_precision(args, dev):
    """Precision configuration: 6M Gaussians, 30 % beyond 80 deg latitude, one 4096x2048 view;
    fwd+bwd ms/view of the plain FP32 path vs the precision mode (BF16 SH + FP64 poles)."""
    import torch

    from omnigs_b200 import batch, lonlat, scenes

    P, W, H = 6_000_000, 4096, 2048
    g = scenes.make_gaussians(P, seed=4, pole_fraction=0.3)
    gt = lonlat.GaussianTensors.from_numpy(g, dev)
    view = scenes.identity_view(W, H)
    dpix = torch.from_numpy(scenes.upstream_grad(W, H, seed=4)).to(dev)
    out = {}
    # plain FP32 single-view path
    cam = lonlat.Camera.from_view(view, dev)
    _, radii0, n0, _ = lonlat.rasterize(gt, cam)
    state = lonlat.LonlatState(P, W, H, n0 + n0 // 8 + 4096, dev)
    img = torch.empty(3, H, W, device=dev)
    radii = torch.empty(P, dtype=torch.int32, device=dev)
    grads = lonlat.Gradients.empty(P, 16, dev)

    def plain():
        state.forward(gt, cam, img, radii)
        state.backward(gt, cam, radii, dpix, grads)

    out["fp32_plain_ms_per_view"] = _time_steps(plain, args, dev)
    del state, grads
    torch.cuda.empty_cache()
    # precision mode through the batched path
    gb = lonlat.GaussianTensors(means3D=gt.means3D, opacities=gt.opacities, shs=gt.shs.to(torch.bfloat16),
                                scales=gt.scales, rotations=gt.rotations)
    cams = batch.BatchCameras.from_views([view], dev)
    _, per, sizing = batch.render_batch(gb, cams, fp64_poles=True)
    del sizing
    bstate = batch.BatchState(P, cams.sizes, per[0] + per[0] // 8 + 4096, dev)
    bgr = batch.BatchGradients.empty(P, 16, dev)

    def prec():
        bstate.forward(gb, cams, [img], fp64_poles=True)
        bstate.backward(gb, cams, [dpix], bgr, fp64_poles=True)

    out["precision_ms_per_view"] = _time_steps(prec, args, dev)
    out["num_rendered"] = int(n0)
    out["workload"] = "6M Gaussians (30% beyond 80 deg latitude), one 4096x2048 view, fwd+bwd"
    del bstate, bgr, gt, gb
    torch.cuda.empty_cache()
    return out


def run_peak_memory(dev):
    """Peak device memory of one fwd+bwd at 4096x2048 over 3M Gaussians through the plain path,
    with the per-pixel state stored (final T and last contributor, 8 B per pixel) and with
    transmittance checkpointing (recomputed in the backward, nothing stored per pixel)."""
    import torch

    from omnigs_b200 import lonlat, scenes

    P, W, H = 3_000_000, 4096, 2048
    g = scenes.make_gaussians(P, seed=3)
    gt = lonlat.GaussianTensors.from_numpy(g, dev)
    cam = lonlat.Camera.from_view(scenes.identity_view(W, H), dev)
    dpix = torch.from_numpy(scenes.upstream_grad(W, H, seed=3)).to(dev)
    out = {"workload": "3M Gaussians, one 4096x2048 view, fwd+bwd (plain path)"}
    for key, recompute in (("stored_T", False), ("recompute_T", True)):
        torch.cuda.synchronize()
        torch.cuda.empty_cache()
        base = torch.cuda.memory_allocated(dev)
        torch.cuda.reset_peak_memory_stats(dev)
        img, radii, n, state = lonlat.rasterize(gt, cam, capacity=1, recompute_T=recompute)  # exact sizing
        grads = lonlat.Gradients.empty(P, 16, dev)
        state.backward(gt, cam, radii, dpix, grads, R=n)
        torch.cuda.synchronize()
        peak = torch.cuda.max_memory_allocated(dev) - base
        out["num_rendered"] = int(n)
        out[key] = {"peak_bytes_above_inputs": int(peak), "peak_gb": round(peak / 1e9, 3),
                    "image_state_bytes": int(state.image.numel())}
        del state, grads, img, radii
    out["per_pixel_state_bytes"] = 8 * W * H
    del gt
    torch.cuda.empty_cache()
    return out


def run_checkpointing(args, gt, cam, dpix, n0, dev):
    """Headline view (1M Gaussians, 2048x1024) fwd+bwd with transmittance checkpointing: the forward
    stores no per-pixel state and the backward replays the forward's recurrence per tile."""
    import torch

    from omnigs_b200 import lonlat

    P, W, H = gt.P, cam.width, cam.height
    out = {}
    for key, recompute in (("stored_T_ms_per_view", False), ("recompute_T_ms_per_view", True)):
        state = lonlat.LonlatState(P, W, H, n0 + n0 // 8 + 4096, dev, recompute_T=recompute)
        img = torch.empty(3, H, W, device=dev)
        radii = torch.empty(P, dtype=torch.int32, device=dev)
        grads = lonlat.Gradients.empty(P, 16, dev)

        def step():
            state.forward(gt, cam, img, radii)
            state.backward(gt, cam, radii, dpix, grads)

        out[key] = _time_steps(step, args, dev)
        del state, grads, img, radii
    torch.cuda.empty_cache()
    out["saved_bytes_per_pixel"] = 8
    return out


def run_differentiation(args, dev):
    """Differentiation configuration: a perturbed copy of a 500k-Gaussian scene (means + N(0, 0.02 m),
    SH + N(0, 0.1)) optimised for 500 Adam steps on L1 + 0.2 D-SSIM towards 24 target views at
    2048x1024 (camera positions uniform in a 2 m cube, random yaw), one view per step in a seeded
    random order per pass over the views, as the reference's trainer picks keyframes
    (src/gaussian_mapper.cpp:384-432).  Each step runs through the LibTorch autograd Function:
    GaussianRasterizer forward, the fused L1 + D-SSIM kernel for dL/dimage, image.backward() (the
    C++ Function's backward, RasterizeGaussiansBackwardCUDA), fused Adam on the activated-value
    gradients.  The targets are rendered from the unperturbed scene by the same rasterizer."""
    import torch

    from omnigs_b200 import GaussianRasterizationSettings, GaussianRasterizer, lonlat, scenes, train

    P, W, H, V, STEPS = 500_000, 2048, 1024, 24, 500
    gt_scene = scenes.make_gaussians(P, seed=6)
    views = scenes.random_views(V, [(W, H)], seed=7, cube=2.0, pitch_deg=0.0)
    cams = [lonlat.Camera.from_view(v, dev) for v in views]
    gtt = lonlat.GaussianTensors.from_numpy(gt_scene, dev)
    targets = []
    for c in cams:
        img, _, _, st = lonlat.rasterize(gtt, c)
        targets.append(img.clone())
        del st
    del gtt
    rng = np.random.Generator(np.random.PCG64(8))
    pert = scenes.Gaussians(
        (gt_scene.means3D + rng.normal(0.0, 0.02, gt_scene.means3D.shape)).astype(np.float32),
        gt_scene.scales.copy(), gt_scene.rotations.copy(), gt_scene.opacities.copy(),
        (gt_scene.shs + rng.normal(0.0, 0.1, gt_scene.shs.shape)).astype(np.float32))
    model = train.GaussianModelState.from_activated(pert, device=dev)
    settings = [GaussianRasterizationSettings(H, W, 0.0, 0.0, c.background, 1.0, c.viewmatrix, c.viewmatrix, 3,
                                              c.campos) for c in cams]
    order = np.concatenate([rng.permutation(V) for _ in range((STEPS + V - 1) // V)])[:STEPS]
    losses = torch.zeros(STEPS, 3, device=dev)
    loss_ws = train.l1_dssim_workspace(3, H, W, dev)

    def render(i, leaves):
        return GaussianRasterizer(settings[i])(leaves[0], leaves[1], leaves[2], shs=leaves[3], scales=leaves[4],
                                               rotations=leaves[5])[0]

    def psnr_all():
        t = model.tensors()
        vals = []
        with torch.no_grad():
            for i in range(V):
                img = render(i, (t.means3D, torch.zeros_like(t.means3D), t.opacities, t.shs, t.scales,
                                 t.rotations))
                mse = float(((img - targets[i]) ** 2).mean())
                vals.append(10.0 * math.log10(1.0 / max(mse, 1e-20)))
        return round(statistics.mean(vals), 3)

    psnr0 = psnr_all()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0 = time.perf_counter()
    e0.record()
    for k in range(STEPS):
        i = int(order[k])
        t = model.tensors()
        leaves = [t.means3D.detach().requires_grad_(True), torch.zeros_like(t.means3D, requires_grad=True),
                  t.opacities.detach().requires_grad_(True), t.shs.detach().requires_grad_(True),
                  t.scales.detach().requires_grad_(True), t.rotations.detach().requires_grad_(True)]
        img = render(i, leaves)
        _, dimg = train.l1_dssim(img.detach(), targets[i], 0.2, loss=losses[k], workspace=loss_ws)
        img.backward(dimg)
        model.adam_step(leaves[0].grad, leaves[3].grad, leaves[2].grad, leaves[4].grad, leaves[5].grad)
    e1.record()
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    ms = e0.elapsed_time(e1) / STEPS
    psnr1 = psnr_all()
    curve = losses[:, 0].cpu().numpy()
    windows = {str(s): round(float(curve[max(0, s - V + 1):s + 1].mean()), 6)
               for s in (V - 1, 49, 99, 199, 299, 399, STEPS - 1)}
    out = {"workload": f"{P} Gaussians (perturbed copy: means + N(0,0.02), SH + N(0,0.1)), {V} target views "
                       f"{W}x{H} from positions uniform in a 2 m cube with random yaw, {STEPS} Adam steps on "
                       "L1 + 0.2 D-SSIM, one view per step, through the LibTorch autograd Function",
           "ms_per_step": round(ms, 4), "wall_s": round(wall, 3), "steps": STEPS,
           "loss_first": round(float(curve[0]), 6), "loss_last": round(float(curve[-1]), 6),
           "loss_mean_of_last_24_views_at_step": windows,
           "psnr_db_mean_over_views": {"before": psnr0, "after": psnr1},
           "adam_step_count": model.step_count}
    del model, targets
    torch.cuda.empty_cache()
    return out


def run_reference_gpu(args):
    """The reference's own CUDA rasterizer rebuilt for sm_100a from its sources (oracle/ref/Makefile)
    on this arm's workload (1M Gaussians, one 2048x1024 view), device-timed like the main line with
    its own clock record: forward + backward of one view per step (its forward copies num_rendered
    to the host mid-pass, as its LibTorch layer does; gradient outputs zero-initialised as that
    layer allocates them).  Plus its peak device memory at the peak-memory workload.  The
    like-for-like GPU comparison; None where the library was not built (no reference checkout at
    build time) or no GPU is visible."""
    import torch

    from omnigs_b200 import lonlat, scenes
    from oracle import refcuda

    if not (refcuda.available() and torch.cuda.is_available()):
        return None
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    g = scenes.make_gaussians(P_GAUSS, seed=0)
    gt = lonlat.GaussianTensors.from_numpy(g, dev)
    cam = lonlat.Camera.from_view(scenes.identity_view(WIDTH, HEIGHT), dev)
    dpix = torch.from_numpy(scenes.upstream_grad(WIDTH, HEIGHT, seed=2)).to(dev)
    gpu_uuid = None
    try:
        gpu_uuid = "GPU-" + str(torch.cuda.get_device_properties(dev).uuid)
    except Exception:
        pass
    ref = refcuda.ReferenceRasterizer()
    out = torch.zeros(3, cam.height, cam.width, device=dev)
    radii = torch.zeros(g.P, dtype=torch.int32, device=dev)
    n = [0]

    def step():
        _, r, n[0] = ref.forward(gt, cam, sync=False, out=out, radii=radii)
        ref.backward(gt, cam, r, dpix, sync=False)

    for _ in range(max(3, args.warmup)):
        step()
    torch.cuda.synchronize()
    cur = torch.cuda.current_stream(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with clock_sampler(gpu_uuid) as clocks:
        e0.record(cur)
        for _ in range(args.steps):
            step()
        e1.record(cur)
        torch.cuda.synchronize()
    ref.close()
    ms = e0.elapsed_time(e1) / args.steps
    del out, radii, gt, dpix
    torch.cuda.empty_cache()
    return {"impl": "reference CUDA rasterizer (cuda_rasterizer/, LonlatRasterizer::forward/backward) rebuilt "
                    "for sm_100a", "workload": WORKLOAD, "ms_per_view": round(ms, 4),
            "views_per_s": round(1000.0 / ms, 3), "steps": args.steps, "warmup": max(3, args.warmup),
            "num_rendered": int(n[0]), "clocks": clocks.summary(),
            "peak_memory": reference_peak_memory(dev)}


def reference_peak_memory(dev):
    """Peak device memory of one fwd+bwd of the rebuilt reference rasterizer at the peak-memory
    workload: its state buffers (cudaMalloc'ed, measured as the drop in free device memory while
    they are held) plus the output and gradient tensors its LibTorch layer would allocate."""
    import torch

    from omnigs_b200 import lonlat, scenes
    from oracle import refcuda

    if not refcuda.available():
        return None
    P, W, H = 3_000_000, 4096, 2048
    g = scenes.make_gaussians(P, seed=3)
    gt = lonlat.GaussianTensors.from_numpy(g, dev)
    cam = lonlat.Camera.from_view(scenes.identity_view(W, H), dev)
    dpix = torch.from_numpy(scenes.upstream_grad(W, H, seed=3)).to(dev)
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    free0 = torch.cuda.mem_get_info(dev)[0]
    reserved0 = torch.cuda.memory_reserved(dev)
    base = torch.cuda.memory_allocated(dev)
    torch.cuda.reset_peak_memory_stats(dev)
    ref = refcuda.ReferenceRasterizer()
    _, radii, n = ref.forward(gt, cam)
    grads = ref.backward(gt, cam, radii, dpix)
    torch.cuda.synchronize()
    free1 = torch.cuda.mem_get_info(dev)[0]
    torch_peak = torch.cuda.max_memory_allocated(dev) - base
    state_bytes = (free0 - free1) - (torch.cuda.memory_reserved(dev) - reserved0)
    ref.close()
    del grads, radii, gt
    torch.cuda.empty_cache()
    peak = state_bytes + torch_peak
    return {"num_rendered": int(n), "peak_bytes_above_inputs": int(peak), "peak_gb": round(peak / 1e9, 3),
            "state_buffers_bytes": int(state_bytes), "per_pixel_state_bytes": 16 * W * H,
            "method": "state buffers from the drop in free device memory + torch peak of outputs and gradients"}


def _time_steps(fn, args, dev):
    import torch

    for _ in range(max(1, args.warmup)):
        fn()
    torch.cuda.synchronize()
    cur = torch.cuda.current_stream(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    k = max(2, args.steps // 4)
    e0.record(cur)
    for _ in range(k):
        fn()
    e1.record(cur)
    torch.cuda.synchronize()
    return round(e0.elapsed_time(e1) / k, 4)


# ---------------------------------------------------------------- omnigs arm --------------------
def run_omnigs(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist

    from omnigs_b200 import capi, lonlat, scenes, torch_ext

    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    g = scenes.make_gaussians(args.gaussians, seed=0)
    view = scenes.identity_view(args.width, args.height)
    dpix_np = scenes.upstream_grad(args.width, args.height, seed=2 + rank)
    gt = lonlat.GaussianTensors.from_numpy(g, dev)
    cam = lonlat.Camera.from_view(view, dev)
    dpix = torch.from_numpy(dpix_np).to(dev)
    P, W, H = g.P, args.width, args.height

    # sizing pass (untimed): exact instance count, then a fixed capacity for the timed steps
    _, radii0, n0, _ = lonlat.rasterize(gt, cam)
    V = int((radii0 > 0).sum())
    capacity = n0 + n0 // 8 + 4096
    state = lonlat.LonlatState(P, W, H, capacity, dev)
    out = torch.empty(3, H, W, device=dev)
    radii = torch.empty(P, dtype=torch.int32, device=dev)
    # one flat buffer holds every gradient output, so N > 1 reduces it with a single all-reduce
    sizes = [P * 3, P * 3, P, P * 3, P * 6, P * 16 * 3, P * 3, P * 4]
    flat = torch.empty(sum(sizes), device=dev)
    parts = torch.split(flat, sizes)
    grads = lonlat.Gradients(parts[0].view(P, 3), parts[1].view(P, 3), parts[2].view(P, 1),
                             parts[3].view(P, 3), parts[4].view(P, 6), parts[5].view(P, 16, 3),
                             parts[6].view(P, 3), parts[7].view(P, 4))

    def step():
        state.forward(gt, cam, out, radii)
        state.backward(gt, cam, radii, dpix, grads)
        if world > 1:
            dist.all_reduce(flat)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    nr, st = state.status()
    assert st == 0 and nr == n0, (nr, st)

    gpu_uuid = None
    try:
        gpu_uuid = "GPU-" + str(torch.cuda.get_device_properties(dev).uuid)
    except Exception:
        pass
    stream = torch.cuda.current_stream(dev)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = capi.kernel_launches()
    with clock_sampler(gpu_uuid) as clocks:
        ev0.record(stream)
        for _ in range(args.steps):
            step()
        ev1.record(stream)
        torch.cuda.synchronize()
    launches = capi.kernel_launches() - launches0
    if world > 1:
        dist.barrier()
    ms_total = ev0.elapsed_time(ev1)
    if world > 1:
        t = torch.tensor([ms_total], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_total = float(t.item())
    ms_per_step = ms_total / args.steps
    value = world * args.steps / (ms_total / 1000.0)

    # ---- per-kernel device times (library event timing) for the roofline ----
    capi.timing_enable(True)
    for _ in range(args.steps):
        step()
    torch.cuda.synchronize()
    stages = capi.timing_read()
    capi.timing_enable(False)
    iv = state.image_view()
    pairs_bwd = int(iv["n_contrib"].to(torch.int64).sum())
    Tl = ((W + 15) // 16) * ((H + 15) // 16)
    sbytes = stage_bytes(P, V, n0, W * H, Tl)
    hbm_peak, sm_max_mhz, peak_kind = measured_peaks()
    traffic = traffic_from_profiles()
    kernels = {}
    for name, nbytes in sbytes.items():
        ms, nl = stages[name]
        if nl == 0:
            continue
        per_step_ms = ms / args.steps
        kernels[name] = {"ms_per_step": round(per_step_ms, 4), "launches_per_step": nl // args.steps,
                         "algorithmic_bytes": nbytes, "GBps": round(nbytes / (per_step_ms * 1e-3) / 1e9, 1)}
    dominant = max(kernels, key=lambda k: kernels[k]["ms_per_step"])
    dk = kernels[dominant]
    launch_ms = stages[dominant][0] / max(stages[dominant][1], 1)
    bytes_per_launch = sbytes[dominant] / max(dk["launches_per_step"], 1)
    achieved = bytes_per_launch / (launch_ms * 1e-3) / 1e9
    roofline = {"bound": "hbm", "kernel": dominant, "achieved": round(achieved, 1), "peak": hbm_peak,
                "unit": "GB/s", "frac": round(achieved / hbm_peak, 4),
                "traffic": traffic.get(dominant), "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)"}
    fp32_peak = 148 * 128 * 2 * sm_max_mhz * 1e6 / 1e12
    flops_fwd = pairs_bwd * 24
    flops_bwd = pairs_bwd * 64
    rf = {}
    for k, fl in (("render_forward", flops_fwd), ("render_backward", flops_bwd)):
        if k in kernels:
            tf = fl / (kernels[k]["ms_per_step"] * 1e-3) / 1e12
            rf[k] = {"achieved_tflops": round(tf, 2), "frac": round(tf / fp32_peak, 4), "pairs": pairs_bwd,
                     "flops_per_pair": 24 if k == "render_forward" else 64}
    roofline_fp32 = {"bound": "fp32", "peak_tflops": round(fp32_peak, 1),
                     "peak_source": "nominal 148 SM x 128 FP32 lanes x 2 x sm_max_mhz", **rf}
    # whole-path roofline: each stage's lower-bound time (its algorithmic bytes at the HBM peak, or
    # for the blends its FP32 work at the FP32 peak, whichever is longer) summed over the stages,
    # over the measured step time
    stage_flops = {"render_forward": flops_fwd, "render_backward": flops_bwd}
    bound_ms = {k: max(sbytes[k] / (hbm_peak * 1e9), stage_flops.get(k, 0) / (fp32_peak * 1e12)) * 1e3
                for k in kernels}
    path_roofline = {"frac": round(sum(bound_ms.values()) / ms_per_step, 4),
                     "bound_ms_per_step": round(sum(bound_ms.values()), 4), "measured_ms_per_step": round(ms_per_step, 4),
                     "stage_bound_ms": {k: round(v, 4) for k, v in bound_ms.items()},
                     "formula": "sum over stages of max(algorithmic bytes / HBM peak, FP32 flops / FP32 peak), "
                                "over the measured fwd+bwd step time"}

    # ---- end to end through the reference-facing LibTorch API with host buffers ----
    e2e = None
    if not args.no_e2e:
        ext = torch_ext()
        h_dpix = torch.from_numpy(dpix_np).pin_memory()
        h_view = torch.from_numpy(view.viewmatrix).pin_memory()
        h_campos = torch.from_numpy(view.campos).pin_memory()
        h_bg = torch.zeros(3).pin_memory()
        empty = torch.empty(0, device=dev)
        # Pipelined like a training loop would be: step k+1's inputs are copied host->device on one
        # copy stream while step k computes, and step k's image is copied device->host on another
        # as soon as its forward is done.  Every step still moves its own inputs and result.
        copy_in, copy_out = torch.cuda.Stream(dev), torch.cuda.Stream(dev)
        slots = [(torch.empty_like(dpix), torch.empty(4, 4, device=dev), torch.empty(3, device=dev),
                  torch.empty(3, device=dev)) for _ in range(2)]
        h_img = [torch.empty(3, H, W).pin_memory() for _ in range(2)]
        in_ready = [torch.cuda.Event() for _ in range(2)]

        def h2d(k):
            d_dpix, d_view, d_campos, d_bg = slots[k % 2]
            with torch.cuda.stream(copy_in):
                d_dpix.copy_(h_dpix, non_blocking=True)
                d_view.copy_(h_view, non_blocking=True)
                d_campos.copy_(h_campos, non_blocking=True)
                d_bg.copy_(h_bg, non_blocking=True)
                in_ready[k % 2].record(copy_in)

        def e2e_step(k, last):
            d_dpix, d_view, d_campos, d_bg = slots[k % 2]
            stream.wait_event(in_ready[k % 2])
            n, color, rad, gb, bb, ib = ext.rasterize_gaussians_cuda(
                d_bg, gt.means3D, empty, gt.opacities, gt.scales, gt.rotations, 1.0, empty, d_view, d_view,
                0.0, 0.0, H, W, gt.shs, 3, d_campos, False, 3, False)
            # the forward returned once this step's binning had run on the compute stream, which
            # follows step k-1's backward (the last reader of the other slot): prefetch step k+1's
            # inputs into it
            if not last:
                h2d(k + 1)
            img_ready = torch.cuda.Event()
            img_ready.record(stream)
            with torch.cuda.stream(copy_out):
                copy_out.wait_event(img_ready)
                h_img[k % 2].copy_(color, non_blocking=True)
                color.record_stream(copy_out)
            ext.rasterize_gaussians_backward_cuda(
                d_bg, gt.means3D, rad, empty, gt.scales, gt.rotations, 1.0, empty, d_view, d_view, 0.0, 0.0,
                d_dpix, gt.shs, 3, d_campos, gb, n, bb, ib, 3)

        def run_pipeline(steps):
            copy_in.wait_stream(stream)
            h2d(0)
            for k in range(steps):
                e2e_step(k, k == steps - 1)
            stream.wait_stream(copy_out)

        run_pipeline(max(2, args.warmup))
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        run_pipeline(args.steps)
        e1.record(stream)
        torch.cuda.synchronize()
        ems = e0.elapsed_time(e1)
        if world > 1:
            t = torch.tensor([ems], device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ems = float(t.item())
        e2e = {"value": world * args.steps / (ems / 1000.0), "unit": UNIT,
               "h2d_bytes_per_step": int(h_dpix.numel() * 4 + 16 * 4 + 3 * 4 + 3 * 4),
               "d2h_bytes_per_step": int(h_img[0].numel() * 4 + 4),
               "api": "RasterizeGaussiansCUDA + RasterizeGaussiansBackwardCUDA (LibTorch layer)",
               "copies": "pinned host buffers; next step's inputs and this step's image copied on two copy "
                         "streams, overlapped with compute"}

    batched = None
    extra = None
    headline = (P, W, H) == (P_GAUSS, WIDTH, HEIGHT)
    if world == 1 and not args.no_batch and headline:
        batched = run_batched(args, g, gt, dev, value)
    if world == 1 and not args.no_extra and headline:
        extra = {"precision": run_precision(args, dev), "peak_memory": run_peak_memory(dev),
                 "checkpointing": run_checkpointing(args, gt, cam, dpix, n0, dev),
                 "differentiation": run_differentiation(args, dev)}


    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(g, view, dpix_np)

    if rank == 0:
        workload = WORKLOAD if (P, W, H) == (P_GAUSS, WIDTH, HEIGHT) else \
            f"profiling case: {P} Gaussians, {W}x{H} (not a bench line)"
        line = {"metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_per_step, 4),
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic (seeded generators of the reference's config shapes)",
                "config": {"workload": workload, "gaussians": P, "width": W, "height": H,
                           "num_rendered": n0, "visible": V, "parallelism": f"dp{world} (views)",
                           "l2": "inputs larger than L2 (SH alone 192 MB > 126 MB), no flush"},
                "gpu_launches": int(launches), "clocks": clocks.summary(), "roofline": roofline,
                "roofline_fp32": roofline_fp32, "path_roofline": path_roofline, "kernels": kernels, "e2e": e2e,
                "batched": batched, "configs": extra, "cpu_baseline": cpu}
        print(json.dumps(line), flush=True)


def main():
    args = parse()
    rank, world, local_rank = dist_env()
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        # bind this rank's GPU before NCCL sets up its communicator
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))
    try:
        run_omnigs(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
