"""TEST INFRASTRUCTURE ONLY: like-for-like speed of the reference CUDA rasterizer (rebuilt for
sm_100a from its own sources, oracle/_ref/libomnigs_ref.so) and omnigs_b200 on the same scene,
view and GPU.  Both arms run forward + backward of one view per step with device-resident
inputs, timed with CUDA events over K steps after W warm-up steps:

* reference: CudaRasterizer::LonlatRasterizer::forward (which copies num_rendered to the host
  mid-pass) + zero-initialised gradient outputs, as its LibTorch layer allocates them, + ::backward;
* omnigs_b200: omnigs_lonlat_forward + omnigs_lonlat_backward through the C ABI.

    python oracle/ref/compare_speed.py [--gaussians P] [--width W] [--height H] [--steps K]
"""
import argparse
import json
import os
import sys

import torch

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import refcuda  # noqa: E402
from omnigs_b200 import lonlat, scenes  # noqa: E402


def timed(step, steps, warmup):
    for _ in range(warmup):
        step()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        step()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gaussians", type=int, default=1_000_000)
    ap.add_argument("--width", type=int, default=2048)
    ap.add_argument("--height", type=int, default=1024)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    a = ap.parse_args()
    g = scenes.make_gaussians(a.gaussians, seed=0)
    gt = lonlat.GaussianTensors.from_numpy(g)
    cam = lonlat.Camera.from_view(scenes.identity_view(a.width, a.height))
    dpix = torch.from_numpy(scenes.upstream_grad(a.width, a.height)).cuda()

    ref = refcuda.ReferenceRasterizer()
    out = torch.zeros(3, a.height, a.width, device="cuda")
    radii = torch.zeros(g.P, dtype=torch.int32, device="cuda")

    def ref_step():
        _, r, _ = ref.forward(gt, cam, sync=False, out=out, radii=radii)
        ref.backward(gt, cam, r, dpix, sync=False)

    ref_ms = timed(ref_step, a.steps, a.warmup)
    ref.close()

    _, _, n, _ = lonlat.rasterize(gt, cam)
    state = lonlat.LonlatState(g.P, a.width, a.height, n + n // 8 + 4096)
    grads = lonlat.Gradients.empty(g.P, 16, "cuda")

    def our_step():
        state.forward(gt, cam, out, radii)
        state.backward(gt, cam, radii, dpix, grads)

    our_ms = timed(our_step, a.steps, a.warmup)
    print(json.dumps({"workload": f"{g.P} Gaussians, {a.width}x{a.height}, fwd+bwd per view",
                      "reference_ms_per_view": round(ref_ms, 4), "omnigs_ms_per_view": round(our_ms, 4),
                      "reference_views_per_s": round(1000 / ref_ms, 2),
                      "omnigs_views_per_s": round(1000 / our_ms, 2),
                      "speedup": round(ref_ms / our_ms, 3), "num_rendered": n}))


if __name__ == "__main__":
    main()
