"""The LibTorch autograd path (GaussianRasterizer -> the C++ torch::autograd::Function ->
RasterizeGaussiansCUDA / RasterizeGaussiansBackwardCUDA) against FP64 central finite differences.

The differentiation configuration's check: a 1,000-Gaussian scene with the benchmark's generators,
one posed 256x128 equirect view, L = <dL/dpix, image> with dL/dpix ~ N(0, 1).  The GPU gradients
of means3D, scales, rotations, opacities and SH come from `.backward()` through the autograd
Function; each sampled parameter's derivative is also taken by FP64 central differences of the
oracle's forward (the reference's forward formulas in double precision), with the step rounded to
the float32 inputs.  Every sampled parameter must agree within 1e-3 relative, relative to
max(|fd|, |autograd|, 1e-3 max|gradient of that parameter field|) so that near-zero derivatives
are not judged on their rounding noise.  (On this scene the FP64 analytic backward of the oracle
meets the same differences within ~6e-5, so the bar measures the GPU path.)
"""
import numpy as np
import pytest
import torch

import oracle
from omnigs_b200 import GaussianRasterizationSettings, GaussianRasterizer, lonlat, scenes

pytestmark = pytest.mark.gpu

REL_TOL = 1e-3


def test_autograd_gradients_match_fp64_central_differences(cuda):
    W, H = 256, 128
    g = scenes.make_gaussians(1000, seed=5)
    v = scenes.make_view(W, H, (0.3, -0.2, 0.1), scenes.rotation_yaw_pitch(0.7, 0.0))
    dpix_np = scenes.upstream_grad(W, H, seed=5)
    cam = lonlat.Camera.from_view(v)
    settings = GaussianRasterizationSettings(H, W, 0.0, 0.0, cam.background, 1.0, cam.viewmatrix,
                                             cam.viewmatrix, 3, cam.campos)
    params = {f: torch.from_numpy(np.ascontiguousarray(getattr(g, f))).cuda().requires_grad_(True)
              for f in ("means3D", "scales", "rotations", "opacities", "shs")}
    means2D = torch.zeros_like(params["means3D"], requires_grad=True)
    color, radii = GaussianRasterizer(settings)(
        params["means3D"], means2D, params["opacities"], shs=params["shs"],
        scales=params["scales"], rotations=params["rotations"])
    (color * torch.from_numpy(dpix_np).cuda()).sum().backward()
    torch.cuda.synchronize()
    assert float(means2D.grad.abs().max()) > 0.0

    def loss(gs):
        out = oracle.forward_backward(gs, v, dpix_np)
        return float((out["image"] * dpix_np).sum())

    vis = np.nonzero(radii.cpu().numpy() > 0)[0]
    assert len(vis) > 500
    sel = np.random.default_rng(0).choice(vis, 25, replace=False)
    report = {}
    for field, eps in (("means3D", 1e-4), ("scales", 2e-5), ("rotations", 1e-4),
                       ("opacities", 1e-5), ("shs", 1e-4)):
        arr = getattr(g, field)
        flat = arr.reshape(arr.shape[0], -1)
        ana_all = params[field].grad.detach().double().cpu().numpy().reshape(arr.shape[0], -1)
        floor = 1e-3 * np.abs(ana_all).max()
        errs = []
        for i in sel:
            for k in range(min(flat.shape[1], 8)):
                orig = flat[i, k]
                step = np.float32(eps) * max(np.float32(1.0), abs(orig))
                flat[i, k] = orig + step
                hi = float(flat[i, k])
                lp = loss(g)
                flat[i, k] = orig - step
                lo = float(flat[i, k])
                lm = loss(g)
                flat[i, k] = orig
                fd = (lp - lm) / (hi - lo)
                ana = ana_all[i, k]
                errs.append(abs(fd - ana) / max(abs(fd), abs(ana), floor))
        report[field] = float(np.max(errs))
    assert all(e <= REL_TOL for e in report.values()), report
