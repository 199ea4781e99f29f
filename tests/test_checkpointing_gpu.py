"""Transmittance checkpointing (OMNIGS_FLAG_RECOMPUTE_T) against the stored per-pixel state.

With the flag, the forward keeps no per-pixel state (the image buffer holds only the tile ranges)
and the backward blend first replays the forward's front-to-back recurrence for each tile to
recompute every pixel's final transmittance and last contributor.  The replay is the forward's own
code without colour, so those values are the ones the forward would have stored, and the image and
gradients must equal the stored mode's: the image bit for bit, the gradients to the run-to-run
variation of the blend's float atomics (1e-5 normwise).  Checked through the C ABI (small view and
the 1M-Gaussian 2048x1024 headline view, with a background) and through the LibTorch layer.
"""
import pytest
import torch

import helpers
from omnigs_b200 import GaussianRasterizationSettings, GaussianRasterizer, capi, lonlat, scenes, torch_ext

pytestmark = pytest.mark.gpu

GRADS = ("dL_dmeans2D", "dL_dcolors", "dL_dopacity", "dL_dmeans3D", "dL_dcov3D", "dL_dsh", "dL_dscales",
         "dL_drotations")


def _fwd_bwd(gt, cam, dpix, recompute):
    P, W, H = gt.P, cam.width, cam.height
    _, _, n, _ = lonlat.rasterize(gt, cam)
    state = lonlat.LonlatState(P, W, H, n + 1024, recompute_T=recompute)
    out = torch.empty(3, H, W, device="cuda")
    radii = torch.empty(P, dtype=torch.int32, device="cuda")
    state.forward(gt, cam, out, radii)
    grads = lonlat.Gradients.empty(P, gt.M, "cuda")
    state.backward(gt, cam, radii, dpix, grads)
    n2, st = state.status()
    assert st == 0 and n2 == n
    return out, radii, grads, state.image.numel()


@pytest.mark.parametrize("P,W,H", [(20_000, 512, 256), (1_000_000, 2048, 1024)])
def test_recomputed_transmittance_equals_stored(cuda, P, W, H):
    g = scenes.make_gaussians(P, seed=61)
    gt = lonlat.GaussianTensors.from_numpy(g)
    v = scenes.make_view(W, H, (0.1, 0.2, -0.1), scenes.rotation_yaw_pitch(-0.6, 0.3))
    cam = lonlat.Camera.from_view(v, background=(0.2, 0.1, 0.3))
    dpix = torch.from_numpy(scenes.upstream_grad(W, H, seed=61)).cuda()
    img0, radii0, g0, bytes0 = _fwd_bwd(gt, cam, dpix, recompute=False)
    img1, radii1, g1, bytes1 = _fwd_bwd(gt, cam, dpix, recompute=True)
    assert bytes1 < bytes0 and bytes0 - bytes1 >= 8 * W * H
    assert torch.equal(radii0, radii1)
    assert torch.equal(img0, img1)
    for name in GRADS:
        e = helpers.normwise_rel(helpers.to_np(getattr(g1, name)), helpers.to_np(getattr(g0, name)))
        assert e < 1e-5, (name, e)


def test_recompute_through_the_libtorch_layer(cuda):
    W, H, P = 512, 256, 20_000
    g = scenes.make_gaussians(P, seed=62)
    gt = lonlat.GaussianTensors.from_numpy(g)
    cam = lonlat.Camera.from_view(scenes.identity_view(W, H))
    dpix = torch.from_numpy(scenes.upstream_grad(W, H, seed=62)).cuda()
    settings = GaussianRasterizationSettings(H, W, 0.0, 0.0, cam.background, 1.0, cam.viewmatrix,
                                             cam.viewmatrix, 3, cam.campos)
    ext = torch_ext()
    results = {}
    try:
        for mode in (False, True):
            ext.set_recompute_transmittance(mode)
            leaves = {k: getattr(gt, k).clone().requires_grad_(True)
                      for k in ("means3D", "opacities", "shs", "scales", "rotations")}
            means2D = torch.zeros_like(leaves["means3D"], requires_grad=True)
            color, _ = GaussianRasterizer(settings)(leaves["means3D"], means2D, leaves["opacities"],
                                                    shs=leaves["shs"], scales=leaves["scales"],
                                                    rotations=leaves["rotations"])
            (color * dpix).sum().backward()
            torch.cuda.synchronize()
            results[mode] = (color.detach(), means2D.grad, *[leaves[k].grad for k in leaves])
            # the image buffer the forward returns
            empty = torch.empty(0, device="cuda")
            out = ext.rasterize_gaussians_cuda(cam.background, gt.means3D, empty, gt.opacities, gt.scales,
                                               gt.rotations, 1.0, empty, cam.viewmatrix, cam.viewmatrix, 0.0, 0.0,
                                               H, W, gt.shs, 3, cam.campos, False, 3, False)
            assert out[5].numel() == capi.image_bytes(W, H, capi.FLAG_RECOMPUTE_T if mode else 0)
    finally:
        ext.set_recompute_transmittance(False)
    assert torch.equal(results[False][0], results[True][0])
    for a, b in zip(results[False][1:], results[True][1:]):
        assert helpers.normwise_rel(helpers.to_np(b), helpers.to_np(a)) < 1e-5
