"""GPU comparison with the reference CUDA rasterizer itself, rebuilt for sm_100a from its own
sources (oracle/ref/Makefile -> oracle/_ref/libomnigs_ref.so).

Integer stages are compared bit for bit: radii, tiles_touched, inclusive offsets, num_rendered,
sorted keys, point list, tile ranges and last-contributor indices.  Float outputs: the image
within 1e-4 absolute (the blend evaluates the reference's expressions, so it is expected to be
identical), gradients within 1e-3 normwise relative (the reference accumulates with
order-nondeterministic float atomics).
"""
import numpy as np
import pytest
import torch

import helpers
from omnigs_b200 import lonlat, scenes

refcuda = pytest.importorskip("oracle.refcuda")

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not refcuda.available(), reason="reference rasterizer not built")]


def _compare(P, W, H, seed, view=None, bg=(0.0, 0.0, 0.0), pole_fraction=0.0):
    g = scenes.make_gaussians(P, seed=seed, pole_fraction=pole_fraction)
    v = view or scenes.identity_view(W, H)
    gt = lonlat.GaussianTensors.from_numpy(g)
    cam = lonlat.Camera.from_view(v, background=bg)
    dpix = torch.from_numpy(scenes.upstream_grad(W, H, seed=seed)).cuda()
    cu = helpers.run_cuda(gt, cam, dpix)
    ref = refcuda.ReferenceRasterizer()
    r_img, r_radii, r_n = ref.forward(gt, cam)
    rs = ref.state()
    r_grads = ref.backward(gt, cam, r_radii, dpix)
    ref.close()

    # ---- integer stages: bit-exact ----
    torch.testing.assert_close(cu["radii"], r_radii, rtol=0, atol=0)
    assert cu["num_rendered"] == r_n
    torch.testing.assert_close(cu["tiles_touched"], rs["tiles_touched"], rtol=0, atol=0)
    torch.testing.assert_close(torch.cumsum(cu["tiles_touched"].to(torch.int64), 0).to(torch.int32),
                               rs["point_offsets"], rtol=0, atol=0)
    torch.testing.assert_close(cu["keys"], rs["keys"], rtol=0, atol=0)
    torch.testing.assert_close(cu["point_list"], rs["point_list"], rtol=0, atol=0)
    torch.testing.assert_close(cu["ranges"], rs["ranges"], rtol=0, atol=0)
    torch.testing.assert_close(cu["n_contrib"], rs["n_contrib"], rtol=0, atol=0)
    # ---- float outputs ----
    vis = cu["radii"] > 0
    torch.testing.assert_close(cu["means2D"][vis], rs["means2D"][vis], rtol=0, atol=0)
    torch.testing.assert_close(cu["depths"][vis], rs["depths"][vis], rtol=0, atol=0)
    torch.testing.assert_close(cu["conic_opacity"][vis], rs["conic_opacity"][vis], rtol=0, atol=0)
    torch.testing.assert_close(cu["rgb"][vis], rs["rgb"][vis], rtol=0, atol=1e-6)
    img_err = float((cu["image"] - r_img).abs().max())
    assert img_err <= 1e-4, img_err
    torch.testing.assert_close(cu["final_T"], rs["final_T"], rtol=0, atol=1e-6)
    gr = cu["grads"]
    for name in ("dL_dmeans2D", "dL_dcolors", "dL_dopacity", "dL_dmeans3D", "dL_dcov3D", "dL_dsh",
                 "dL_dscales", "dL_drotations"):
        e = helpers.normwise_rel(helpers.to_np(getattr(gr, name)), helpers.to_np(r_grads[name]))
        assert e < 1e-3, (name, e)
    return img_err


def test_small_config_matches_reference(cuda):
    _compare(10_000, 512, 256, seed=0)


def test_posed_view_odd_size_and_background(cuda):
    v = scenes.make_view(500, 250, (0.3, 0.1, -0.2), scenes.rotation_yaw_pitch(-1.1, 0.4))
    _compare(10_000, 500, 250, seed=1, view=v, bg=(0.2, 0.4, 0.6))


def test_pole_heavy_scene_matches_reference(cuda):
    _compare(20_000, 1024, 512, seed=2, pole_fraction=0.3)


def test_full_size_matches_reference(cuda):
    """1M Gaussians, 2048 x 1024, identity pose: the headline workload."""
    _compare(1_000_000, 2048, 1024, seed=0)


@pytest.mark.parametrize("P,W,H", [(10_000, 512, 256), (1_000_000, 2048, 1024)])
def test_autograd_layer_matches_reference(cuda, P, W, H):
    """The reference-facing LibTorch surface as a trainer uses it: GaussianRasterizer (the C++
    torch::autograd::Function over RasterizeGaussiansCUDA / RasterizeGaussiansBackwardCUDA),
    `.backward()` of <dL/dpix, image>, against the reference rasterizer's forward and backward.
    Every input gradient is compared, including the viewspace-point gradient means2D.grad that the
    trainer's densification reads (src/gaussian_renderer.cpp:184-191)."""
    from omnigs_b200 import GaussianRasterizationSettings, GaussianRasterizer

    g = scenes.make_gaussians(P, seed=7)
    v = scenes.make_view(W, H, (0.2, -0.1, 0.15), scenes.rotation_yaw_pitch(0.4, -0.2))
    gt = lonlat.GaussianTensors.from_numpy(g)
    cam = lonlat.Camera.from_view(v, background=(0.3, 0.2, 0.1))
    dpix = torch.from_numpy(scenes.upstream_grad(W, H, seed=7)).cuda()
    ref = refcuda.ReferenceRasterizer()
    r_img, r_radii, _ = ref.forward(gt, cam)
    r_grads = ref.backward(gt, cam, r_radii, dpix)
    ref.close()

    settings = GaussianRasterizationSettings(H, W, 0.0, 0.0, cam.background, 1.0, cam.viewmatrix,
                                             cam.viewmatrix, 3, cam.campos)
    leaves = {k: getattr(gt, k).clone().requires_grad_(True)
              for k in ("means3D", "opacities", "shs", "scales", "rotations")}
    means2D = torch.zeros_like(leaves["means3D"], requires_grad=True)
    color, radii = GaussianRasterizer(settings)(leaves["means3D"], means2D, leaves["opacities"],
                                                shs=leaves["shs"], scales=leaves["scales"],
                                                rotations=leaves["rotations"])
    (color * dpix).sum().backward()
    torch.cuda.synchronize()
    torch.testing.assert_close(radii, r_radii, rtol=0, atol=0)
    assert float((color.detach() - r_img).abs().max()) <= 1e-4
    pairs = [(means2D.grad, "dL_dmeans2D"), (leaves["means3D"].grad, "dL_dmeans3D"),
             (leaves["opacities"].grad, "dL_dopacity"), (leaves["shs"].grad, "dL_dsh"),
             (leaves["scales"].grad, "dL_dscales"), (leaves["rotations"].grad, "dL_drotations")]
    for got, name in pairs:
        e = helpers.normwise_rel(helpers.to_np(got), helpers.to_np(r_grads[name]))
        assert e < 1e-3, (name, e)
