"""The FP64 oracle pinned directly to the reference rasterizer (rebuilt from its own sources for
sm_100a by oracle/ref/Makefile), with no CUDA path of this package in between.

The reference ships no tests or golden vectors, so its own outputs on seeded scenes are the pin.
Every oracle stage is fed with the reference's float intermediates of the previous stage, so each
stage is judged on its own:

* preprocess (FP64 throughout): radii may differ only where the FP32 and FP64 evaluations of
  ceil(3 sqrt(lambda)) straddle an integer (counted, at most 0.1 %); means2D within 2e-3 px
  divided by cos(latitude) (atan2 and asin lose FP32 accuracy as 1/cos(latitude) towards the
  poles), depth, conic (below 80 deg latitude) and colour to FP32 accuracy;
* binning (float tile rects from the reference's float means2D): keys, point list and ranges
  bit-exact;
* forward blend (FP64 accumulation against the reference's FP32 over up to hundreds of splats per
  pixel): image within 1e-4 at the 99.99th percentile and 1e-3 at most, last contributors equal on
  all but 0.1 % of the pixels (a transmittance or alpha test that FP32 and FP64 decide differently);
* backward blend and backward preprocess (fed the reference's final transmittance, last
  contributors and screen-space gradients): gradients within 1e-3 normwise relative (the
  backward preprocess below 85 deg latitude, and within 1e-3 L2-relative over all Gaussians).
"""
import numpy as np
import pytest
import torch

import helpers
import oracle
from omnigs_b200 import lonlat, scenes

refcuda = pytest.importorskip("oracle.refcuda")

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not refcuda.available(), reason="reference rasterizer not built")]

np_ = helpers.to_np


def _pin(P, W, H, seed, view=None, bg=(0.0, 0.0, 0.0), pole_fraction=0.0):
    g = scenes.make_gaussians(P, seed=seed, pole_fraction=pole_fraction)
    v = view or scenes.identity_view(W, H)
    gt = lonlat.GaussianTensors.from_numpy(g)
    cam = lonlat.Camera.from_view(v, background=bg)
    dpix_np = scenes.upstream_grad(W, H, seed=seed)
    ref = refcuda.ReferenceRasterizer()
    r_img, r_radii, R = ref.forward(gt, cam)
    rs = ref.state()
    r_grads = ref.backward(gt, cam, r_radii, torch.from_numpy(dpix_np).cuda())
    ref.close()
    bg_np = np.asarray(bg, np.float32)

    # ---- preprocess, FP64 ----
    pre = oracle.preprocess(g.means3D, g.scales, g.rotations, g.opacities, g.shs, v.viewmatrix,
                            v.campos, W, H)
    radii = np_(r_radii)
    mism = int((pre["radii"] != radii).sum())
    assert mism <= max(2, P // 1000), f"{mism} radii differ from the reference"
    both = (pre["radii"] > 0) & (radii > 0)
    m2_ref = np_(rs["means2D"]).astype(np.float64)
    lat = (0.5 - (m2_ref[:, 1] + 0.5) / H) * np.pi  # latitude of the projected centre
    coslat = np.maximum(np.cos(lat), 1e-4)[:, None]
    assert (np.abs(pre["means2D"] - m2_ref)[both] * coslat[both]).max() < 2e-3
    np.testing.assert_allclose(pre["depths"][both], np_(rs["depths"])[both], rtol=1e-6)
    ok = both & (np.abs(lat) < np.radians(80.0))
    con_r = np_(rs["conic_opacity"]).astype(np.float64)[ok]
    con_o = pre["conic_opacity"][ok]
    assert (np.abs(con_o[:, :3] - con_r[:, :3]) / np.abs(con_r[:, :3]).max(1, keepdims=True)).max() < 1e-3
    np.testing.assert_array_equal(con_o[:, 3], con_r[:, 3])
    np.testing.assert_allclose(pre["rgb"][both], np_(rs["rgb"])[both], atol=2e-5)
    assert (pre["clamped"][both] != np_(rs["clamped"])[both]).mean() < 1e-3

    # ---- binning, from the reference's float intermediates: bit-exact ----
    m2 = np_(rs["means2D"]).astype(np.float32)
    b = oracle.binning(W, H, radii, m2, np_(rs["depths"]), np_(rs["tiles_touched"]).view(np.uint32),
                       f32=True)
    assert b["num_rendered"] == R
    np.testing.assert_array_equal(b["keys"], np_(rs["keys"]).view(np.uint64))
    np.testing.assert_array_equal(b["point_list"], np_(rs["point_list"]).view(np.uint32))
    ranges = np_(rs["ranges"]).view(np.uint32)
    np.testing.assert_array_equal(b["ranges"], ranges)

    # ---- forward blend ----
    con = np_(rs["conic_opacity"]).astype(np.float64)
    rgb = np_(rs["rgb"]).astype(np.float64)
    fw = oracle.render_forward(W, H, ranges, b["point_list"], m2, con, rgb, bg_np)
    err = np.abs(fw["image"] - np_(r_img))
    assert np.quantile(err, 0.9999) <= 1e-4 and err.max() <= 1e-3, (np.quantile(err, 0.9999), err.max())
    assert (fw["n_contrib"] != np_(rs["n_contrib"]).view(np.uint32)).mean() < 1e-3

    # ---- backward blend and backward preprocess ----
    bw = oracle.render_backward(P, W, H, ranges, b["point_list"], m2, con, rgb, bg_np,
                                np_(rs["final_T"]).astype(np.float64),
                                np_(rs["n_contrib"]).view(np.uint32), dpix_np)
    for ours, theirs in (("dL_dmean2D", "dL_dmeans2D"), ("dL_dcolor", "dL_dcolors")):
        e = helpers.normwise_rel(bw[ours], np_(r_grads[theirs]))
        assert e < 1e-3, (ours, e)
    e = helpers.normwise_rel(bw["dL_dopacity"], np_(r_grads["dL_dopacity"]).reshape(-1))
    assert e < 1e-3, ("dL_dopacity", e)
    r_dconic = np_(r_grads["dL_dconic"]).reshape(P, 4).astype(np.float64)
    e = helpers.normwise_rel(bw["dL_dconic"][:, [0, 1, 3]], r_dconic[:, [0, 1, 3]])
    assert e < 1e-3, ("dL_dconic", e)
    pb = oracle.preprocess_backward(g.means3D, radii, g.shs, np_(rs["clamped"]), g.scales,
                                    g.rotations, v.viewmatrix, v.campos, W, H,
                                    np_(r_grads["dL_dmeans2D"]).astype(np.float64), r_dconic,
                                    np_(r_grads["dL_dcolors"]).astype(np.float64))
    below85 = np.abs(lat) < np.radians(85.0)
    for name in ("dL_dmeans3D", "dL_dsh", "dL_dscales", "dL_drotations"):
        want = np_(r_grads[name]).astype(np.float64)
        e = helpers.normwise_rel(pb[name][below85], want[below85])
        assert e < 1e-3, (name, e)
        l2 = np.linalg.norm(pb[name] - want) / max(np.linalg.norm(want), 1e-300)
        assert l2 < 1e-3, (name, l2)
    return mism


def test_oracle_matches_reference_small_config(cuda):
    _pin(10_000, 512, 256, seed=0)


def test_oracle_matches_reference_posed_view_with_background(cuda):
    v = scenes.make_view(500, 250, (0.3, 0.1, -0.2), scenes.rotation_yaw_pitch(-1.1, 0.4))
    _pin(10_000, 500, 250, seed=1, view=v, bg=(0.2, 0.4, 0.6))


def test_oracle_matches_reference_pole_heavy(cuda):
    _pin(20_000, 1024, 512, seed=2, pole_fraction=0.3)
