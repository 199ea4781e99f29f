"""The seam-wrapping mode of the batched path against the FP64 oracle's seam-wrapping mode.

The reference clamps tile rects at the image edges (getRect, forward.cu:680); its unused
getRectCyclic (auxiliary.h:68-83) describes the cyclic range.  The oracle restates that mode
(cyclic tile columns with the floor and one-width cap this package documents, x offsets to the
splat copy nearest the centre of each pixel's 8-column block) and is checked on its own on the CPU
(exact quarter-turn roll, central differences).  Here a scene with 30 % of its splats straddling longitude +-pi is rendered
and back-propagated through the batched entry points with seam_wrap on, two views at once, and
every stage is compared with the oracle fed the CUDA path's float intermediates:

* binning: per view, the sorted tile ids and splat indices, and the tile ranges, bit-exact;
* forward blend: image within 1e-4, last contributors equal on all but 0.1 % of the pixels (as in
  the other stage-isolated parity tests: FP64 and FP32 may decide a threshold differently);
* backward (blend + preprocess, summed over the views): gradients within 1e-3 normwise relative.

The posed view puts some splats within a metre of the camera, wider than the whole image (their
cyclic rects span every column): for those the copy nearest each 8-column block is what both
compute.
"""
import numpy as np
import pytest
import torch

import helpers
import oracle
from omnigs_b200 import batch, lonlat, scenes

pytestmark = pytest.mark.gpu

np_ = helpers.to_np


def test_seam_wrap_matches_the_oracle(cuda):
    P = 20_000
    g = scenes.make_gaussians(P, seed=41, seam_fraction=0.3)
    gt = lonlat.GaussianTensors.from_numpy(g)
    views = [scenes.identity_view(1024, 512),
             scenes.make_view(800, 400, (0.2, -0.1, 0.3), scenes.rotation_yaw_pitch(0.05, 0.2))]
    cams = batch.BatchCameras.from_views(views, background=(0.1, 0.2, 0.3))
    images, per_view, state = batch.render_batch(gt, cams, seam_wrap=True)
    dpix = [torch.from_numpy(scenes.upstream_grad(v.width, v.height, seed=41 + i)).cuda()
            for i, v in enumerate(views)]
    grads = batch.BatchGradients.empty(P, 16, "cuda")
    sv = state.state_view()
    total = sum(per_view)
    bv = state.binning_view(total)
    tile_ids, point_list = np_(bv["tile_ids"]).view(np.uint32), np_(bv["point_list"]).view(np.uint32)
    state.backward(gt, cams, dpix, grads, seam_wrap=True)
    torch.cuda.synchronize()
    bg = np.array([0.1, 0.2, 0.3], np.float32)
    sums = {k: 0.0 for k in ("dL_dmeans3D", "dL_dsh", "dL_dopacity", "dL_dscales", "dL_drotations")}
    wrapped = 0
    for v, view in enumerate(views):
        W, H = view.width, view.height
        radii = np_(sv["radii"][v])
        splat = np_(sv["splat"][v])
        m2 = np.ascontiguousarray(splat[:, :2])
        depth = np_(sv["depth"][v])
        b = oracle.binning(W, H, radii, m2, depth, None, f32=True, seam_wrap=True)
        assert b["num_rendered"] == per_view[v]
        # this view's instances are one contiguous run of the batch's sorted list
        tb, nt = sv["tile_base"][v], ((W + 15) // 16) * ((H + 15) // 16)
        sel = (tile_ids >= tb) & (tile_ids < tb + nt)
        assert int(sel.sum()) == per_view[v]
        start = int(np.argmax(sel))
        np.testing.assert_array_equal(tile_ids[sel] - tb, (b["keys"] >> 32).astype(np.uint32))
        np.testing.assert_array_equal(point_list[sel] - np.uint32(v * P), b["point_list"])
        rg = np_(sv["ranges"][v]).view(np.uint32).astype(np.int64)
        nonempty = b["ranges"][:, 1] > b["ranges"][:, 0]
        np.testing.assert_array_equal(rg[nonempty] - start, b["ranges"][nonempty])
        assert (rg[~nonempty, 0] == rg[~nonempty, 1]).all()
        gx = (W + 15) // 16
        cols = (b["keys"] >> 32) % gx
        wrapped += int(((cols == 0) | (cols == gx - 1)).sum())
        # forward blend
        con = np.concatenate([splat[:, 2:5], splat[:, 5:6]], 1).astype(np.float64)
        rgb = np_(sv["color"][v])[:, :3].astype(np.float64)
        fw = oracle.render_forward(W, H, b["ranges"], b["point_list"], m2, con, rgb, bg, seam_wrap=True)
        assert np.abs(np_(images[v]) - fw["image"]).max() <= 1e-4
        n_contrib = np_(sv["n_contrib"][v]).view(np.uint32)
        assert (n_contrib != fw["n_contrib"]).mean() < 1e-3
        # backward blend + preprocess, fed the CUDA path's transmittance and last contributors
        bw = oracle.render_backward(P, W, H, b["ranges"], b["point_list"], m2, con, rgb, bg,
                                    np_(sv["final_T"][v]).astype(np.float64), n_contrib, np_(dpix[v]),
                                    seam_wrap=True)
        bits = np_(sv["color"][v])[:, 3].view(np.uint32)
        clamped = np.stack([(bits >> k) & 1 for k in range(3)], 1).astype(np.uint8)
        pb = oracle.preprocess_backward(g.means3D, radii, g.shs, clamped, g.scales, g.rotations,
                                        view.viewmatrix, view.campos, W, H, bw["dL_dmean2D"],
                                        bw["dL_dconic"], bw["dL_dcolor"])
        pb["dL_dopacity"] = bw["dL_dopacity"].reshape(-1, 1)
        for k in sums:
            sums[k] = sums[k] + pb[k]
    assert wrapped > 1000  # many instances sit in the seam columns
    for k, want in sums.items():
        e = helpers.normwise_rel(np_(getattr(grads, k)), want)
        assert e < 1e-3, (k, e)
