"""GPU parity of the batched multi-view path (omnigs_batch_* through the C ABI).

The single-view path is pinned bit for bit to the reference rasterizer (test_reference_gpu.py), so
the batch is checked against it: every view's instance count, last contributors, transmittance and
image are identical to a single-view forward of that view; the parameter gradients equal the sum
of the single-view backwards within 1e-4 normwise relative (the per-splat accumulators are summed
with float atomics in run-dependent order, and the batch sums the views in another order); the
densification statistics equal the trainer's per-view accumulation.  BF16 SH storage is checked
against the FP32 path fed with the same bf16-rounded coefficients (images bit-identical), and the
FP64 pole mode against the FP64 oracle.
"""
import numpy as np
import pytest
import torch

import helpers
import oracle
from omnigs_b200 import batch, capi, lonlat, scenes

pytestmark = pytest.mark.gpu

GRAD_RTOL = 1e-4


def _rel(a, b):
    a, b = helpers.to_np(a).astype(np.float64), helpers.to_np(b).astype(np.float64)
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-30)


def _views(sizes, seed):
    """Identity pose for the first view, then positions within a 2 m cube and random yaw/pitch."""
    rng = np.random.Generator(np.random.PCG64(seed + 10))
    views = [scenes.identity_view(*sizes[0])]
    for w, h in sizes[1:]:
        R = scenes.rotation_yaw_pitch(rng.uniform(-np.pi, np.pi), np.radians(rng.uniform(-30, 30)))
        views.append(scenes.make_view(w, h, rng.uniform(-1.0, 1.0, 3), R))
    return views


def _plain(gt, view, dpix, bg):
    cam = lonlat.Camera.from_view(view, background=bg)
    return helpers.run_cuda(gt, cam, torch.from_numpy(dpix).cuda())


def _batch(gt, views, dpix_list, bg, fp64_poles=False, capacity=None):
    cams = batch.BatchCameras.from_views(views, background=bg)
    images, per_view, state = batch.render_batch(gt, cams, fp64_poles=fp64_poles, capacity=capacity)
    grads = batch.BatchGradients.empty(gt.P, gt.M, gt.means3D.device, stats=True)
    dl = [torch.from_numpy(d).cuda() for d in dpix_list]
    state.backward(gt, cams, dl, grads, fp64_poles=fp64_poles)
    torch.cuda.synchronize()
    return images, per_view, state, grads


# Four 3072x1536 views and one 512x256 hold 74,240 tiles: global tile ids need 17 bits (three sort
# passes), view-local ones 15 (two), so the tile sort runs per view; with P = 200 (< 256) the batch
# falls back to the global tile sort.
PER_VIEW_SIZES = [(3072, 1536)] * 4 + [(512, 256)]


@pytest.mark.parametrize("sizes,P,seed", [
    ([(512, 256)], 10_000, 0),
    ([(512, 256), (1024, 512), (96, 48), (500, 250)], 20_000, 1),
    ([(2048, 1024), (512, 256), (3072, 1536)], 60_000, 2),
    (PER_VIEW_SIZES, 20_000, 5),
    (PER_VIEW_SIZES, 200, 6),
])
def test_batch_matches_single_views(cuda, sizes, P, seed):
    g = scenes.make_gaussians(P, seed=seed)
    gt = lonlat.GaussianTensors.from_numpy(g)
    views = _views(sizes, seed)
    bg = (0.1, 0.2, 0.3)
    dpix = [scenes.upstream_grad(w, h, seed=seed + 20 + i) for i, (w, h) in enumerate(sizes)]
    images, per_view, state, grads = _batch(gt, views, dpix, bg)
    sv = state.state_view()
    sums = {k: 0.0 for k in ("dL_dmeans3D", "dL_dsh", "dL_dopacity", "dL_dscales", "dL_drotations")}
    stat_norm = torch.zeros(P, device=cuda, dtype=torch.float64)
    stat_cnt = torch.zeros(P, device=cuda, dtype=torch.float64)
    max_r = torch.zeros(P, device=cuda, dtype=torch.int32)
    for v, view in enumerate(views):
        cu = _plain(gt, view, dpix[v], bg)
        assert per_view[v] == cu["num_rendered"]
        torch.testing.assert_close(sv["radii"][v], cu["radii"], rtol=0, atol=0)
        torch.testing.assert_close(sv["n_contrib"][v], cu["n_contrib"], rtol=0, atol=0)
        torch.testing.assert_close(sv["final_T"][v], cu["final_T"], rtol=0, atol=0)
        torch.testing.assert_close(images[v], cu["image"], rtol=0, atol=0)
        for k in sums:
            sums[k] = sums[k] + getattr(cu["grads"], k).double()
        vis = cu["radii"] > 0
        m2 = cu["grads"].dL_dmeans2D.double()
        stat_norm += torch.where(vis, torch.linalg.norm(m2[:, :2], dim=1), 0.0)
        stat_cnt += vis.double()
        max_r = torch.maximum(max_r, torch.where(vis, cu["radii"], 0))
    for k, ref in sums.items():
        assert _rel(getattr(grads, k), ref) < GRAD_RTOL, k
    assert _rel(grads.grad_accum[:, 0], stat_norm) < 1e-5
    torch.testing.assert_close(grads.denom[:, 0].double(), stat_cnt, rtol=0, atol=0)
    torch.testing.assert_close(grads.max_radii, max_r.float(), rtol=0, atol=0)


def test_bf16_sh_equals_fp32_path_on_rounded_coefficients(cuda):
    g = scenes.make_gaussians(20_000, seed=3)
    gt = lonlat.GaussianTensors.from_numpy(g)
    sh16 = gt.shs.to(torch.bfloat16)
    g16 = lonlat.GaussianTensors(means3D=gt.means3D, opacities=gt.opacities, shs=sh16,
                                 scales=gt.scales, rotations=gt.rotations)
    grounded = lonlat.GaussianTensors(means3D=gt.means3D, opacities=gt.opacities, shs=sh16.float(),
                                      scales=gt.scales, rotations=gt.rotations)
    views = [scenes.identity_view(512, 256), scenes.make_view(1024, 512, (0.3, -0.2, 0.5))]
    dpix = [scenes.upstream_grad(w.width, w.height, seed=5 + i) for i, w in enumerate(views)]
    cams = batch.BatchCameras.from_views(views)
    out = {}
    for name, gg in (("bf16", g16), ("fp32", grounded)):
        images, per_view, state = batch.render_batch(gg, cams)
        grads = batch.BatchGradients.empty(gg.P, gg.M, cuda)
        state.backward(gg, cams, [torch.from_numpy(d).cuda() for d in dpix], grads)
        torch.cuda.synchronize()
        out[name] = (images, per_view, grads)
    assert out["bf16"][1] == out["fp32"][1]
    for a, b in zip(out["bf16"][0], out["fp32"][0]):
        torch.testing.assert_close(a, b, rtol=0, atol=0)
    # same coefficients, same formulas: the two kernel instantiations may fuse a few products
    # differently, so gradients agree to FP32 rounding rather than bit for bit
    for k in ("dL_dmeans3D", "dL_dsh", "dL_dopacity", "dL_dscales", "dL_drotations"):
        assert _rel(getattr(out["bf16"][2], k), getattr(out["fp32"][2], k)) < GRAD_RTOL, k


@pytest.mark.parametrize("sizes", [[(512, 256), (256, 128)], PER_VIEW_SIZES])
def test_capacity_overflow_resumes(cuda, sizes):
    g = scenes.make_gaussians(10_000, seed=4)
    gt = lonlat.GaussianTensors.from_numpy(g)
    views = [scenes.identity_view(*sizes[0])] + [scenes.make_view(w, h, (0.5, 0.1 * i, 0.0))
                                                 for i, (w, h) in enumerate(sizes[1:])]
    cams = batch.BatchCameras.from_views(views)
    ref_images, ref_per, _ = batch.render_batch(gt, cams)
    small = batch.BatchState(gt.P, cams.sizes, capacity=1000)
    images = [torch.empty(3, h, w, device=cuda) for w, h in cams.sizes]
    small.forward(gt, cams, images)
    n, per, st = small.status()
    assert st & capi.STATUS_CAPACITY and n == sum(ref_per) and per == ref_per
    small.resize_capacity(n)
    small.render(gt, cams, images)
    n2, per2, st2 = small.status()
    assert st2 == 0 and per2 == ref_per
    for a, b in zip(images, ref_images):
        torch.testing.assert_close(a, b, rtol=0, atol=0)


def test_fp64_poles_tracks_the_fp64_oracle_closer(cuda):
    """Pole-heavy scene: the conics of Gaussians beyond 85 degrees from the FP64 pole mode are
    closer to the FP64 oracle's than the FP32 path's; elsewhere both are identical."""
    P, W, H = 20_000, 1024, 512
    g = scenes.make_gaussians(P, seed=6, pole_fraction=0.3, pole_min_lat_deg=84.0)
    gt = lonlat.GaussianTensors.from_numpy(g)
    view = scenes.identity_view(W, H)
    cams = batch.BatchCameras.from_views([view])
    _, _, s32 = batch.render_batch(gt, cams, fp64_poles=False)
    _, _, s64 = batch.render_batch(gt, cams, fp64_poles=True)
    pre = oracle.preprocess(g.means3D, g.scales, g.rotations, g.opacities, g.shs, view.viewmatrix,
                            view.campos, W, H)
    lat = np.degrees(np.arcsin(np.abs(g.means3D[:, 1]) / np.linalg.norm(g.means3D, axis=1)))
    c32 = helpers.to_np(s32.state_view()["splat"][0])[:, 2:5].astype(np.float64)
    c64 = helpers.to_np(s64.state_view()["splat"][0])[:, [2, 3, 4]].astype(np.float64)
    r32 = helpers.to_np(s32.state_view()["radii"][0])
    r64 = helpers.to_np(s64.state_view()["radii"][0])
    ref = pre["conic_opacity"][:, :3]
    vis = (r32 > 0) & (r64 > 0) & (pre["radii"] > 0)
    pole, rest = vis & (lat > 85.5), vis & (lat < 84.5)
    assert pole.sum() > 100
    np.testing.assert_array_equal(c32[rest], c64[rest])
    scale = np.abs(ref).max(1)
    e32 = (np.abs(c32 - ref).max(1) / scale)[pole]
    e64 = (np.abs(c64 - ref).max(1) / scale)[pole]
    msg = f"FP32 max {e32.max():.3g} mean {e32.mean():.3g}; FP64 poles max {e64.max():.3g} mean {e64.mean():.3g}"
    assert e64.mean() <= e32.mean(), msg
    assert e64.max() <= max(e32.max(), 1e-6), msg


def test_blend_batch_sizes_and_autotuner(cuda):
    """Every staging batch size gives the identical image and gradients within tolerance; the
    autotuner picks one of the candidates and leaves the state ready for the backward."""
    g = scenes.make_gaussians(30_000, seed=8)
    gt = lonlat.GaussianTensors.from_numpy(g)
    views = _views([(1024, 512), (512, 256)], 8)
    cams = batch.BatchCameras.from_views(views)
    dl = [torch.from_numpy(scenes.upstream_grad(v.width, v.height, seed=30 + i)).cuda() for i, v in enumerate(views)]
    out = {}
    try:
        for b in (128, 256, 512):
            batch.set_blend_batch(b, b)
            images, per, state = batch.render_batch(gt, cams)
            grads = batch.BatchGradients.empty(gt.P, gt.M, cuda)
            state.backward(gt, cams, dl, grads)
            torch.cuda.synchronize()
            out[b] = (images, grads)
        for b in (128, 512):
            for x, y in zip(out[b][0], out[256][0]):
                torch.testing.assert_close(x, y, rtol=0, atol=0)
            for k in ("dL_dmeans3D", "dL_dsh", "dL_dopacity", "dL_dscales", "dL_drotations"):
                assert _rel(getattr(out[b][1], k), getattr(out[256][1], k)) < GRAD_RTOL, (b, k)
        batch.set_blend_batch(256, 256)
        images, per, state = batch.render_batch(gt, cams)
        res = state.autotune(gt, cams, images, dl)
        assert res["forward_batch"] in (128, 256, 512) and res["backward_batch"] in (128, 256, 512)
        assert batch.get_blend_batch() == (res["forward_batch"], res["backward_batch"])
        assert all(t > 0 for t in res["forward_ms"] + res["backward_ms"])
        for x, y in zip(images, out[256][0]):
            torch.testing.assert_close(x, y, rtol=0, atol=0)
        grads = batch.BatchGradients.empty(gt.P, gt.M, cuda)
        state.backward(gt, cams, dl, grads)
        torch.cuda.synchronize()
        for k in ("dL_dmeans3D", "dL_dsh", "dL_dopacity", "dL_dscales", "dL_drotations"):
            assert _rel(getattr(grads, k), getattr(out[256][1], k)) < GRAD_RTOL, k
    finally:
        batch.set_blend_batch(128, 128)  # the library's defaults


def test_batch_edge_cases(cuda):
    """No Gaussians (images are the zeros the reference returns), a view where every Gaussian is
    culled (camera inside the near-cull sphere of the only Gaussian), and the maximum of 32 views
    with tiny and ragged sizes, each view matching its single-view render."""
    bgc = (0.2, 0.4, 0.6)
    # P = 0
    empty = lonlat.GaussianTensors(means3D=torch.zeros(0, 3, device=cuda), opacities=torch.zeros(0, 1, device=cuda),
                                   shs=torch.zeros(0, 16, 3, device=cuda), scales=torch.zeros(0, 3, device=cuda),
                                   rotations=torch.zeros(0, 4, device=cuda))
    cams = batch.BatchCameras.from_views([scenes.identity_view(64, 32), scenes.identity_view(48, 16)], background=bgc)
    st = batch.BatchState(0, cams.sizes, 1024)
    images = [torch.full((3, h, w), 7.0, device=cuda) for w, h in cams.sizes]
    st.forward(empty, cams, images)
    torch.cuda.synchronize()
    for im in images:
        assert float(im.abs().max()) == 0.0
    grads = batch.BatchGradients.empty(0, 16, cuda)
    st.backward(empty, cams, [torch.zeros(3, h, w, device=cuda) for w, h in cams.sizes], grads)
    # every Gaussian culled in one view (r^2 <= 0.04 around the camera), visible in the other
    one = scenes.make_gaussians(1, seed=1)
    one = scenes.Gaussians(np.array([[0.0, 0.0, 1.0]], np.float32), one.scales, one.rotations, one.opacities, one.shs)
    g1 = lonlat.GaussianTensors.from_numpy(one)
    views = [scenes.make_view(64, 32, (0.0, 0.0, 1.05)), scenes.identity_view(64, 32)]
    images, per, state = batch.render_batch(g1, batch.BatchCameras.from_views(views, background=bgc))
    assert per[0] == 0 and per[1] > 0
    torch.testing.assert_close(images[0], torch.tensor(bgc, device=cuda).view(3, 1, 1).expand(3, 32, 64),
                               rtol=0, atol=0)
    # 32 views, tiny and ragged sizes, against single-view renders
    g = scenes.make_gaussians(5_000, seed=12)
    gt = lonlat.GaussianTensors.from_numpy(g)
    rng = np.random.Generator(np.random.PCG64(12))
    sizes = [(int(rng.integers(8, 200)), int(rng.integers(4, 100))) for _ in range(capi.MAX_BATCH_VIEWS)]
    views = _views(sizes, 12)
    images, per, state = batch.render_batch(gt, batch.BatchCameras.from_views(views, background=bgc))
    for v, view in enumerate(views):
        cu = _plain(gt, view, scenes.upstream_grad(view.width, view.height), bgc)
        assert per[v] == cu["num_rendered"], v
        torch.testing.assert_close(images[v], cu["image"], rtol=0, atol=0)
    with pytest.raises(capi.OmnigsError):
        batch.BatchState(100, [(64, 32)] * (capi.MAX_BATCH_VIEWS + 1), 1024)


def test_seam_wrap_turns_yaw_into_a_roll(cuda):
    """With seam wrapping, turning the camera by k pixels' worth of yaw rolls the equirect image by
    k pixels (up to FP32 rounding of the projection); with the reference's clamped tile rects the
    image is cut at the seam, so the columns at both seams differ."""
    W, H, k = 512, 256, 100
    g = scenes.make_gaussians(20_000, seed=13)
    gt = lonlat.GaussianTensors.from_numpy(g)
    yaw = 2 * np.pi * k / W
    views = [scenes.identity_view(W, H), scenes.make_view(W, H, (0.0, 0.0, 0.0), scenes.rotation_yaw_pitch(yaw, 0.0))]
    cams = batch.BatchCameras.from_views(views)
    seam = torch.zeros(W, dtype=torch.bool, device=cuda)
    for c in (W - k, 0):  # image 0's seam after the roll, image 1's own seam
        for d in range(-6, 6):
            seam[(c + d) % W] = True
    err = {}
    for wrap in (False, True):
        imgs, _, state = batch.render_batch(gt, cams, seam_wrap=wrap)
        diff = (torch.roll(imgs[0], shifts=-k, dims=2) - imgs[1]).abs()
        err[wrap] = (float(diff[:, :, seam].mean()), float(diff[:, :, ~seam].mean()))
        dl = [torch.from_numpy(scenes.upstream_grad(W, H, seed=40 + i)).cuda() for i in range(2)]
        grads = batch.BatchGradients.empty(gt.P, gt.M, cuda)
        state.backward(gt, cams, dl, grads, seam_wrap=wrap)
        torch.cuda.synchronize()
        assert all(bool(torch.isfinite(getattr(grads, n)).all()) for n in ("dL_dmeans3D", "dL_dsh", "dL_dscales"))
    assert err[False][0] > 20 * err[False][1], err       # the clamped rects cut the image at the seam
    assert err[True][0] < 3 * err[True][1] + 1e-5, err    # wrapped: the seam is like any other column
    assert err[True][0] < 0.05 * err[False][0], err


def test_seam_wrap_changes_nothing_away_from_the_seam(cuda):
    """Gaussians whose tile rects stay inside the image get identical instances and images."""
    g = scenes.make_gaussians(5_000, seed=14)
    m = g.means3D.copy()
    m[:, 2] = np.abs(m[:, 2]) + 1.5        # in front of the camera: longitude within (-90, 90) deg
    g = scenes.Gaussians(m, g.scales, g.rotations, g.opacities, g.shs)
    gt = lonlat.GaussianTensors.from_numpy(g)
    cams = batch.BatchCameras.from_views([scenes.identity_view(512, 256)])
    a, pa, _ = batch.render_batch(gt, cams, seam_wrap=False)
    b, pb, _ = batch.render_batch(gt, cams, seam_wrap=True)
    assert pa == pb
    torch.testing.assert_close(a[0], b[0], rtol=0, atol=0)


def test_per_view_tile_sort_with_seam_wrap_matches_one_view_batches(cuda):
    """The per-view tile sort (PER_VIEW_SIZES) with seam wrapping: every view of the batch equals the
    same view rendered as a batch of one (whose tile sort is the global one) -- instance counts,
    last contributors, transmittance and image bit for bit, gradients to FP32 summation order."""
    P = 20_000
    g = scenes.make_gaussians(P, seed=17)
    gt = lonlat.GaussianTensors.from_numpy(g)
    views = _views(PER_VIEW_SIZES, 17)
    cams = batch.BatchCameras.from_views(views)
    imgs, per, state = batch.render_batch(gt, cams, seam_wrap=True)
    dl = [torch.from_numpy(scenes.upstream_grad(v.width, v.height, seed=60 + i)).cuda() for i, v in enumerate(views)]
    grads = batch.BatchGradients.empty(gt.P, gt.M, cuda)
    state.backward(gt, cams, dl, grads, seam_wrap=True)
    torch.cuda.synchronize()
    sv = state.state_view()
    sums = {k: 0.0 for k in ("dL_dmeans3D", "dL_dsh", "dL_dopacity")}
    for v, view in enumerate(views):
        one = batch.BatchCameras.from_views([view])
        img1, per1, st1 = batch.render_batch(gt, one, seam_wrap=True)
        g1 = batch.BatchGradients.empty(gt.P, gt.M, cuda)
        st1.backward(gt, one, [dl[v]], g1, seam_wrap=True)
        torch.cuda.synchronize()
        sv1 = st1.state_view()
        assert per[v] == per1[0]
        torch.testing.assert_close(sv["n_contrib"][v], sv1["n_contrib"][0], rtol=0, atol=0)
        torch.testing.assert_close(sv["final_T"][v], sv1["final_T"][0], rtol=0, atol=0)
        torch.testing.assert_close(imgs[v], img1[0], rtol=0, atol=0)
        for k in sums:
            sums[k] = sums[k] + getattr(g1, k).double()
    for k, ref in sums.items():
        assert _rel(getattr(grads, k), ref) < GRAD_RTOL, k
