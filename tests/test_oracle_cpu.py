"""CPU tests of the FP64 oracle: known-answer cases derived from the lonlat model, sort/range
semantics, and an FP64 central finite-difference check of its backward.

The reference ships no tests or golden vectors, so these cases are built from first principles
(cuda_rasterizer/auxiliary.h:51-66, 198-248 and forward.cu:130-189, 592-703); the oracle is
additionally pinned to the reference's own outputs in test_oracle_golden.py.
"""
import math

import numpy as np
import pytest

import oracle
from omnigs_b200 import scenes

W, H = 512, 256


def one(mean, scale=0.02, opacity=0.8, q=(1.0, 0.0, 0.0, 0.0), W=W, H=H, sh=None):
    v = scenes.identity_view(W, H)
    shs = np.zeros((1, 16, 3), np.float32) if sh is None else sh
    return oracle.preprocess(np.array([mean], np.float32), np.full((1, 3), scale, np.float32),
                             np.array([q], np.float32), np.array([[opacity]], np.float32), shs,
                             v.viewmatrix, v.campos, W, H)


def test_equator_center_maps_to_image_center():
    pre = one((0.0, 0.0, 2.0))
    assert pre["radii"][0] > 0
    np.testing.assert_allclose(pre["means2D"][0], [(W - 1) / 2, (H - 1) / 2], atol=1e-9)
    assert pre["depths"][0] == pytest.approx(2.0)


def test_seam_maps_to_left_edge_and_rect_is_clamped():
    # lon = atan2(x, z) -> -pi just past the seam: px ~ -0.5, the rect is clamped at column 0
    pre = one((-1e-6, 0.0, -2.0))
    assert pre["means2D"][0][0] == pytest.approx(-0.5, abs=1e-3)
    assert pre["radii"][0] > 0
    r = pre["radii"][0]
    tiles_x_expected = int((pre["means2D"][0][0] + r + 15) // 16)  # rect [0, ceil) after clamp
    ty0 = int((pre["means2D"][0][1] - r) // 16)
    ty1 = int((pre["means2D"][0][1] + r + 15) // 16)
    assert pre["tiles_touched"][0] == tiles_x_expected * (ty1 - ty0)


def test_pole_rect_spans_full_width():
    pre = one((1e-4, 2.0, 1e-4), scale=0.05)  # latitude ~ +90 deg
    assert pre["radii"][0] > 0
    r = int(pre["radii"][0])
    assert r > W  # the lonlat Jacobian blows up near the pole
    gx = W // 16
    rows = int(min(H // 16, (pre["means2D"][0][1] + r + 15) // 16)) - int(max(0, (pre["means2D"][0][1] - r) // 16))
    assert pre["tiles_touched"][0] == gx * rows


@pytest.mark.parametrize("r,visible", [(0.2 * (1 - 1e-4), False), (0.2 * (1 + 1e-4), True)])
def test_near_cull_threshold(r, visible):
    pre = one((0.0, 0.0, r), scale=0.001)
    assert (pre["radii"][0] > 0) == visible


def test_isotropic_equator_covariance_matches_closed_form():
    d, s = 3.0, 0.02
    pre = one((0.0, 0.0, d), scale=s)
    # J at t = (0, 0, d): dpx/dtx = W / (2 pi d), dpy/dty = H / (pi d); cov2D = J S J^T + 0.3 I
    eps = float(np.float32(1e-7))
    jx = W / (2 * math.pi) * d / (d * d + eps)
    jy = H / math.pi * d / (d * d + eps)
    a = jx * jx * s * s + float(np.float32(0.3))
    c = jy * jy * s * s + float(np.float32(0.3))
    con = pre["conic_opacity"][0]
    np.testing.assert_allclose(con[:3], [1 / a, 0.0, 1 / c], rtol=1e-5, atol=1e-12)
    assert pre["radii"][0] == math.ceil(3 * math.sqrt(max(a, c)))


def test_higher_msb_matches_reference_bit_counts():
    assert oracle.higher_msb(512) == 10      # 512 x 256 image, 16 x 16 tiles
    assert oracle.higher_msb(8192) == 14     # 2048 x 1024
    assert oracle.higher_msb(32768) == 16    # 4096 x 2048
    assert oracle.higher_msb(1) == 1


def test_sort_is_stable_and_ranges_cover_tiles():
    # two Gaussians with identical depth in the same tile keep index order; a third behind them
    P = 3
    m2 = np.array([[100.5, 50.5], [101.0, 51.0], [102.0, 52.0]], np.float32)
    depth = np.array([2.0, 2.0, 1.0], np.float32)
    radii = np.array([1, 1, 1], np.int32)
    tt = np.array([1, 1, 1], np.uint32)
    b = oracle.binning(W, H, radii, m2, depth, tt, f32=True)
    assert list(b["point_list"]) == [2, 0, 1]
    tile = (50 // 16) * (W // 16) + 100 // 16
    assert list(b["ranges"][tile]) == [0, 3]
    assert int((b["ranges"][:, 1] - b["ranges"][:, 0]).sum()) == P


def test_binning_f32_matches_numpy_restatement():
    g = scenes.make_gaussians(2000, seed=3)
    v = scenes.identity_view(W, H)
    pre = oracle.preprocess(g.means3D, g.scales, g.rotations, g.opacities, g.shs, v.viewmatrix,
                            v.campos, W, H)
    m2 = pre["means2D"].astype(np.float32)
    d32 = pre["depths"].astype(np.float32)
    b = oracle.binning(W, H, pre["radii"], m2, d32, pre["tiles_touched"], f32=True)
    # independent numpy restatement of duplicateWithKeys + stable sort
    keys, vals = [], []
    gx, gy = W // 16, H // 16
    for i in range(g.P):
        r = int(pre["radii"][i])
        if r <= 0:
            continue
        px, py = np.float32(m2[i, 0]), np.float32(m2[i, 1])
        f = np.float32
        x0 = min(gx, max(0, int((px - f(r)) / f(16))))
        y0 = min(gy, max(0, int((py - f(r)) / f(16))))
        x1 = min(gx, max(0, int((px + f(r) + f(16) - f(1)) / f(16))))
        y1 = min(gy, max(0, int((py + f(r) + f(16) - f(1)) / f(16))))
        dbits = int(d32[i:i + 1].view(np.uint32)[0])
        for y in range(y0, y1):
            for x in range(x0, x1):
                keys.append(((y * gx + x) << 32) | dbits)
                vals.append(i)
    keys = np.array(keys, np.uint64)
    order = np.argsort(keys, kind="stable")
    np.testing.assert_array_equal(b["keys"], keys[order])
    np.testing.assert_array_equal(b["point_list"], np.array(vals, np.uint32)[order])


def test_empty_scene_renders_background():
    v = scenes.identity_view(64, 32)
    ranges = np.zeros((4 * 2, 2), np.uint32)
    out = oracle.render_forward(64, 32, ranges, np.zeros(0, np.uint32), np.zeros((0, 2)),
                                np.zeros((0, 4)), np.zeros((0, 3)), np.array([0.1, 0.2, 0.3], np.float32))
    np.testing.assert_allclose(out["image"][:, 5, 7], [0.1, 0.2, 0.3], rtol=1e-6)
    assert out["final_T"].min() == 1.0 and out["n_contrib"].max() == 0
    del v


def _loss(g, v, dpix, W, H):
    out = oracle.forward_backward(g, v, dpix, nthreads=1)
    return float((out["image"] * dpix).sum()), out


@pytest.mark.parametrize("seed", [0, 1])
def test_backward_matches_fp64_central_differences(seed):
    """FP64 central differences of L = <dL/dpix, image> against the oracle's analytic backward,
    i.e. against the reference's gradient formulas (incl. the lonlat second derivatives)."""
    Wf, Hf = 128, 64
    rng = np.random.default_rng(seed)
    g = scenes.make_gaussians(40, seed=10 + seed)
    # larger, well-separated splats so that few pixels sit on a threshold
    g.scales[:] = np.exp(rng.normal(np.log(0.06), 0.2, g.scales.shape)).astype(np.float32)
    v = scenes.make_view(Wf, Hf, (0.1, -0.05, 0.2), scenes.rotation_yaw_pitch(0.3, 0.1))
    dpix = scenes.upstream_grad(Wf, Hf, seed=seed)
    L0, out = _loss(g, v, dpix, Wf, Hf)
    vis = np.nonzero(out["pre"]["radii"] > 0)[0]
    assert len(vis) > 10
    checks = [("means3D", "dL_dmeans3D", 1e-4), ("scales", "dL_dscales", 1e-5),
              ("rotations", "dL_drotations", 1e-4), ("opacities", "dL_dopacity", 1e-5),
              ("shs", "dL_dsh", 1e-4)]
    errs = []
    for field, gname, eps in checks:
        arr = getattr(g, field)
        ana_all = out[gname].reshape(arr.shape[0], -1)
        for i in vis[:12]:
            flat = arr.reshape(arr.shape[0], -1)
            for k in range(min(flat.shape[1], 6)):
                ana = ana_all[i, k]
                orig = flat[i, k]
                flat[i, k] = orig + eps
                hi = float(flat[i, k])
                Lp, _ = _loss(g, v, dpix, Wf, Hf)
                flat[i, k] = orig - eps
                lo = float(flat[i, k])
                Lm, _ = _loss(g, v, dpix, Wf, Hf)
                flat[i, k] = orig
                fd = (Lp - Lm) / (hi - lo)  # the float32-representable step
                scale = max(abs(fd), abs(ana), 1e-3 * np.abs(ana_all).max())
                errs.append(abs(fd - ana) / scale)
    errs = np.array(errs)
    # inputs are float32, so perturbations are float32-rounded; compare robustly
    assert np.median(errs) < 1e-3, np.percentile(errs, [50, 90, 99])
    assert np.percentile(errs, 90) < 2e-2, np.percentile(errs, [50, 90, 99])
