"""CPU tests of the FP64 oracle: known-answer cases derived from the lonlat model, sort/range
semantics, and an FP64 central finite-difference check of its backward.

The reference ships no tests or golden vectors, so these cases are built from first principles
(cuda_rasterizer/auxiliary.h:51-66, 198-248 and forward.cu:130-189, 592-703); the oracle is
additionally pinned to the reference's own outputs, stage by stage, in
test_oracle_vs_reference_gpu.py.
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


# ---------------------------------------------------------------- seam-wrapping mode ----------
def _yaw90_view(W, H):
    """Camera turned by exactly 90 degrees of yaw about +y (integer rotation matrix, so the view
    matrix is exact in float32): every longitude decreases by pi / 2, i.e. W / 4 pixels."""
    R_wc = np.array([[0.0, 0.0, 1.0], [0.0, 1.0, 0.0], [-1.0, 0.0, 0.0]])
    return scenes.make_view(W, H, (0.0, 0.0, 0.0), R_wc)


def test_seam_wrap_known_answer_single_splat():
    """A splat centred half a pixel left of the right image edge (longitude just below +pi): with
    seam wrapping its tile rect continues in column 0 and it colours pixels of column 0; with the
    reference's clamped rects it does not."""
    W, H = 256, 128
    g = scenes.make_gaussians(1, seed=0)
    lon = math.pi - math.pi / W  # half a pixel left of the seam: px = W - 1
    g.means3D[0] = np.array([2.0 * math.sin(lon), 0.0, 2.0 * math.cos(lon)], np.float32)
    g.scales[0] = 0.05
    g.opacities[0] = 0.9
    v = scenes.identity_view(W, H)
    bg = np.zeros(3, np.float32)
    for wrap in (False, True):
        pre = oracle.preprocess(g.means3D, g.scales, g.rotations, g.opacities, g.shs, v.viewmatrix,
                                v.campos, W, H, seam_wrap=wrap)
        assert pre["radii"][0] > 0 and abs(pre["means2D"][0, 0] - (W - 1)) < 1.0
        b = oracle.binning(W, H, pre["radii"], pre["means2D"], pre["depths"], pre["tiles_touched"],
                           f32=False, seam_wrap=wrap)
        cols = set(int(k >> 32) % (W // 16) for k in b["keys"])
        fw = oracle.render_forward(W, H, b["ranges"], b["point_list"], pre["means2D"],
                                   pre["conic_opacity"], pre["rgb"], bg, seam_wrap=wrap)
        col0 = float(1.0 - fw["final_T"].reshape(H, W)[:, 0].min())
        if wrap:
            assert 0 in cols and W // 16 - 1 in cols
            assert col0 > 0.1  # the splat's wrapped half
        else:
            assert 0 not in cols
            assert col0 == 0.0


@pytest.mark.parametrize("wrap", [False, True])
def test_seam_wrap_yaw_by_a_quarter_turn_rolls_the_image(wrap):
    """Turning the camera by exactly 90 degrees of yaw rolls the equirect image by W / 4 pixels (a
    whole number of tiles).  With seam wrapping this holds to FP64 rounding everywhere, including
    the splats that straddle the seam, and the gradients with respect to the Gaussians are
    unchanged; with the reference's clamped rects the columns at the two seams differ."""
    W, H = 256, 128
    g = scenes.make_gaussians(3000, seed=31, seam_fraction=0.4)
    dpix = scenes.upstream_grad(W, H, seed=31)
    a = oracle.forward_backward(g, scenes.identity_view(W, H), dpix, seam_wrap=wrap)
    b = oracle.forward_backward(g, _yaw90_view(W, H), np.roll(dpix, -W // 4, axis=2), seam_wrap=wrap)
    rolled = np.roll(a["image"], -W // 4, axis=2)
    diff = np.abs(b["image"] - rolled)
    seam_cols = np.zeros(W, bool)
    for c in (W - W // 4, 0):  # image a's seam after the roll, image b's own seam
        for d in range(-16, 16):
            seam_cols[(c + d) % W] = True
    if wrap:
        assert diff.max() < 1e-9, diff.max()
        for name in ("dL_dmeans3D", "dL_dsh", "dL_dopacity", "dL_dscales", "dL_drotations"):
            ga, gb = a[name], b[name]
            assert np.abs(ga - gb).max() <= 1e-9 * max(np.abs(ga).max(), 1e-30), name
    else:
        assert diff[:, :, ~seam_cols].max() < 1e-9
        assert diff[:, :, seam_cols].max() > 1e-2


def test_seam_wrap_backward_matches_fp64_central_differences():
    """FP64 central differences of L = <dL/dpix, image> against the oracle's backward in seam
    wrapping mode, on splats straddling the seam (x offsets to the nearest copy)."""
    Wf, Hf = 128, 64
    rng = np.random.default_rng(3)
    g = scenes.make_gaussians(40, seed=13, seam_fraction=1.0, seam_width_deg=6.0)
    g.scales[:] = np.exp(rng.normal(np.log(0.06), 0.2, g.scales.shape)).astype(np.float32)
    v = scenes.identity_view(Wf, Hf)
    dpix = scenes.upstream_grad(Wf, Hf, seed=3)

    def loss(gs):
        out = oracle.forward_backward(gs, v, dpix, nthreads=1, seam_wrap=True)
        return float((out["image"] * dpix).sum()), out

    _, out = loss(g)
    vis = np.nonzero(out["pre"]["radii"] > 0)[0]
    assert len(vis) > 10
    # some splats really do straddle: their rects wrap
    assert (out["pre"]["tiles_touched"] > 0).sum() == len(vis)
    errs = []
    for field, gname, eps in (("means3D", "dL_dmeans3D", 1e-4), ("opacities", "dL_dopacity", 1e-5),
                              ("shs", "dL_dsh", 1e-4), ("scales", "dL_dscales", 1e-5)):
        arr = getattr(g, field)
        flat = arr.reshape(arr.shape[0], -1)
        ana_all = out[gname].reshape(arr.shape[0], -1)
        for i in vis[:10]:
            for k in range(min(flat.shape[1], 3)):
                orig = flat[i, k]
                flat[i, k] = orig + eps
                hi = float(flat[i, k])
                lp, _ = loss(g)
                flat[i, k] = orig - eps
                lo = float(flat[i, k])
                lm, _ = loss(g)
                flat[i, k] = orig
                fd = (lp - lm) / (hi - lo)
                ana = ana_all[i, k]
                errs.append(abs(fd - ana) / max(abs(fd), abs(ana), 1e-3 * np.abs(ana_all).max()))
    errs = np.array(errs)
    assert errs.max() < 1e-4, np.percentile(errs, [50, 90, 99])
