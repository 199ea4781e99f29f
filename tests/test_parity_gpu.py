"""GPU parity of the CUDA path (through the C ABI) against the FP64 oracle.

Each stage is compared on the same inputs: the oracle's binning and blend stages are fed with the
CUDA preprocess's float outputs, so integer stages are compared bit for bit and float stages within
tolerance.  Tolerances: image <= 1e-4 absolute; gradients <= 1e-3 normwise relative
(max |a - b| / max |b| per tensor).
"""
import numpy as np
import pytest
import torch

import helpers
import oracle
from omnigs_b200 import lonlat, scenes

pytestmark = pytest.mark.gpu

IMG_ATOL = 1e-4
GRAD_RTOL = 1e-3


def _scene(P, W, H, seed=0, view=None, bg=(0.0, 0.0, 0.0)):
    g = scenes.make_gaussians(P, seed=seed)
    v = view or scenes.identity_view(W, H)
    return g, v, lonlat.GaussianTensors.from_numpy(g), lonlat.Camera.from_view(v, background=bg)


def test_preprocess_matches_fp64_oracle(cuda):
    g, v, gt, cam = _scene(10_000, 512, 256)
    cu = helpers.run_cuda(gt, cam)
    pre = oracle.preprocess(g.means3D, g.scales, g.rotations, g.opacities, g.shs, v.viewmatrix,
                            v.campos, 512, 256)
    radii = helpers.to_np(cu["radii"])
    vis = (radii > 0) & (pre["radii"] > 0)
    # integer outputs may differ from FP64 only where a value sits on a ceil/truncation boundary
    assert (radii != pre["radii"]).mean() < 2e-3
    assert (helpers.to_np(cu["tiles_touched"]).view(np.uint32) != pre["tiles_touched"]).mean() < 2e-3
    lat = np.degrees(np.arcsin(np.abs(g.means3D[:, 1]) / np.linalg.norm(g.means3D, axis=1)))
    ok = vis & (lat < 80)
    np.testing.assert_allclose(helpers.to_np(cu["means2D"])[ok], pre["means2D"][ok], atol=2e-3, rtol=0)
    np.testing.assert_allclose(helpers.to_np(cu["depths"])[vis], pre["depths"][vis], rtol=1e-6)
    np.testing.assert_allclose(helpers.to_np(cu["rgb"])[vis], pre["rgb"][vis], atol=1e-5)
    con = helpers.to_np(cu["conic_opacity"])
    np.testing.assert_allclose(con[ok, 3], pre["conic_opacity"][ok, 3], rtol=0, atol=0)
    rel = np.abs(con[ok, :3] - pre["conic_opacity"][ok, :3]) / np.abs(pre["conic_opacity"][ok, :3]).max(1, keepdims=True)
    assert rel.max() < 1e-3


def test_binning_is_bit_exact_with_the_oracle(cuda):
    g, v, gt, cam = _scene(10_000, 512, 256)
    cu = helpers.run_cuda(gt, cam)
    ref = helpers.oracle_stagewise(cu, g, v, None, np.zeros(3, np.float32))["binning"]
    assert cu["num_rendered"] == ref["num_rendered"]
    np.testing.assert_array_equal(helpers.to_np(cu["keys"]).view(np.uint64), ref["keys"])
    np.testing.assert_array_equal(helpers.to_np(cu["point_list"]).view(np.uint32), ref["point_list"])
    np.testing.assert_array_equal(helpers.to_np(cu["ranges"]).view(np.uint32), ref["ranges"])


@pytest.mark.parametrize("W,H,seed", [(512, 256, 0), (500, 250, 1), (96, 48, 2)])
def test_forward_and_backward_match_the_oracle(cuda, W, H, seed):
    P = 10_000 if W >= 500 else 800
    view = scenes.make_view(W, H, (0.2, -0.1, 0.3), scenes.rotation_yaw_pitch(0.7, 0.2)) if seed else None
    g, v, gt, cam = _scene(P, W, H, seed=seed, view=view, bg=(0.1, 0.3, 0.6) if seed == 1 else (0, 0, 0))
    dpix = scenes.upstream_grad(W, H, seed=seed)
    cu = helpers.run_cuda(gt, cam, torch.from_numpy(dpix).cuda())
    o = helpers.oracle_stagewise(cu, g, v, dpix, helpers.to_np(cam.background))
    img = helpers.to_np(cu["image"])
    err = np.abs(img - o["forward"]["image"])
    assert err.max() <= IMG_ATOL, err.max()
    assert (helpers.to_np(cu["n_contrib"]).view(np.uint32) != o["forward"]["n_contrib"]).mean() < 1e-3
    np.testing.assert_allclose(helpers.to_np(cu["final_T"]), o["forward"]["final_T"], atol=1e-6, rtol=1e-4)
    gr = cu["grads"]
    rb, pb = o["render_backward"], o["preprocess_backward"]
    pairs = [("dL_dmeans2D", rb["dL_dmean2D"]), ("dL_dcolors", rb["dL_dcolor"]),
             ("dL_dopacity", rb["dL_dopacity"].reshape(-1, 1)), ("dL_dmeans3D", pb["dL_dmeans3D"]),
             ("dL_dcov3D", pb["dL_dcov3D"]), ("dL_dsh", pb["dL_dsh"]), ("dL_dscales", pb["dL_dscales"]),
             ("dL_drotations", pb["dL_drotations"])]
    for name, want in pairs:
        got = helpers.to_np(getattr(gr, name))
        assert helpers.normwise_rel(got, want) < GRAD_RTOL, (name, helpers.normwise_rel(got, want))
    con = helpers.to_np(gr.dL_dconic)
    assert helpers.normwise_rel(con[:, [0, 1, 3]], rb["dL_dconic"][:, [0, 1, 3]]) < GRAD_RTOL


def test_end_to_end_against_the_pure_fp64_pipeline(cuda):
    """Whole-pipeline comparison against the FP64 oracle (its own preprocess and binning)."""
    W, H = 512, 256
    g, v, gt, cam = _scene(10_000, W, H, seed=4)
    dpix = scenes.upstream_grad(W, H, seed=4)
    cu = helpers.run_cuda(gt, cam, torch.from_numpy(dpix).cuda())
    ref = oracle.forward_backward(g, v, dpix)
    err = np.abs(helpers.to_np(cu["image"]) - ref["image"])
    mse = float((err ** 2).mean())
    psnr_gap = 10 * np.log10(1.0 / max(mse, 1e-30))
    assert np.quantile(err, 0.999) < IMG_ATOL and psnr_gap > 60, (err.max(), psnr_gap)
    for name, key in [("dL_dmeans3D", "dL_dmeans3D"), ("dL_dsh", "dL_dsh"), ("dL_dopacity", "dL_dopacity")]:
        got = helpers.to_np(getattr(cu["grads"], name))
        assert helpers.normwise_rel(got, ref[key]) < 2e-2, (name, helpers.normwise_rel(got, ref[key]))


def test_precomputed_colors_and_covariance_paths(cuda):
    W, H = 256, 128
    g, v, gt, cam = _scene(3000, W, H, seed=5)
    pre = oracle.preprocess(g.means3D, g.scales, g.rotations, g.opacities, g.shs, v.viewmatrix,
                            v.campos, W, H)
    colors = np.random.default_rng(0).random((g.P, 3)).astype(np.float32)
    gt2 = lonlat.GaussianTensors(means3D=gt.means3D, opacities=gt.opacities,
                                 colors_precomp=torch.from_numpy(colors).cuda(),
                                 cov3D_precomp=torch.from_numpy(pre["cov3D"].astype(np.float32)).cuda())
    dpix = scenes.upstream_grad(W, H, seed=5)
    cu = helpers.run_cuda(gt2, cam, torch.from_numpy(dpix).cuda())
    np.testing.assert_array_equal(helpers.to_np(cu["rgb"])[helpers.to_np(cu["radii"]) > 0],
                                  colors[helpers.to_np(cu["radii"]) > 0])
    o = helpers.oracle_stagewise(cu, g, v, None, np.zeros(3, np.float32))
    assert np.abs(helpers.to_np(cu["image"]) - o["forward"]["image"]).max() <= IMG_ATOL
    gr = cu["grads"]
    assert gr.dL_dsh.shape == (g.P, 0, 3)
    assert float(gr.dL_dscales.abs().sum()) == 0.0 and float(gr.dL_drotations.abs().sum()) == 0.0
    assert float(gr.dL_dcov3D.abs().sum()) > 0.0 and float(gr.dL_dcolors.abs().sum()) > 0.0


@pytest.mark.parametrize("D", [0, 1, 2])
def test_lower_sh_degrees(cuda, D):
    W, H = 256, 128
    g, v, gt, cam = _scene(2000, W, H, seed=6)
    dpix = scenes.upstream_grad(W, H, seed=6)
    cu = helpers.run_cuda(gt, cam, torch.from_numpy(dpix).cuda(), D=D)
    pre = oracle.preprocess(g.means3D, g.scales, g.rotations, g.opacities, g.shs, v.viewmatrix,
                            v.campos, W, H, D=D)
    vis = helpers.to_np(cu["radii"]) > 0
    np.testing.assert_allclose(helpers.to_np(cu["rgb"])[vis], pre["rgb"][vis], atol=1e-5)
    dsh = helpers.to_np(cu["grads"].dL_dsh)
    assert np.abs(dsh[:, (D + 1) ** 2:]).max() == 0.0
    assert np.abs(dsh[:, :(D + 1) ** 2]).max() > 0.0


def test_edge_cases_empty_and_fully_culled(cuda):
    W, H = 64, 32
    cam = lonlat.Camera.from_view(scenes.identity_view(W, H), background=(0.25, 0.5, 0.75))
    # every Gaussian inside the r^2 <= 0.04 near-cull sphere
    g = scenes.make_gaussians(500, seed=7)
    g.means3D *= 0.15 / np.linalg.norm(g.means3D, axis=1, keepdims=True)
    gt = lonlat.GaussianTensors.from_numpy(g)
    dpix = torch.randn(3, H, W, device="cuda")
    cu = helpers.run_cuda(gt, cam, dpix)
    assert cu["num_rendered"] == 0 and int(cu["radii"].abs().sum()) == 0
    np.testing.assert_allclose(helpers.to_np(cu["image"])[:, 3, 5], [0.25, 0.5, 0.75])
    for name in ("dL_dmeans3D", "dL_dsh", "dL_dscales", "dL_drotations", "dL_dopacity", "dL_dmeans2D"):
        assert float(getattr(cu["grads"], name).abs().sum()) == 0.0
    # no Gaussians at all: the reference returns its zero-initialised image
    e = lonlat.GaussianTensors(means3D=torch.zeros(0, 3, device="cuda"), opacities=torch.zeros(0, 1, device="cuda"),
                               shs=torch.zeros(0, 16, 3, device="cuda"), scales=torch.zeros(0, 3, device="cuda"),
                               rotations=torch.zeros(0, 4, device="cuda"))
    img, radii, n, _ = lonlat.rasterize(e, cam)
    assert n == 0 and float(img.abs().sum()) == 0.0


def test_capacity_overflow_is_reported_and_resumable(cuda):
    W, H = 256, 128
    g, v, gt, cam = _scene(3000, W, H, seed=8)
    state = lonlat.LonlatState(g.P, W, H, capacity=100)
    out = torch.empty(3, H, W, device="cuda")
    radii = torch.empty(g.P, dtype=torch.int32, device="cuda")
    state.forward(gt, cam, out, radii)
    n, st = state.status()
    assert st & 1 and n > 100
    state.resize_capacity(n)
    state.render(gt, cam, out, radii)
    n2, st2 = state.status()
    assert st2 == 0 and n2 == n
    full = helpers.run_cuda(gt, cam)
    torch.testing.assert_close(out, full["image"], rtol=0, atol=0)


def test_forward_early_status_matches_forward_and_read_status(cuda):
    """The forward that returns num_rendered and the status once the binning has run gives the same
    image, radii, per-pixel state, count and status as forward + read_status, also when the
    binning capacity is too small (then the count is the required capacity)."""
    W, H = 1024, 512
    g, v, gt, cam = _scene(40_000, W, H, seed=21)
    runs = {}
    for mode in ("read_status", "early"):
        state = lonlat.LonlatState(g.P, W, H, capacity=2_000_000)
        out = torch.empty(3, H, W, device="cuda")
        radii = torch.empty(g.P, dtype=torch.int32, device="cuda")
        for _ in range(2):  # the second call reuses the thread's pinned status slot
            if mode == "early":
                n, st = state.forward_early_status(gt, cam, out, radii)
            else:
                state.forward(gt, cam, out, radii)
                n, st = state.status()
        torch.cuda.synchronize()
        iv = state.image_view()
        runs[mode] = (n, st, out.clone(), radii.clone(), iv["final_T"].clone(), iv["n_contrib"].clone())
    a, b = runs["read_status"], runs["early"]
    assert a[0] == b[0] and a[0] > 0 and a[1] == b[1] == 0
    for x, y in zip(a[2:], b[2:]):
        assert torch.equal(x, y)
    small = lonlat.LonlatState(g.P, W, H, capacity=100)
    out = torch.empty(3, H, W, device="cuda")
    radii = torch.empty(g.P, dtype=torch.int32, device="cuda")
    n, st = small.forward_early_status(gt, cam, out, radii)
    assert st & 1 and n == a[0]
    small.resize_capacity(n)
    small.render(gt, cam, out, radii)
    assert small.status() == (a[0], 0)
    assert torch.equal(out, a[2])


def test_repeated_backward_is_consistent(cuda):
    """A second backward on the same state gives the same gradients (the accumulator records are
    consumed and cleared, nothing leaks between calls).  The blend adds its per-splat sums with
    float atomics whose order varies between runs, so the comparison is normwise (max |a - b| over
    max |b|, per tensor) at 1e-5; a leaked accumulation would show as an error of order 1."""
    W, H = 256, 128
    g, v, gt, cam = _scene(3000, W, H, seed=9)
    img, radii, n, state = lonlat.rasterize(gt, cam)
    dpix = torch.randn(3, H, W, device="cuda")
    g1 = lonlat.Gradients.empty(g.P, 16, "cuda")
    g2 = lonlat.Gradients.empty(g.P, 16, "cuda")
    state.backward(gt, cam, radii, dpix, g1, R=n)
    state.backward(gt, cam, radii, dpix, g2, R=n)
    for name in ("dL_dmeans3D", "dL_dsh", "dL_dopacity", "dL_dmeans2D"):
        a, b = getattr(g1, name).double(), getattr(g2, name).double()
        assert float((a - b).abs().max()) <= 1e-5 * float(b.abs().max()), name


def test_full_size_properties(cuda):
    """1M Gaussians at 2048 x 1024: size-independent properties of every stage."""
    W, H = 2048, 1024
    g, v, gt, cam = _scene(1_000_000, W, H, seed=0)
    dpix = torch.from_numpy(scenes.upstream_grad(W, H)).cuda()
    cu = helpers.run_cuda(gt, cam, dpix)
    n = cu["num_rendered"]
    tt = helpers.to_np(cu["tiles_touched"]).view(np.uint32).astype(np.int64)
    assert n == int(tt.sum()) and n > 1_000_000
    keys = helpers.to_np(cu["keys"]).view(np.uint64)
    assert np.all(keys[1:] >= keys[:-1])
    pl = helpers.to_np(cu["point_list"]).astype(np.int64)
    # every Gaussian appears exactly tiles_touched times; ties keep index order
    np.testing.assert_array_equal(np.bincount(pl, minlength=g.P), tt)
    tie = keys[1:] == keys[:-1]
    assert np.all(pl[1:][tie] > pl[:-1][tie])
    r = helpers.to_np(cu["ranges"]).astype(np.int64)
    assert int((r[:, 1] - r[:, 0]).sum()) == n
    tile_of = (keys >> np.uint64(32)).astype(np.int64)
    nonempty = r[:, 1] > r[:, 0]
    assert np.all(tile_of[r[nonempty, 0]] == np.nonzero(nonempty)[0])
    assert torch.isfinite(cu["image"]).all()
    for name in ("dL_dmeans3D", "dL_dsh", "dL_dscales", "dL_drotations", "dL_dopacity"):
        assert torch.isfinite(getattr(cu["grads"], name)).all(), name
    # the whole blend against the FP64 oracle, from the same intermediates.  Pixels here blend
    # ~450 splats before saturating, so FP32 accumulation differs from FP64 by a few 1e-4 at
    # worst; the FP32 path itself is compared bit for bit with the reference in
    # test_reference_gpu.py.
    o = helpers.oracle_stagewise(cu, g, v, None, np.zeros(3, np.float32))
    err = np.abs(helpers.to_np(cu["image"]) - o["forward"]["image"])
    assert np.quantile(err, 0.9999) <= IMG_ATOL and err.max() <= 1e-3, (np.quantile(err, 0.9999), err.max())


@pytest.mark.parametrize("clustered", [False, True])
def test_binning_is_bit_exact_with_long_tiles(cuda, clustered):
    """A tight cluster of splats puts more than 4096 instances in single tiles (and many equal
    depths are impossible to order except by index); binning stays bit-exact."""
    W, H = 512, 256
    g = scenes.make_gaussians(6000, seed=12)
    if clustered:
        rng = np.random.default_rng(12)
        d = np.array([0.0, 0.0, 1.0]) + 0.004 * rng.standard_normal((g.P, 3))
        d /= np.linalg.norm(d, axis=1, keepdims=True)
        g.means3D[:] = (d * np.linalg.norm(g.means3D, axis=1, keepdims=True)).astype(np.float32)
        src = g.means3D[1::7].copy()
        g.means3D[0:7 * len(src):7] = src  # duplicated positions: equal depths
    v = scenes.identity_view(W, H)
    gt, cam = lonlat.GaussianTensors.from_numpy(g), lonlat.Camera.from_view(v)
    dpix = scenes.upstream_grad(W, H, seed=12)
    cu = helpers.run_cuda(gt, cam, torch.from_numpy(dpix).cuda())
    r = helpers.to_np(cu["ranges"]).astype(np.int64)
    longest = int((r[:, 1] - r[:, 0]).max())
    assert (longest > 4096) == clustered
    o = helpers.oracle_stagewise(cu, g, v, dpix, np.zeros(3, np.float32))
    np.testing.assert_array_equal(helpers.to_np(cu["keys"]).view(np.uint64), o["binning"]["keys"])
    np.testing.assert_array_equal(helpers.to_np(cu["point_list"]).view(np.uint32), o["binning"]["point_list"])
    np.testing.assert_array_equal(r.astype(np.uint32), o["binning"]["ranges"])
    assert np.abs(helpers.to_np(cu["image"]) - o["forward"]["image"]).max() <= IMG_ATOL


def test_depth_order_is_a_stable_sort_by_depth_bits(cuda):
    g = scenes.make_gaussians(50_000, seed=13)
    g.means3D[1::3] = g.means3D[0::3][: len(g.means3D[1::3])]  # many exactly equal depths
    gt, cam = lonlat.GaussianTensors.from_numpy(g), lonlat.Camera.from_view(scenes.identity_view(256, 128))
    cu = helpers.run_cuda(gt, cam)
    bits = helpers.to_np(cu["depths"]).view(np.uint32)
    want = np.argsort(bits, kind="stable").astype(np.int32)
    np.testing.assert_array_equal(helpers.to_np(cu["depth_order"]), want)
