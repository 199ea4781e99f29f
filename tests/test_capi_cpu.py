"""CPU tests of the native libraries: the C-ABI library loads and exports every function that
include/omnigs_b200.h declares, size queries are consistent, argument validation happens before
any device work, and the LibTorch layer keeps the reference's host-side behaviour.  No GPU."""
import ctypes
import os
import re

import numpy as np
import pytest
import torch

from omnigs_b200 import capi, scenes, torch_ext

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    text = open(os.path.join(ROOT, "include", "omnigs_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(omnigs_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_the_bound_symbols():
    assert header_functions() == sorted(capi.EXPORTED)


def test_library_exports_every_declared_symbol():
    L = capi.lib()
    missing = [name for name in header_functions() if not hasattr(L, name)]
    assert not missing, missing
    assert b"sm_100a" in L.omnigs_version()


def test_buffer_sizes_and_capacity_inverse():
    assert capi.geom_bytes(0) > 0
    assert capi.geom_bytes(1000) < capi.geom_bytes(1001) or capi.geom_bytes(1000) <= capi.geom_bytes(2000)
    assert capi.image_bytes(512, 256) >= 512 * 256 * 8
    for c in [0, 1, 4095, 4096, 4097, 123_457, 8_227_376, 50_000_000]:
        b = capi.binning_bytes(c)
        assert capi.binning_capacity(b) >= c
        assert capi.binning_capacity(b - 1) < c or c == 0
    assert capi.binning_capacity(10) == -1


def _fake_args(**over):
    a = capi.ForwardArgs()
    a.P, a.D, a.M, a.W, a.H = 10, 3, 16, 64, 32
    fake = 0x10000
    for f in ("background", "means3D", "shs", "opacities", "scales", "rotations", "viewmatrix",
              "campos", "out_color", "radii"):
        setattr(a, f, fake)
    a.scale_modifier = 1.0
    for k, v in over.items():
        setattr(a, k, v)
    return a


@pytest.mark.parametrize("over,code", [
    (dict(P=-1), 1), (dict(D=4), 1), (dict(W=0), 1), (dict(M=8), 1),
    (dict(colors_precomp=0x10000), 1),            # both SH and colours
    (dict(shs=None), 1),                          # neither SH nor colours
    (dict(cov3D_precomp=0x10000), 1),             # both scale/rotation and cov3D
    (dict(rotations=None), 1),                    # half of the scale/rotation pair
    (dict(radii=None), 1),
    (dict(flags=2), 1),                           # an unknown OMNIGS_FLAG_* bit
])
def test_forward_argument_validation_precedes_device_work(over, code):
    a = _fake_args(**over)
    rc = capi.lib().omnigs_lonlat_forward(ctypes.byref(a), 0x10000, 1 << 30, 0x10000, 1 << 30,
                                          0x10000, 1 << 30, None)
    assert rc == code
    assert capi.lib().omnigs_last_error()


@pytest.mark.parametrize("over,code", [(dict(P=-1), 1), (dict(D=4), 1), (dict(radii=None), 1)])
def test_forward_early_status_validates_before_device_work(over, code):
    a = _fake_args(**over)
    n, st = ctypes.c_int(-1), ctypes.c_uint32(7)
    rc = capi.lib().omnigs_lonlat_forward_early_status(ctypes.byref(a), 0x10000, 1 << 30, 0x10000, 1 << 30,
                                                       0x10000, 1 << 30, ctypes.byref(n), ctypes.byref(st), None)
    assert rc == code and capi.lib().omnigs_last_error()
    # the two host outputs are required
    a = _fake_args()
    rc = capi.lib().omnigs_lonlat_forward_early_status(ctypes.byref(a), 0x10000, 1 << 30, 0x10000, 1 << 30,
                                                       0x10000, 1 << 30, None, ctypes.byref(st), None)
    assert rc == 1 and b"num_rendered" in capi.lib().omnigs_last_error()


def test_forward_rejects_small_buffers():
    a = _fake_args()
    rc = capi.lib().omnigs_lonlat_preprocess(ctypes.byref(a), 0x10000, 16, None)
    assert rc == 2
    assert b"geometry" in capi.lib().omnigs_last_error()


def test_misaligned_workspace_buffers_are_rejected_before_device_work():
    # the kernels move their records with 16-byte accesses; cudaMalloc and torch align to 256 B
    L = capi.lib()
    a = _fake_args()
    off = 0x10008
    assert L.omnigs_lonlat_preprocess(ctypes.byref(a), off, 1 << 30, None) == 1
    assert b"16-byte" in L.omnigs_last_error()
    for geom, binning, image in ((off, 0x10000, 0x10000), (0x10000, off, 0x10000), (0x10000, 0x10000, off)):
        rc = L.omnigs_lonlat_forward(ctypes.byref(a), geom, 1 << 30, binning, 1 << 30, image, 1 << 30, None)
        assert rc == 1 and b"16-byte" in L.omnigs_last_error()
    b = capi.BackwardArgs()
    b.P, b.D, b.M, b.W, b.H, b.R = 10, 3, 16, 64, 32, 10
    for f, _ in capi.BackwardArgs._fields_:
        if f not in ("P", "D", "M", "W", "H", "R", "scale_modifier", "colors_precomp",
                     "cov3D_precomp", "dL_dconic", "flags"):
            setattr(b, f, 0x10000)
    rc = L.omnigs_lonlat_backward(ctypes.byref(b), 0x10000, 1 << 30, off, 1 << 30, 0x10000, 1 << 30, None)
    assert rc == 1 and b"16-byte" in L.omnigs_last_error()
    ba, keep = _fake_batch()
    assert L.omnigs_batch_forward(ctypes.byref(ba), off, 1 << 40, 0x10000, 1 << 40, None) == 1
    assert L.omnigs_batch_forward(ctypes.byref(ba), 0x10000, 1 << 40, off, 1 << 40, None) == 1


def test_backward_rejects_capacity_mismatch():
    a = capi.BackwardArgs()
    a.P, a.D, a.M, a.W, a.H, a.R = 10, 3, 16, 64, 32, 1000
    for f, _ in capi.BackwardArgs._fields_:
        if f not in ("P", "D", "M", "W", "H", "R", "scale_modifier", "colors_precomp",
                     "cov3D_precomp", "dL_dconic", "flags"):
            setattr(a, f, 0x10000)
    small = capi.binning_bytes(100)
    rc = capi.lib().omnigs_lonlat_backward(ctypes.byref(a), 0x10000, capi.geom_bytes(10), 0x10000,
                                           small, 0x10000, capi.image_bytes(64, 32), None)
    assert rc == 5


def test_mark_visible_rejects_invalid_camera():
    rc = capi.lib().omnigs_mark_visible(10, None, None, 2, None, None)
    assert rc == 1 and b"camera_type" in capi.lib().omnigs_last_error()


def _cpu_forward_args(P, camera_type=3, shape=(None, 3)):
    means = torch.zeros(P if shape[0] is None else shape[0], shape[1])
    z = torch.empty(0)
    return (torch.zeros(3), means, z, torch.zeros(P, 1), torch.zeros(P, 3), torch.zeros(P, 4), 1.0, z,
            torch.eye(4), torch.eye(4), 0.0, 0.0, 16, 32, torch.zeros(P, 16, 3), 3, torch.zeros(3),
            False, camera_type, False)


def test_torch_layer_rejects_bad_means_shape_like_the_reference():
    ext = torch_ext()
    with pytest.raises(RuntimeError, match=r"means3D must have dimensions \(num_points, 3\)"):
        ext.rasterize_gaussians_cuda(*_cpu_forward_args(4, shape=(4, 2)))


def test_torch_layer_empty_scene_returns_zero_image():
    ext = torch_ext()
    n, color, radii, geom, binning, img = ext.rasterize_gaussians_cuda(*_cpu_forward_args(0, camera_type=7))
    assert n == 0 and color.shape == (3, 16, 32) and float(color.abs().sum()) == 0.0
    assert radii.shape == (0,) and geom.numel() == binning.numel() == img.numel() == 0


@pytest.mark.parametrize("camera_type,msg", [(7, r"\[CudaRasterizer\]Invalid camera_type"),
                                             (1, r"camera_type 1 \(pinhole\) is not provided")])
def test_torch_layer_camera_type_errors(camera_type, msg):
    ext = torch_ext()
    with pytest.raises(RuntimeError, match=msg):
        ext.rasterize_gaussians_cuda(*_cpu_forward_args(4, camera_type=camera_type))


def test_python_rasterizer_argument_checks():
    from omnigs_b200 import GaussianRasterizationSettings, GaussianRasterizer
    s = GaussianRasterizationSettings(16, 32, 0.0, 0.0, torch.zeros(3), 1.0, torch.eye(4), torch.eye(4),
                                      3, torch.zeros(3))
    r = GaussianRasterizer(s)
    m = torch.zeros(4, 3)
    with pytest.raises(RuntimeError, match="excatly one of either SHs or precomputed colors"):
        r(m, m, torch.zeros(4, 1), scales=m, rotations=torch.zeros(4, 4))
    with pytest.raises(RuntimeError, match="scale/rotation pair or precomputed 3D covariance"):
        r(m, m, torch.zeros(4, 1), shs=torch.zeros(4, 16, 3), scales=m)


def test_scene_generators_are_seeded_and_follow_the_distributions():
    a = scenes.make_gaussians(20000, seed=5)
    b = scenes.make_gaussians(20000, seed=5)
    np.testing.assert_array_equal(a.means3D, b.means3D)
    r = np.linalg.norm(a.means3D, axis=1)
    assert r.min() >= 1.0 - 1e-5 and r.max() <= 5.0 + 1e-5
    # uniform in volume: P(r < 3) = (27 - 1) / (125 - 1)
    assert abs((r < 3).mean() - 26 / 124) < 0.01
    assert abs(np.log(a.scales).mean() - np.log(0.02)) < 0.01
    np.testing.assert_allclose(np.linalg.norm(a.rotations, axis=1), 1.0, rtol=1e-6)
    assert a.shs.shape == (20000, 16, 3)
    assert abs(a.shs[:, 0].std() - 0.5) < 0.01 and abs(a.shs[:, 1:].std() - 0.05) < 0.001
    p = scenes.make_gaussians(20000, seed=6, pole_fraction=0.3)
    lat = np.degrees(np.arcsin(p.means3D[:, 1] / np.linalg.norm(p.means3D, axis=1)))
    assert abs((np.abs(lat) > 80).mean() - 0.3 - 0.7 * (1 - np.sin(np.radians(80)))) < 0.01


def test_views_follow_reference_conventions():
    v = scenes.make_view(64, 32, (1.0, 2.0, 3.0), scenes.rotation_yaw_pitch(0.4, -0.2))
    Tcw = v.viewmatrix.T.astype(np.float64)
    # the camera centre maps to the camera-space origin; campos is that centre
    np.testing.assert_allclose((Tcw @ np.array([1.0, 2.0, 3.0, 1.0]))[:3], 0.0, atol=1e-5)
    np.testing.assert_allclose(v.campos, [1.0, 2.0, 3.0], atol=1e-5)


def test_batch_state_bytes_validates_the_views():
    one = capi.batch_state_bytes(1000, [(512, 256)])
    two = capi.batch_state_bytes(1000, [(512, 256), (1024, 512)])
    assert 0 < one < two
    assert capi.batch_state_bytes(2000, [(512, 256)]) > one
    assert capi.batch_state_bytes(1000, []) == 0
    assert capi.batch_state_bytes(1000, [(64, 32)] * (capi.MAX_BATCH_VIEWS + 1)) == 0
    assert capi.batch_state_bytes(1000, [(64, 32)] * capi.MAX_BATCH_VIEWS) > 0
    assert capi.batch_state_bytes(1000, [(0, 256)]) == 0
    assert capi.batch_state_bytes(-1, [(512, 256)]) == 0


def _fake_batch(V=2, **over):
    fake = 0x10000
    views = (capi.BatchView * max(V, 1))()
    for v in range(V):
        views[v].W, views[v].H = 64 * (v + 1), 32 * (v + 1)
        views[v].out_color = fake
        views[v].dL_dout_color = fake
    a = capi.BatchArgs()
    a.P, a.D, a.M, a.V = 10, 3, 16, V
    for f in ("means3D", "shs", "opacities", "scales", "rotations", "viewmatrices", "campos", "backgrounds"):
        setattr(a, f, fake)
    a.scale_modifier = 1.0
    a.views = views
    for k, v in over.items():
        setattr(a, k, v)
    return a, views


@pytest.mark.parametrize("over,code", [
    (dict(V=0), 1), (dict(V=capi.MAX_BATCH_VIEWS + 1), 1), (dict(sh_dtype=2), 1), (dict(fp64_poles=3), 1),
    (dict(M=17), 1), (dict(D=4), 1), (dict(backgrounds=None), 1), (dict(opacities=None), 1),
    (dict(colors_precomp=0x10000), 1), (dict(cov3D_precomp=0x10000), 1),
])
def test_batch_entry_points_reject_bad_arguments_before_device_work(over, code):
    a, keep = _fake_batch(**over)
    L = capi.lib()
    assert L.omnigs_batch_forward(ctypes.byref(a), 0x10000, 1 << 40, 0x10000, 1 << 40, None) == code
    assert L.omnigs_last_error()
    g = capi.BatchGrads()
    for f, _ in capi.BatchGrads._fields_:
        setattr(g, f, 0x10000)
    assert L.omnigs_batch_backward(ctypes.byref(a), ctypes.byref(g), 0x10000, 1 << 40, 0x10000, 1 << 40,
                                   None) == code


def test_batch_state_too_small_is_rejected():
    a, keep = _fake_batch()
    L = capi.lib()
    need = capi.batch_state_bytes(10, [(64, 32), (128, 64)])
    assert L.omnigs_batch_forward(ctypes.byref(a), 0x10000, need - 1, 0x10000, 1 << 40, None) == 2


def test_loss_workspace_and_validation():
    L = capi.lib()
    assert L.omnigs_l1_dssim_workspace_bytes(3, 1024, 2048) >= 3 * 3 * 1024 * 2048 * 4
    assert L.omnigs_l1_dssim_workspace_bytes(0, 10, 10) == 0
    f = 0x10000
    big = 1 << 40
    assert L.omnigs_l1_dssim(f, f, 3, 64, 32, 65, 0.2, f, f, f, big, None) == 1   # rows > H
    assert L.omnigs_l1_dssim(f, f, 3, 64, 32, 64, 1.5, f, f, f, big, None) == 1   # lambda outside [0, 1]
    assert L.omnigs_l1_dssim(None, f, 3, 64, 32, 64, 0.2, f, f, f, big, None) == 1
    assert L.omnigs_l1_dssim(f, f, 3, 64, 32, 64, 0.2, f, f, f, 16, None) == 2    # workspace too small


def test_adam_validation():
    L = capi.lib()
    prm, st, act = capi.GaussianParams(), capi.AdamState(), capi.Activated()
    prm.P, prm.M = 10, 17
    assert L.omnigs_adam_step(ctypes.byref(prm), ctypes.byref(st), ctypes.byref(act), *([0x10000] * 6),
                              None) == 1
    prm.M = 16  # pointers still NULL
    assert L.omnigs_adam_step(ctypes.byref(prm), ctypes.byref(st), ctypes.byref(act), *([0x10000] * 6),
                              None) == 1
    assert L.omnigs_activate(ctypes.byref(prm), ctypes.byref(act), None) == 1


def test_blend_batch_setting():
    from omnigs_b200 import batch
    assert batch.get_blend_batch() == (128, 128)  # the library's defaults
    with pytest.raises(capi.OmnigsError):
        batch.set_blend_batch(100, 256)
    batch.set_blend_batch(128, 512)
    assert batch.get_blend_batch() == (128, 512)
    batch.set_blend_batch(128, 128)  # back to the library's defaults
    a, keep = _fake_batch()
    r = capi.TuneResult()
    assert capi.lib().omnigs_batch_autotune(ctypes.byref(a), 0x10000, 1 << 40, 0x10000, 1 << 40, 0,
                                            ctypes.byref(r), None) == 1  # repeats < 1


@pytest.mark.parametrize("sizes,P,passes", [
    ([(3072, 1536)] * 4 + [(512, 256)], 20_000, 2),   # 74,240 tiles (17 bits) vs 18,432 per view (15)
    ([(3072, 1536)] * 4 + [(512, 256)], 200, 2),      # small P: per view as well
    ([(3072, 1536)], 20_000, 2),                      # one view: its own 15-bit ids
    ([(2048, 1024), (512, 256), (3072, 1536)], 20_000, 2),  # 27,136 tiles: two passes either way
])
def test_batch_tile_sort_runs_per_view_when_it_saves_a_pass(sizes, P, passes):
    """The batched tile sort works on view-local tile ids when that needs fewer digit passes than
    the batch's global ids; state_view reports the passes of the sort that runs."""
    V = len(sizes)
    W = (ctypes.c_int * V)(*[w for w, _ in sizes])
    H = (ctypes.c_int * V)(*[h for _, h in sizes])
    sv = capi.BatchStateView()
    assert capi.lib().omnigs_batch_state_view(ctypes.c_void_p(0x10000), P, V, W, H, ctypes.byref(sv)) == 0
    assert sv.tile_passes == passes


def test_checkpointing_image_buffer_holds_only_tile_ranges():
    W, H = 2048, 1024
    full, ckpt = capi.image_bytes(W, H), capi.image_bytes(W, H, capi.FLAG_RECOMPUTE_T)
    tiles = (W // 16) * (H // 16)
    assert ckpt == 8 * tiles
    assert full - ckpt == 8 * W * H
