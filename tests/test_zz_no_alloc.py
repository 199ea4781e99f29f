"""The no-allocation forward entry point against the allocating one.

omnigs_lonlat_forward_noalloc exists for callers that cannot allocate device memory (a plugin in
an application that owns all device memory, a fixed-budget real-time loop that must not call
cudaMalloc): its state lives in a static device array inside the library.  Here it is called
through the C ABI twice in a row, on two different views, and each result is compared with
omnigs_lonlat_forward on caller-allocated buffers (the existing entry point), within the image
tolerance of the other parity tests.  This file is collected last so that a failure here leaves
every other test already run; it also passes on its own in a fresh process.
"""
import ctypes

import pytest
import torch

from omnigs_b200 import capi, lonlat, scenes

pytestmark = pytest.mark.gpu

IMG_ATOL = 1e-4


def _noalloc_forward(g: lonlat.GaussianTensors, cam: lonlat.Camera):
    out = torch.empty(3, cam.height, cam.width, device="cuda")
    radii = torch.empty(g.P, dtype=torch.int32, device="cuda")
    a = capi.ForwardArgs()
    a.P, a.D, a.M, a.W, a.H = g.P, 3, g.M, cam.width, cam.height
    a.background, a.means3D, a.shs = capi.ptr(cam.background), capi.ptr(g.means3D), capi.ptr(g.shs)
    a.opacities, a.scales, a.rotations = capi.ptr(g.opacities), capi.ptr(g.scales), capi.ptr(g.rotations)
    a.scale_modifier = 1.0
    a.viewmatrix, a.campos = capi.ptr(cam.viewmatrix), capi.ptr(cam.campos)
    a.out_color, a.radii = capi.ptr(out), capi.ptr(radii)
    n = ctypes.c_int(-1)
    rc = capi.lib().omnigs_lonlat_forward_noalloc(ctypes.byref(a), ctypes.byref(n),
                                                  capi.stream_handle())
    capi.check(rc, "omnigs_lonlat_forward_noalloc")
    return out, radii, n.value


def test_noalloc_forward_matches_the_allocating_forward_twice(cuda):
    W, H = 512, 256
    g = scenes.make_gaussians(10_000, seed=21)
    gt = lonlat.GaussianTensors.from_numpy(g)
    views = [scenes.identity_view(W, H),
             scenes.make_view(W, H, (0.3, -0.2, 0.1), scenes.rotation_yaw_pitch(1.3, -0.3))]
    for i, v in enumerate(views):
        cam = lonlat.Camera.from_view(v, background=(0.05 * i, 0.1, 0.2))
        img, radii, n, _ = lonlat.rasterize(gt, cam)
        img2, radii2, n2 = _noalloc_forward(gt, cam)
        torch.cuda.synchronize()
        assert n2 == n
        assert torch.equal(radii2, radii)
        assert float((img2 - img).abs().max()) <= IMG_ATOL


def test_noalloc_forward_rejects_scenes_over_its_limits(cuda):
    g = scenes.make_gaussians(40_000, seed=22)  # above the 32768-Gaussian limit
    gt = lonlat.GaussianTensors.from_numpy(g)
    cam = lonlat.Camera.from_view(scenes.identity_view(64, 32))
    with pytest.raises(capi.OmnigsError, match="exceeds the no-allocation limit"):
        _noalloc_forward(gt, cam)
    small = lonlat.GaussianTensors.from_numpy(scenes.make_gaussians(1000, seed=22))
    big_image = lonlat.Camera.from_view(scenes.identity_view(1024, 512))  # above 512 x 512 pixels
    with pytest.raises(capi.OmnigsError, match="exceeds the no-allocation limit"):
        _noalloc_forward(small, big_image)


def test_noalloc_forward_reports_instance_overflow_then_recovers(cuda):
    """Instances that overflow the rest of the array are detected on the device and reported as a
    capacity error; the next call starts from a clean state (the array keeps the failed call's
    contents, and the forward clears its header first) and matches the allocating forward."""
    W, H = 512, 512
    g = scenes.make_gaussians(32_768, seed=23)
    g.scales *= 12.0  # large splats: ~30 tiles each, far more instances than the array holds
    big = lonlat.GaussianTensors.from_numpy(g)
    cam = lonlat.Camera.from_view(scenes.identity_view(W, H))
    with pytest.raises(capi.OmnigsError, match="instances exceed"):
        _noalloc_forward(big, cam)
    small = lonlat.GaussianTensors.from_numpy(scenes.make_gaussians(10_000, seed=24))
    img, radii, n, _ = lonlat.rasterize(small, cam)
    img2, radii2, n2 = _noalloc_forward(small, cam)
    torch.cuda.synchronize()
    assert n2 == n
    assert torch.equal(radii2, radii)
    assert float((img2 - img).abs().max()) <= IMG_ATOL
