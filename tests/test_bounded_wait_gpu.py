"""A bounded device wait made to run out, end to end through the C ABI.

The duplicate pass joins a decoupled look-back across blocks: block t waits for block t-1's scan
word.  Every such wait is bounded: after its poll limit it gives up, sets OMNIGS_STATUS_LOOKBACK in
the status word and lets the kernel finish (no trap, no hang).  omnigs_debug_lookback_timeout runs
a forward up to that pass with scan tile 0 taken by no block, so tile 1 waits on a word that nothing
ever sets; the test checks that the call comes back promptly with OMNIGS_ERR_DEVICE and the status
bit, and that the same buffers then serve a normal forward whose image equals a fresh one (the
context and the state stay usable).
"""
import ctypes
import time

import pytest
import torch

from omnigs_b200 import capi, lonlat, scenes

pytestmark = pytest.mark.gpu

STATUS_LOOKBACK = 2
ERR_DEVICE = 6


def test_lookback_wait_that_nothing_satisfies_gives_up_and_reports(cuda):
    W, H, P = 512, 256, 10_000
    g = lonlat.GaussianTensors.from_numpy(scenes.make_gaussians(P, seed=51))
    cam = lonlat.Camera.from_view(scenes.identity_view(W, H))
    ref_img, ref_radii, n, _ = lonlat.rasterize(g, cam)
    state = lonlat.LonlatState(P, W, H, n + n // 4 + 4096)
    out = torch.empty(3, H, W, device="cuda")
    radii = torch.empty(P, dtype=torch.int32, device="cuda")
    a = state._fwd_args(g, cam, out, radii, 3, 1.0)
    status = ctypes.c_uint32(0)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    rc = capi.lib().omnigs_debug_lookback_timeout(
        ctypes.byref(a), state.geom.data_ptr(), state.geom.numel(), state.binning.data_ptr(),
        state.binning.numel(), state.image.data_ptr(), state.image.numel(), 2000, ctypes.byref(status),
        capi.stream_handle())
    elapsed = time.perf_counter() - t0
    assert rc == ERR_DEVICE, (rc, capi.lib().omnigs_last_error())
    assert status.value & STATUS_LOOKBACK
    assert b"gave up" in capi.lib().omnigs_last_error()
    assert elapsed < 10.0, elapsed
    # the context and the buffers are still good: a normal forward on them matches a fresh one
    state.forward(g, cam, out, radii)
    n2, st = state.status()
    assert st == 0 and n2 == n
    assert torch.equal(radii, ref_radii)
    assert torch.equal(out, ref_img)
