"""TEST INFRASTRUCTURE ONLY: ctypes driver of the reference CUDA rasterizer rebuilt for sm_100a.

``oracle/_ref/libomnigs_ref.so`` is built by ``oracle/ref/Makefile`` from the reference's own
cuda_rasterizer sources.  Tests use it as the like-for-like GPU comparison: its integer stages
(radii, tiles_touched, offsets, sorted keys, point list, tile ranges) are the bit-exact target.
``available()`` is False where the library was not built (e.g. without the reference checkout).
"""
from __future__ import annotations

import ctypes
import os

import torch

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_ref", "libomnigs_ref.so")
_vp = ctypes.c_void_p
_lib = None


class RefStateView(ctypes.Structure):
    _fields_ = [(n, _vp) for n in ("tiles_touched", "point_offsets", "depths", "means2D",
                                   "conic_opacity", "rgb", "clamped", "cov3D", "keys",
                                   "point_list", "keys_unsorted", "point_list_unsorted", "ranges",
                                   "n_contrib", "accum_alpha")]


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        L = ctypes.CDLL(LIB_PATH)
        L.ref_create.restype = _vp
        L.ref_destroy.argtypes = [_vp]
        L.ref_forward.restype = ctypes.c_int
        L.ref_forward.argtypes = [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp, ctypes.c_int,
                                  ctypes.c_int, _vp, _vp, _vp, _vp, _vp, ctypes.c_float, _vp, _vp,
                                  _vp, _vp, _vp, _vp]
        L.ref_backward.argtypes = [_vp, ctypes.c_int, ctypes.c_int] + [_vp] * 5 + \
            [ctypes.c_float] + [_vp] * 15
        L.ref_copy.restype = ctypes.c_int
        L.ref_copy.argtypes = [_vp, _vp, ctypes.c_size_t]
        L.ref_state.restype = ctypes.c_int
        L.ref_state.argtypes = [_vp, ctypes.POINTER(RefStateView)]
        _lib = L
    return _lib


def _p(t):
    if t is None or t.numel() == 0:
        return None
    assert t.is_cuda and t.is_contiguous()
    return t.data_ptr()


def _copy_out(address: int, count: int, dtype) -> torch.Tensor:
    """Copy `count` elements at a raw device address into a new tensor."""
    out = torch.empty(count, dtype=dtype, device="cuda")
    if count:
        rc = lib().ref_copy(out.data_ptr(), address, count * out.element_size())
        assert rc == 0, f"cudaMemcpy failed: {rc}"
    return out


class ReferenceRasterizer:
    """One reference rasterizer instance (owns its growable state buffers)."""

    def __init__(self):
        self.h = lib().ref_create()

    def close(self):
        if self.h:
            lib().ref_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def forward(self, g, cam, D=3, scale_modifier=1.0, sync=True, out=None, radii=None):
        """Returns (image [3,H,W], radii [P], num_rendered).  ``g``/``cam`` as in omnigs_b200.lonlat.
        ``sync=False`` skips this wrapper's own device synchronisation (for timing)."""
        if sync:
            torch.cuda.synchronize()
        out = torch.zeros(3, cam.height, cam.width, dtype=torch.float32, device="cuda") if out is None else out
        radii = torch.zeros(g.P, dtype=torch.int32, device="cuda") if radii is None else radii
        R = lib().ref_forward(self.h, g.P, D, g.M, _p(cam.background), cam.width, cam.height,
                              _p(g.means3D), _p(g.shs), _p(g.colors_precomp), _p(g.opacities),
                              _p(g.scales), scale_modifier, _p(g.rotations), _p(g.cov3D_precomp),
                              _p(cam.viewmatrix), _p(cam.campos), _p(out), _p(radii))
        if sync:
            torch.cuda.synchronize()
        self.P, self.W, self.H = g.P, cam.width, cam.height
        return out, radii, int(R)

    def backward(self, g, cam, radii, dL_dpix, D=3, scale_modifier=1.0, sync=True):
        """Zero-initialised gradient outputs as the reference's LibTorch layer allocates them
        (src/rasterize_points.cu:200-208), then the reference backward."""
        P, M = g.P, g.M
        z = lambda *s: torch.zeros(*s, dtype=torch.float32, device="cuda")  # noqa: E731
        out = dict(dL_dmeans2D=z(P, 3), dL_dconic=z(P, 2, 2), dL_dopacity=z(P, 1),
                   dL_dcolors=z(P, 3), dL_dmeans3D=z(P, 3), dL_dcov3D=z(P, 6), dL_dsh=z(P, M, 3),
                   dL_dscales=z(P, 3), dL_drotations=z(P, 4))
        if sync:
            torch.cuda.synchronize()
        lib().ref_backward(self.h, D, M, _p(cam.background), _p(g.means3D), _p(g.shs),
                           _p(g.colors_precomp), _p(g.scales), scale_modifier, _p(g.rotations),
                           _p(g.cov3D_precomp), _p(cam.viewmatrix), _p(cam.campos), _p(radii),
                           _p(dL_dpix.contiguous()), _p(out["dL_dmeans2D"]), _p(out["dL_dconic"]),
                           _p(out["dL_dopacity"]), _p(out["dL_dcolors"]), _p(out["dL_dmeans3D"]),
                           _p(out["dL_dcov3D"]), _p(out["dL_dsh"]), _p(out["dL_dscales"]),
                           _p(out["dL_drotations"]))
        if sync:
            torch.cuda.synchronize()
        return out

    def state(self) -> dict:
        """Copies of the reference's intermediate arrays after the last forward."""
        v = RefStateView()
        R = lib().ref_state(self.h, ctypes.byref(v))
        P, N = self.P, self.W * self.H
        tiles = ((self.W + 15) // 16) * ((self.H + 15) // 16)
        return dict(
            num_rendered=int(R),
            tiles_touched=_copy_out(v.tiles_touched, P, torch.int32),
            point_offsets=_copy_out(v.point_offsets, P, torch.int32),
            depths=_copy_out(v.depths, P, torch.float32),
            means2D=_copy_out(v.means2D, 2 * P, torch.float32).view(P, 2),
            conic_opacity=_copy_out(v.conic_opacity, 4 * P, torch.float32).view(P, 4),
            rgb=_copy_out(v.rgb, 3 * P, torch.float32).view(P, 3),
            clamped=_copy_out(v.clamped, 3 * P, torch.uint8).view(P, 3),
            keys=_copy_out(v.keys, R, torch.int64),
            point_list=_copy_out(v.point_list, R, torch.int32),
            ranges=_copy_out(v.ranges, 2 * tiles, torch.int32).view(tiles, 2),
            n_contrib=_copy_out(v.n_contrib, N, torch.int32),
            final_T=_copy_out(v.accum_alpha, N, torch.float32),
        )
