"""Device-resident lonlat rasterization through the C ABI.

``LonlatState`` owns the three opaque state buffers (geometry, binning, image) of one view size and
runs the forward / backward entry points of include/omnigs_b200.h on torch CUDA tensors.  It is the
path the parity tests, the benchmark and the smoke test drive; the LibTorch surface
(``RasterizeGaussiansCUDA`` ...) sits on the same C ABI.
"""
from __future__ import annotations

import ctypes
import dataclasses

import torch

from . import capi


@dataclasses.dataclass
class GaussianTensors:
    """Scene parameters on the device, in the reference's layouts."""
    means3D: torch.Tensor                  # [P,3]
    opacities: torch.Tensor                # [P,1]
    shs: torch.Tensor | None = None        # [P,M,3]
    scales: torch.Tensor | None = None     # [P,3]
    rotations: torch.Tensor | None = None  # [P,4]
    colors_precomp: torch.Tensor | None = None  # [P,3]
    cov3D_precomp: torch.Tensor | None = None   # [P,6]

    @property
    def P(self) -> int:
        return int(self.means3D.shape[0])

    @property
    def M(self) -> int:
        return 0 if self.shs is None else int(self.shs.shape[1])

    @staticmethod
    def from_numpy(g, device="cuda") -> "GaussianTensors":
        t = lambda a: torch.from_numpy(a).to(device).contiguous()  # noqa: E731
        return GaussianTensors(means3D=t(g.means3D), opacities=t(g.opacities), shs=t(g.shs),
                               scales=t(g.scales), rotations=t(g.rotations))


@dataclasses.dataclass
class Camera:
    width: int
    height: int
    viewmatrix: torch.Tensor  # [4,4] (row-major Tcw^T)
    campos: torch.Tensor      # [3]
    background: torch.Tensor  # [3]

    @staticmethod
    def from_view(v, device="cuda", background=(0.0, 0.0, 0.0)) -> "Camera":
        return Camera(v.width, v.height, torch.from_numpy(v.viewmatrix).to(device).contiguous(),
                      torch.from_numpy(v.campos).to(device).contiguous(),
                      torch.tensor(background, dtype=torch.float32, device=device))


@dataclasses.dataclass
class Gradients:
    dL_dmeans2D: torch.Tensor
    dL_dcolors: torch.Tensor
    dL_dopacity: torch.Tensor
    dL_dmeans3D: torch.Tensor
    dL_dcov3D: torch.Tensor
    dL_dsh: torch.Tensor
    dL_dscales: torch.Tensor
    dL_drotations: torch.Tensor
    dL_dconic: torch.Tensor | None = None

    @staticmethod
    def empty(P: int, M: int, device, with_conic: bool = False) -> "Gradients":
        e = lambda *s: torch.empty(*s, dtype=torch.float32, device=device)  # noqa: E731
        return Gradients(e(P, 3), e(P, 3), e(P, 1), e(P, 3), e(P, 6), e(P, M, 3), e(P, 3), e(P, 4),
                         e(P, 4) if with_conic else None)


def _view_tensor(base: torch.Tensor, address: int, count: int, dtype) -> torch.Tensor:
    off = address - base.data_ptr()
    itemsize = torch.empty((), dtype=dtype).element_size()
    assert 0 <= off and off + count * itemsize <= base.numel(), "view outside its buffer"
    return base[off:off + count * itemsize].view(dtype)


class LonlatState:
    """State buffers for P Gaussians rendered at W x H with room for ``capacity`` instances.
    ``recompute_T`` selects transmittance checkpointing (OMNIGS_FLAG_RECOMPUTE_T): no per-pixel
    state is stored and the backward recomputes it."""

    def __init__(self, P: int, W: int, H: int, capacity: int, device="cuda", recompute_T: bool = False):
        self.P, self.W, self.H = P, W, H
        self.device = torch.device(device)
        self.flags = capi.FLAG_RECOMPUTE_T if recompute_T else 0
        u8 = dict(dtype=torch.uint8, device=self.device)
        self.geom = torch.empty(capi.geom_bytes(P), **u8)
        self.image = torch.empty(capi.image_bytes(W, H, self.flags), **u8)
        self.binning = torch.empty(capi.binning_bytes(capacity), **u8)

    @property
    def capacity(self) -> int:
        return capi.binning_capacity(self.binning.numel())

    def resize_capacity(self, capacity: int):
        self.binning = torch.empty(capi.binning_bytes(capacity), dtype=torch.uint8, device=self.device)

    def _fwd_args(self, g: GaussianTensors, cam: Camera, out_color, radii, D, scale_modifier):
        a = capi.ForwardArgs()
        a.P, a.D, a.M, a.W, a.H = g.P, D, g.M, cam.width, cam.height
        a.background = capi.ptr(cam.background)
        a.means3D = capi.ptr(g.means3D)
        a.shs = capi.ptr(g.shs)
        a.colors_precomp = capi.ptr(g.colors_precomp)
        a.opacities = capi.ptr(g.opacities)
        a.scales = capi.ptr(g.scales)
        a.scale_modifier = scale_modifier
        a.rotations = capi.ptr(g.rotations)
        a.cov3D_precomp = capi.ptr(g.cov3D_precomp)
        a.viewmatrix = capi.ptr(cam.viewmatrix)
        a.campos = capi.ptr(cam.campos)
        a.out_color = capi.ptr(out_color)
        a.radii = capi.ptr(radii)
        a.flags = self.flags
        return a

    def forward(self, g: GaussianTensors, cam: Camera, out_color: torch.Tensor, radii: torch.Tensor,
                D: int = 3, scale_modifier: float = 1.0, stream=None):
        """Asynchronous forward on ``stream`` (default: current stream)."""
        assert (cam.width, cam.height) == (self.W, self.H) and g.P == self.P
        a = self._fwd_args(g, cam, out_color, radii, D, scale_modifier)
        rc = capi.lib().omnigs_lonlat_forward(
            ctypes.byref(a), self.geom.data_ptr(), self.geom.numel(), self.binning.data_ptr(),
            self.binning.numel(), self.image.data_ptr(), self.image.numel(),
            capi.stream_handle(stream))
        capi.check(rc, "omnigs_lonlat_forward")

    def forward_early_status(self, g: GaussianTensors, cam: Camera, out_color: torch.Tensor,
                             radii: torch.Tensor, D: int = 3, scale_modifier: float = 1.0,
                             stream=None) -> tuple[int, int]:
        """Forward that returns (num_rendered, status bits) once the binning has run; the blend
        is still executing on ``stream`` when it returns."""
        assert (cam.width, cam.height) == (self.W, self.H) and g.P == self.P
        a = self._fwd_args(g, cam, out_color, radii, D, scale_modifier)
        n = ctypes.c_int(0)
        st = ctypes.c_uint32(0)
        rc = capi.lib().omnigs_lonlat_forward_early_status(
            ctypes.byref(a), self.geom.data_ptr(), self.geom.numel(), self.binning.data_ptr(),
            self.binning.numel(), self.image.data_ptr(), self.image.numel(), ctypes.byref(n),
            ctypes.byref(st), capi.stream_handle(stream))
        capi.check(rc, "omnigs_lonlat_forward_early_status")
        return int(n.value), int(st.value)

    def render(self, g: GaussianTensors, cam: Camera, out_color, radii, D=3, scale_modifier=1.0,
               stream=None):
        """Re-run binning + blend from the current geometry buffer (after a capacity resize)."""
        a = self._fwd_args(g, cam, out_color, radii, D, scale_modifier)
        rc = capi.lib().omnigs_lonlat_render(
            ctypes.byref(a), self.geom.data_ptr(), self.geom.numel(), self.binning.data_ptr(),
            self.binning.numel(), self.image.data_ptr(), self.image.numel(),
            capi.stream_handle(stream))
        capi.check(rc, "omnigs_lonlat_render")

    def status(self, stream=None) -> tuple[int, int]:
        """(num_rendered, status bits); synchronises the stream."""
        n = ctypes.c_int(0)
        st = ctypes.c_uint32(0)
        rc = capi.lib().omnigs_lonlat_read_status(self.geom.data_ptr(), ctypes.byref(n),
                                                  ctypes.byref(st), capi.stream_handle(stream))
        capi.check(rc, "omnigs_lonlat_read_status")
        return int(n.value), int(st.value)

    def backward(self, g: GaussianTensors, cam: Camera, radii: torch.Tensor, dL_dout: torch.Tensor,
                 grads: Gradients, D: int = 3, scale_modifier: float = 1.0, R: int = -1,
                 stream=None):
        a = capi.BackwardArgs()
        a.P, a.D, a.M, a.W, a.H, a.R = g.P, D, g.M, cam.width, cam.height, R
        a.flags = self.flags
        a.background = capi.ptr(cam.background)
        a.means3D = capi.ptr(g.means3D)
        a.shs = capi.ptr(g.shs)
        a.colors_precomp = capi.ptr(g.colors_precomp)
        a.scales = capi.ptr(g.scales)
        a.scale_modifier = scale_modifier
        a.rotations = capi.ptr(g.rotations)
        a.cov3D_precomp = capi.ptr(g.cov3D_precomp)
        a.viewmatrix = capi.ptr(cam.viewmatrix)
        a.campos = capi.ptr(cam.campos)
        a.radii = capi.ptr(radii)
        a.dL_dout_color = capi.ptr(dL_dout)
        for f in ("dL_dmeans2D", "dL_dcolors", "dL_dopacity", "dL_dmeans3D", "dL_dcov3D", "dL_dsh",
                  "dL_dscales", "dL_drotations", "dL_dconic"):
            setattr(a, f, capi.ptr(getattr(grads, f)))
        rc = capi.lib().omnigs_lonlat_backward(
            ctypes.byref(a), self.geom.data_ptr(), self.geom.numel(), self.binning.data_ptr(),
            self.binning.numel(), self.image.data_ptr(), self.image.numel(),
            capi.stream_handle(stream))
        capi.check(rc, "omnigs_lonlat_backward")

    # ---- inspection views (device tensors aliasing the state buffers) ----
    def geom_view(self) -> dict:
        v = capi.GeomView()
        capi.check(capi.lib().omnigs_lonlat_geom_view(self.geom.data_ptr(), self.P, ctypes.byref(v)),
                   "geom_view")
        P = self.P
        splat = _view_tensor(self.geom, v.splat, 8 * P, torch.float32).view(P, 8)
        color = _view_tensor(self.geom, v.color, 4 * P, torch.float32).view(P, 4)
        return dict(means2D=splat[:, 0:2], conic_opacity=torch.cat([splat[:, 2:5], splat[:, 5:6]], 1),
                    cull=splat[:, 6:8], rgb=color[:, :3],
                    clamp_bits=color[:, 3].view(torch.int32),
                    depths=_view_tensor(self.geom, v.depth, P, torch.float32),
                    tiles_touched=_view_tensor(self.geom, v.tiles_touched, P, torch.int32),
                    depth_order=_view_tensor(self.geom, v.depth_order, P, torch.int32))

    def binning_view(self, num_rendered: int) -> dict:
        """Sorted tile ids and point list; ``keys`` rebuilds the reference's 64-bit
        ``tile << 32 | depth_bits`` keys from them."""
        v = capi.BinningView()
        capi.check(capi.lib().omnigs_lonlat_binning_view(self.binning.data_ptr(), self.binning.numel(),
                                                         self.W, self.H, ctypes.byref(v)),
                   "binning_view")
        tiles = _view_tensor(self.binning, v.tile_ids, num_rendered, torch.int32)
        point_list = _view_tensor(self.binning, v.point_list, num_rendered, torch.int32)
        depth_bits = self.geom_view()["depths"].view(torch.int32)[point_list.long()].to(torch.int64)
        keys = (tiles.to(torch.int64) << 32) | (depth_bits & 0xFFFFFFFF)
        return dict(tile_ids=tiles, point_list=point_list, keys=keys)

    def image_view(self) -> dict:
        assert self.flags == 0, "no per-pixel state is stored with recompute_T"
        v = capi.ImageView()
        capi.check(capi.lib().omnigs_lonlat_image_view(self.image.data_ptr(), self.W, self.H,
                                                       ctypes.byref(v)), "image_view")
        N = self.W * self.H
        tiles = ((self.W + 15) // 16) * ((self.H + 15) // 16)
        return dict(final_T=_view_tensor(self.image, v.final_T, N, torch.float32),
                    n_contrib=_view_tensor(self.image, v.n_contrib, N, torch.int32),
                    ranges=_view_tensor(self.image, v.ranges, 2 * tiles, torch.int32).view(tiles, 2))


def rasterize(g: GaussianTensors, cam: Camera, D: int = 3, scale_modifier: float = 1.0,
              capacity: int | None = None, state: LonlatState | None = None, recompute_T: bool = False):
    """One forward pass with exact sizing; returns (image, radii, num_rendered, state)."""
    dev = g.means3D.device
    if state is None:
        state = LonlatState(g.P, cam.width, cam.height, capacity or max(1024, 4 * g.P), dev,
                            recompute_T=recompute_T)
    out = torch.empty(3, cam.height, cam.width, dtype=torch.float32, device=dev)
    radii = torch.empty(g.P, dtype=torch.int32, device=dev)
    state.forward(g, cam, out, radii, D, scale_modifier)
    n, st = state.status()
    if st & capi.STATUS_CAPACITY:
        state.resize_capacity(n)
        state.render(g, cam, out, radii, D, scale_modifier)
        n, st = state.status()
    if st:
        raise capi.OmnigsError(f"device status bits {st}")
    return out, radii, n, state
