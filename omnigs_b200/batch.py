"""Batched multi-view lonlat rasterization through the C ABI (``omnigs_batch_*``).

``BatchState`` owns the state of V equirect views (uneven sizes allowed) over one shared Gaussian
set: one launch per stage renders or back-propagates all views.  Per view the images equal the
single-view path's; the backward returns the parameter gradients summed over the views and
accumulates the trainer's densification statistics (per-view viewspace-gradient norms, visible-view
counts, maximum radii).  SH coefficients may be passed as bfloat16 (``shs.dtype ==
torch.bfloat16``); ``fp64_poles`` evaluates the 2D covariance of Gaussians beyond 85 degrees of
latitude in FP64; ``seam_wrap`` lets splats wrap across the longitude seam (off: the reference's
clamped tile rects).  Nothing here synchronises the host except ``status()``.
"""
from __future__ import annotations

import ctypes
import dataclasses

import numpy as np
import torch

from . import capi
from .lonlat import GaussianTensors, _view_tensor


@dataclasses.dataclass
class BatchCameras:
    """Per-view poses on the device: viewmatrices [V,4,4] (each the row-major Tcw^T of the
    single-view Camera), campos [V,3], backgrounds [V,3], and the host list of (W, H)."""
    sizes: list
    viewmatrices: torch.Tensor
    campos: torch.Tensor
    backgrounds: torch.Tensor

    @property
    def V(self) -> int:
        return len(self.sizes)

    @staticmethod
    def from_views(views, device="cuda", background=(0.0, 0.0, 0.0)) -> "BatchCameras":
        vm = np.stack([v.viewmatrix for v in views]).astype(np.float32)
        cp = np.stack([v.campos for v in views]).astype(np.float32)
        bg = np.tile(np.asarray(background, np.float32), (len(views), 1))
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(device)  # noqa: E731
        return BatchCameras([(v.width, v.height) for v in views], t(vm), t(cp), t(bg))


@dataclasses.dataclass
class BatchGradients:
    """Parameter gradients summed over the views, and densification statistics accumulated in
    place (``grad_accum`` += |dL/dmean2D.xy|, ``denom`` += 1 per visible view, ``max_radii`` =
    max with the radius)."""
    dL_dmeans3D: torch.Tensor
    dL_dsh: torch.Tensor | None
    dL_dopacity: torch.Tensor
    dL_dscales: torch.Tensor
    dL_drotations: torch.Tensor
    dL_dcolors: torch.Tensor | None = None
    dL_dcov3D: torch.Tensor | None = None
    grad_accum: torch.Tensor | None = None
    denom: torch.Tensor | None = None
    max_radii: torch.Tensor | None = None

    @staticmethod
    def empty(P: int, M: int, device, stats: bool = False) -> "BatchGradients":
        e = lambda *s: torch.empty(*s, dtype=torch.float32, device=device)  # noqa: E731
        z = lambda *s: torch.zeros(*s, dtype=torch.float32, device=device)  # noqa: E731
        return BatchGradients(e(P, 3), e(P, M, 3) if M else None, e(P, 1), e(P, 3), e(P, 4),
                              grad_accum=z(P, 1) if stats else None, denom=z(P, 1) if stats else None,
                              max_radii=z(P) if stats else None)


class BatchState:
    """State of ``len(sizes)`` views over P Gaussians with room for ``capacity`` instances in total."""

    def __init__(self, P: int, sizes, capacity: int, device="cuda"):
        self.P, self.sizes = P, [(int(w), int(h)) for w, h in sizes]
        self.V = len(self.sizes)
        self.device = torch.device(device)
        nbytes = capi.batch_state_bytes(P, self.sizes)
        if nbytes == 0:
            raise capi.OmnigsError("invalid batch: " + capi.lib().omnigs_last_error().decode())
        self.state = torch.empty(nbytes, dtype=torch.uint8, device=self.device)
        self.binning = torch.empty(capi.binning_bytes(capacity), dtype=torch.uint8, device=self.device)

    @property
    def capacity(self) -> int:
        return capi.binning_capacity(self.binning.numel())

    def resize_capacity(self, capacity: int):
        self.binning = torch.empty(capi.binning_bytes(capacity), dtype=torch.uint8, device=self.device)

    def _args(self, g: GaussianTensors, cams: BatchCameras, images, dL_dimages, D, scale_modifier,
              fp64_poles, seam_wrap=False):
        assert cams.sizes == self.sizes and g.P == self.P
        a = capi.BatchArgs()
        a.P, a.D, a.M, a.V = g.P, D, g.M, self.V
        bf16 = g.shs is not None and g.shs.dtype == torch.bfloat16
        assert g.shs is None or g.shs.dtype in (torch.float32, torch.bfloat16)
        a.sh_dtype = capi.SH_BF16 if bf16 else capi.SH_FP32
        a.fp64_poles = 1 if fp64_poles else 0
        a.seam_wrap = 1 if seam_wrap else 0
        a.means3D = capi.ptr(g.means3D)
        a.shs = capi.ptr(g.shs)
        a.colors_precomp = capi.ptr(g.colors_precomp)
        a.opacities = capi.ptr(g.opacities)
        a.scales = capi.ptr(g.scales)
        a.scale_modifier = scale_modifier
        a.rotations = capi.ptr(g.rotations)
        a.cov3D_precomp = capi.ptr(g.cov3D_precomp)
        a.viewmatrices = capi.ptr(cams.viewmatrices)
        a.campos = capi.ptr(cams.campos)
        a.backgrounds = capi.ptr(cams.backgrounds)
        views = (capi.BatchView * self.V)()
        for v, (w, h) in enumerate(self.sizes):
            views[v].W, views[v].H = w, h
            if images is not None:
                assert tuple(images[v].shape) == (3, h, w)
                views[v].out_color = capi.ptr(images[v])
            if dL_dimages is not None:
                assert tuple(dL_dimages[v].shape) == (3, h, w)
                views[v].dL_dout_color = capi.ptr(dL_dimages[v])
        a.views = views
        return a, views  # the caller keeps `views` alive for the call

    def forward(self, g: GaussianTensors, cams: BatchCameras, images, D: int = 3,
                scale_modifier: float = 1.0, fp64_poles: bool = False, stream=None, seam_wrap: bool = False):
        """Asynchronous forward of every view into ``images`` (list of [3,H,W] tensors)."""
        a, keep = self._args(g, cams, images, None, D, scale_modifier, fp64_poles, seam_wrap)
        rc = capi.lib().omnigs_batch_forward(ctypes.byref(a), self.state.data_ptr(), self.state.numel(),
                                             self.binning.data_ptr(), self.binning.numel(),
                                             capi.stream_handle(stream))
        capi.check(rc, "omnigs_batch_forward")

    def render(self, g: GaussianTensors, cams: BatchCameras, images, D: int = 3,
               scale_modifier: float = 1.0, fp64_poles: bool = False, stream=None, seam_wrap: bool = False):
        """Binning + blend again from the current preprocess (after a capacity resize)."""
        a, keep = self._args(g, cams, images, None, D, scale_modifier, fp64_poles, seam_wrap)
        rc = capi.lib().omnigs_batch_render(ctypes.byref(a), self.state.data_ptr(), self.state.numel(),
                                            self.binning.data_ptr(), self.binning.numel(),
                                            capi.stream_handle(stream))
        capi.check(rc, "omnigs_batch_render")

    def backward(self, g: GaussianTensors, cams: BatchCameras, dL_dimages, grads: BatchGradients,
                 D: int = 3, scale_modifier: float = 1.0, fp64_poles: bool = False, stream=None,
                 seam_wrap: bool = False):
        a, keep = self._args(g, cams, None, dL_dimages, D, scale_modifier, fp64_poles, seam_wrap)
        bg = capi.BatchGrads()
        for f, _ in capi.BatchGrads._fields_:
            setattr(bg, f, capi.ptr(getattr(grads, f)))
        rc = capi.lib().omnigs_batch_backward(ctypes.byref(a), ctypes.byref(bg), self.state.data_ptr(),
                                              self.state.numel(), self.binning.data_ptr(),
                                              self.binning.numel(), capi.stream_handle(stream))
        capi.check(rc, "omnigs_batch_backward")

    def autotune(self, g: GaussianTensors, cams: BatchCameras, images, dL_dimages, D: int = 3,
                 scale_modifier: float = 1.0, fp64_poles: bool = False, repeats: int = 3, stream=None) -> dict:
        """Chooses the blend staging batch (128 / 256 / 512 splats) per direction by timing the
        blends of this batch; needs a completed forward.  Synchronises; process-wide setting."""
        a, keep = self._args(g, cams, images, dL_dimages, D, scale_modifier, fp64_poles)
        r = capi.TuneResult()
        rc = capi.lib().omnigs_batch_autotune(ctypes.byref(a), self.state.data_ptr(), self.state.numel(),
                                              self.binning.data_ptr(), self.binning.numel(), repeats,
                                              ctypes.byref(r), capi.stream_handle(stream))
        capi.check(rc, "omnigs_batch_autotune")
        return {"candidates": list(r.candidates), "forward_ms": [round(x, 4) for x in r.forward_ms],
                "backward_ms": [round(x, 4) for x in r.backward_ms], "forward_batch": r.forward_batch,
                "backward_batch": r.backward_batch}

    def status(self, stream=None) -> tuple[int, list, int]:
        """(total instances, instances per view, status bits); synchronises the stream."""
        n = ctypes.c_int64(0)
        per = (ctypes.c_int64 * self.V)()
        st = ctypes.c_uint32(0)
        rc = capi.lib().omnigs_batch_read_status(self.state.data_ptr(), self.V, ctypes.byref(n), per,
                                                 ctypes.byref(st), capi.stream_handle(stream))
        capi.check(rc, "omnigs_batch_read_status")
        return int(n.value), [int(x) for x in per], int(st.value)

    def state_view(self) -> dict:
        """Device tensors aliasing the state: radii [V,P], splat [V,P,8], color [V,P,4], depth [V,P],
        and per view final_T / n_contrib [H*W] and ranges [tiles,2]."""
        sv = capi.BatchStateView()
        W = (ctypes.c_int * self.V)(*[w for w, _ in self.sizes])
        H = (ctypes.c_int * self.V)(*[h for _, h in self.sizes])
        capi.check(capi.lib().omnigs_batch_state_view(self.state.data_ptr(), self.P, self.V, W, H,
                                                      ctypes.byref(sv)), "omnigs_batch_state_view")
        P, V = self.P, self.V
        pixels = sum(w * h for w, h in self.sizes)
        tiles = sum(((w + 15) // 16) * ((h + 15) // 16) for w, h in self.sizes)
        final_T = _view_tensor(self.state, sv.final_T, pixels, torch.float32)
        n_contrib = _view_tensor(self.state, sv.n_contrib, pixels, torch.int32)
        ranges = _view_tensor(self.state, sv.ranges, 2 * tiles, torch.int32).view(tiles, 2)
        out = dict(radii=_view_tensor(self.state, sv.radii, V * P, torch.int32).view(V, P),
                   splat=_view_tensor(self.state, sv.splat, 8 * V * P, torch.float32).view(V, P, 8),
                   color=_view_tensor(self.state, sv.color, 4 * V * P, torch.float32).view(V, P, 4),
                   depth=_view_tensor(self.state, sv.depth, V * P, torch.float32).view(V, P),
                   final_T=[], n_contrib=[], ranges=[], tile_base=[], pixel_base=[])
        for v, (w, h) in enumerate(self.sizes):
            pb, tb, nt = sv.pixel_base[v], sv.tile_base[v], ((w + 15) // 16) * ((h + 15) // 16)
            out["final_T"].append(final_T[pb:pb + w * h])
            out["n_contrib"].append(n_contrib[pb:pb + w * h])
            out["ranges"].append(ranges[tb:tb + nt])
            out["tile_base"].append(int(tb))
            out["pixel_base"].append(int(pb))
        return out


    def binning_view(self, num_rendered: int) -> dict:
        """Sorted instance list of the last forward: global tile ids and record indices
        (view * P + Gaussian), device tensors aliasing the binning buffer."""
        bv = capi.BinningView()
        W = (ctypes.c_int * self.V)(*[w for w, _ in self.sizes])
        H = (ctypes.c_int * self.V)(*[h for _, h in self.sizes])
        capi.check(capi.lib().omnigs_batch_binning_view(self.binning.data_ptr(), self.binning.numel(), self.P,
                                                        self.V, W, H, ctypes.byref(bv)), "omnigs_batch_binning_view")
        return dict(tile_ids=_view_tensor(self.binning, bv.tile_ids, num_rendered, torch.int32),
                    point_list=_view_tensor(self.binning, bv.point_list, num_rendered, torch.int32))


def set_blend_batch(forward: int, backward: int):
    """Splats staged per shared-memory batch in the blend kernels (128, 256 or 512 each)."""
    capi.check(capi.lib().omnigs_set_blend_batch(forward, backward), "omnigs_set_blend_batch")


def get_blend_batch() -> tuple[int, int]:
    f, b = ctypes.c_int(0), ctypes.c_int(0)
    capi.lib().omnigs_get_blend_batch(ctypes.byref(f), ctypes.byref(b))
    return int(f.value), int(b.value)


def render_batch(g: GaussianTensors, cams: BatchCameras, D: int = 3, scale_modifier: float = 1.0,
                 fp64_poles: bool = False, capacity: int | None = None, state: BatchState | None = None,
                 seam_wrap: bool = False):
    """Forward of every view with exact capacity sizing; returns (images, num_rendered per view,
    state)."""
    dev = g.means3D.device
    if state is None:
        state = BatchState(g.P, cams.sizes, capacity or max(1024, 4 * g.P * cams.V), dev)
    images = [torch.empty(3, h, w, dtype=torch.float32, device=dev) for w, h in cams.sizes]
    state.forward(g, cams, images, D, scale_modifier, fp64_poles, seam_wrap=seam_wrap)
    n, per, st = state.status()
    if st & capi.STATUS_CAPACITY:
        state.resize_capacity(n)
        state.render(g, cams, images, D, scale_modifier, fp64_poles, seam_wrap=seam_wrap)
        n, per, st = state.status()
    if st:
        raise capi.OmnigsError(f"device status bits {st}")
    return images, per, state
