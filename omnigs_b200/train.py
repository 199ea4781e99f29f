"""Training step around the rasterizer through the C ABI: L1 + D-SSIM loss, fused Adam.

``GaussianModelState`` holds the reference model's raw parameters (xyz, f_dc, f_rest, opacity
before the sigmoid, log scaling, unnormalised rotation; src/gaussian_model.cpp:54-77), their Adam
moments, the activated values the rasterizer reads, and the device-resident Adam hyper-parameters.
``BatchTrainStep`` is one training iteration over a batch of views: batched forward, per-view loss
and image gradient, batched backward, (across ranks: one gradient all-reduce,
``sharding.GradientReducer``), Adam step -- all asynchronous, so the whole step can be captured
once in a CUDA graph and replayed (``capture``).
"""
from __future__ import annotations

import ctypes
import math

import numpy as np
import torch

from . import batch, capi, ply, sharding
from .lonlat import GaussianTensors

# learning rates of the reference's lonlat configurations (cfg/lonlat/*.yaml: Optimization.*),
# in the parameter-group order of gaussian_model.cpp:534-541
DEFAULT_LR = dict(xyz=0.00016, f_dc=0.0025, f_rest=0.0025 / 20.0, opacity=0.05, scaling=0.005, rotation=0.001)
GROUPS = ("xyz", "f_dc", "f_rest", "opacity", "scaling", "rotation")


def l1_dssim_workspace(C: int, H: int, W: int, device="cuda") -> torch.Tensor:
    return torch.empty(capi.lib().omnigs_l1_dssim_workspace_bytes(C, H, W), dtype=torch.uint8, device=device)


def l1_dssim(image: torch.Tensor, gt: torch.Tensor, lambda_dssim: float = 0.2, rows: int | None = None,
             dL_dimage: torch.Tensor | None = None, loss: torch.Tensor | None = None,
             workspace: torch.Tensor | None = None, stream=None):
    """(1 - lambda) L1 + lambda (1 - SSIM) of [C,H,W] images over rows [0, rows); returns
    (loss [3] = (loss, l1, ssim) on the device, dL/dimage)."""
    C, H, W = image.shape
    rows = H if rows is None else rows
    dL_dimage = torch.empty_like(image) if dL_dimage is None else dL_dimage
    loss = torch.empty(3, dtype=torch.float32, device=image.device) if loss is None else loss
    workspace = l1_dssim_workspace(C, H, W, image.device) if workspace is None else workspace
    rc = capi.lib().omnigs_l1_dssim(capi.ptr(image), capi.ptr(gt), C, H, W, rows, lambda_dssim,
                                    capi.ptr(dL_dimage), capi.ptr(loss), workspace.data_ptr(),
                                    workspace.numel(), capi.stream_handle(stream))
    capi.check(rc, "omnigs_l1_dssim")
    return loss, dL_dimage


class GaussianModelState:
    """Raw parameters + Adam moments + activated values of P Gaussians with M SH coefficients."""

    def __init__(self, xyz, features_dc, features_rest, opacity, scaling, rotation, sh_bf16: bool = False,
                 lr: dict | None = None, betas=(0.9, 0.999), eps: float = 1e-15):
        dev = xyz.device
        self.P = int(xyz.shape[0])
        self.M = 1 + int(features_rest.shape[1])
        c = lambda t: t.detach().to(torch.float32).contiguous().clone()  # noqa: E731
        self.xyz, self.features_dc, self.features_rest = c(xyz), c(features_dc), c(features_rest)
        self.opacity, self.scaling, self.rotation = c(opacity), c(scaling), c(rotation)
        self.params = [self.xyz, self.features_dc, self.features_rest, self.opacity, self.scaling, self.rotation]
        self.m = [torch.zeros_like(t) for t in self.params]
        self.v = [torch.zeros_like(t) for t in self.params]
        self.sh_bf16 = sh_bf16
        self.shs = torch.empty(self.P, self.M, 3, dtype=torch.bfloat16 if sh_bf16 else torch.float32, device=dev)
        self.opacities = torch.empty(self.P, 1, device=dev)
        self.scales = torch.empty(self.P, 3, device=dev)
        self.rotations = torch.empty(self.P, 4, device=dev)
        self.lr = dict(DEFAULT_LR if lr is None else lr)
        self.betas, self.eps = betas, eps
        # OmnigsAdamHyper image on the device: 9 doubles (lr[6], beta1, beta2, eps) + the int64 step
        # count, which every adam_step increments on the device (so a captured graph advances it)
        self.hyper = torch.zeros(10, dtype=torch.int64, device=dev)
        self._write_hyper()
        self._prm, self._st, self._act = self._structs()
        rc = capi.lib().omnigs_activate(ctypes.byref(self._prm), ctypes.byref(self._act), capi.stream_handle())
        capi.check(rc, "omnigs_activate")

    @staticmethod
    def from_activated(g, device="cuda", sh_bf16: bool = False, **kw) -> "GaussianModelState":
        """From a scene in activated form (scenes.Gaussians): inverse activations."""
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(device)  # noqa: E731
        op = np.clip(g.opacities.astype(np.float64), 1e-6, 1 - 1e-6)
        return GaussianModelState(t(g.means3D), t(g.shs[:, :1]), t(g.shs[:, 1:]),
                                  t(np.log(op / (1 - op)).astype(np.float32)),
                                  t(np.log(g.scales).astype(np.float32)), t(g.rotations), sh_bf16=sh_bf16, **kw)

    @staticmethod
    def from_ply(path: str, device="cuda", sh_bf16: bool = False, **kw) -> "GaussianModelState":
        """From a scene saved by the reference's savePly (raw parameters; gaussian_model.cpp:860)."""
        g = ply.read_ply(path)
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(device)  # noqa: E731
        return GaussianModelState(t(g.xyz), t(g.features_dc), t(g.features_rest), t(g.opacity), t(g.scaling),
                                  t(g.rotation), sh_bf16=sh_bf16, **kw)

    def save_ply(self, path: str) -> None:
        """Writes the raw parameters in the reference's PLY layout (gaussian_model.cpp:978)."""
        n = lambda x: x.detach().cpu().numpy()  # noqa: E731
        ply.write_ply(path, ply.PlyGaussians(xyz=n(self.xyz), features_dc=n(self.features_dc),
                                             features_rest=n(self.features_rest), opacity=n(self.opacity),
                                             scaling=n(self.scaling), rotation=n(self.rotation)))

    def _structs(self):
        prm = capi.GaussianParams()
        prm.P, prm.M = self.P, self.M
        for f, t in zip(("xyz", "features_dc", "features_rest", "opacity", "scaling", "rotation"), self.params):
            setattr(prm, f, t.data_ptr() if t.numel() else None)
        st = capi.AdamState()
        for name, m, v in zip(("xyz", "dc", "rest", "opacity", "scaling", "rotation"), self.m, self.v):
            setattr(st, "m_" + name, m.data_ptr() if m.numel() else None)
            setattr(st, "v_" + name, v.data_ptr() if v.numel() else None)
        act = capi.Activated()
        act.means3D = self.xyz.data_ptr()
        act.shs = self.shs.data_ptr()
        act.shs_bf16 = 1 if self.sh_bf16 else 0
        act.opacities = self.opacities.data_ptr()
        act.scales = self.scales.data_ptr()
        act.rotations = self.rotations.data_ptr()
        return prm, st, act

    def tensors(self) -> GaussianTensors:
        """The activated values as rasterizer inputs."""
        return GaussianTensors(means3D=self.xyz, opacities=self.opacities, shs=self.shs, scales=self.scales,
                               rotations=self.rotations)

    def _write_hyper(self):
        f = torch.tensor([self.lr[k] for k in GROUPS] + [self.betas[0], self.betas[1], self.eps],
                         dtype=torch.float64)
        self.hyper[:9].copy_(f.view(torch.int64))  # from pageable memory: consumed before returning

    def set_lr(self, **lr):
        """Changes learning rates (by group name) for the following steps."""
        self.lr.update(lr)
        self._write_hyper()

    @property
    def step_count(self) -> int:
        return int(self.hyper[9].item())

    def adam_step(self, dL_dmeans3D, dL_dsh, dL_dopacity, dL_dscales, dL_drotations, stream=None):
        """One fused Adam step: advances the device step count, then updates every group."""
        s = stream if stream is not None else torch.cuda.current_stream()
        with torch.cuda.stream(s):
            self.hyper[9:].add_(1)
        rc = capi.lib().omnigs_adam_step(
            ctypes.byref(self._prm), ctypes.byref(self._st), ctypes.byref(self._act), capi.ptr(dL_dmeans3D),
            capi.ptr(dL_dsh), capi.ptr(dL_dopacity), capi.ptr(dL_dscales), capi.ptr(dL_drotations),
            self.hyper.data_ptr(), capi.stream_handle(stream))
        capi.check(rc, "omnigs_adam_step")


class BatchTrainStep:
    """One training iteration over ``len(views)`` target views: batched forward, per-view
    L1 + D-SSIM loss and image gradient, batched backward (with densification statistics), fused
    Adam.  ``losses`` [V,3] holds each view's (loss, l1, ssim) on the device after a step."""

    def __init__(self, model: GaussianModelState, cams: batch.BatchCameras, targets, capacity: int,
                 lambda_dssim: float = 0.2, D: int = 3, fp64_poles: bool = False, process_group=None,
                 data_parallel: bool = False):
        dev = model.xyz.device
        self.model, self.cams, self.targets = model, cams, targets
        self.lambda_dssim, self.D, self.fp64_poles = lambda_dssim, D, fp64_poles
        self.state = batch.BatchState(model.P, cams.sizes, capacity, dev)
        self.images = [torch.empty(3, h, w, device=dev) for w, h in cams.sizes]
        self.dimages = [torch.empty(3, h, w, device=dev) for w, h in cams.sizes]
        self.losses = torch.empty(cams.V, 3, device=dev)
        W = max(w for w, _ in cams.sizes)
        H = max(h for _, h in cams.sizes)
        self.workspace = l1_dssim_workspace(3, H, W, dev)
        # data parallel (one process per GPU, views sharded with sharding.assign_views): the step's
        # gradients and densification statistics are combined across ranks before Adam
        self.reducer = sharding.GradientReducer(model.P, model.M, dev, stats=True, group=process_group) \
            if data_parallel else None
        self.grads = self.reducer.grads if self.reducer else batch.BatchGradients.empty(model.P, model.M, dev,
                                                                                        stats=True)
        self.graph = None

    def run(self, stream=None):
        """Enqueues one step on ``stream`` (no host synchronisation)."""
        g = self.model.tensors()
        self.state.forward(g, self.cams, self.images, D=self.D, fp64_poles=self.fp64_poles, stream=stream)
        for v in range(self.cams.V):
            l1_dssim(self.images[v], self.targets[v], self.lambda_dssim, dL_dimage=self.dimages[v],
                     loss=self.losses[v], workspace=self.workspace, stream=stream)
        self.state.backward(g, self.cams, self.dimages, self.grads, D=self.D, fp64_poles=self.fp64_poles,
                            stream=stream)
        if self.reducer is not None:
            self.reducer.reduce()
        gr = self.grads
        self.model.adam_step(gr.dL_dmeans3D, gr.dL_dsh, gr.dL_dopacity, gr.dL_dscales, gr.dL_drotations,
                             stream=stream)

    def capture(self):
        """Captures one step in a CUDA graph (after at least one eager step)."""
        self.graph = torch.cuda.CUDAGraph()
        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.graph(self.graph, stream=s):
            self.run()
        torch.cuda.current_stream().wait_stream(s)

    def replay(self):
        self.graph.replay()

    def status(self):
        return self.state.status()


def exponential_lr(step: int, lr_init: float, lr_final: float, delay_mult: float = 1.0, max_steps: int = 30000,
                   delay_steps: int = 0) -> float:
    """The reference's position learning-rate schedule (GaussianModel::exponLrFunc,
    src/gaussian_model.cpp:1140-1160): log-linear from lr_init to lr_final over max_steps."""
    if step < 0 or (lr_init == 0.0 and lr_final == 0.0):
        return 0.0
    if delay_steps > 0:
        delay_rate = delay_mult + (1 - delay_mult) * math.sin(0.5 * math.pi * min(max(step / delay_steps, 0.0), 1.0))
    else:
        delay_rate = 1.0
    t = min(max(step / max_steps, 0.0), 1.0)
    return delay_rate * math.exp(math.log(lr_init) * (1 - t) + math.log(lr_final) * t)
