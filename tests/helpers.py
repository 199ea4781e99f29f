"""Shared helpers of the GPU parity tests: run the CUDA path through the C ABI and feed the
oracle, stage by stage, with the CUDA path's own intermediate arrays."""
from __future__ import annotations

import numpy as np
import torch

import oracle
from omnigs_b200 import lonlat, scenes


def to_np(t):
    return t.detach().cpu().numpy()


def run_cuda(g: lonlat.GaussianTensors, cam: lonlat.Camera, dpix: torch.Tensor | None = None,
             D: int = 3, scale_modifier: float = 1.0, capacity: int | None = None):
    """Forward (+ backward if dpix) through the C ABI; returns dict of device tensors."""
    img, radii, n, state = lonlat.rasterize(g, cam, D=D, scale_modifier=scale_modifier,
                                            capacity=capacity)
    out = dict(image=img, radii=radii, num_rendered=n, state=state)
    gv = state.geom_view()
    out.update({k: v.clone() for k, v in gv.items()})
    out.update({k: v.clone() for k, v in state.binning_view(n).items()})
    out.update({k: v.clone() for k, v in state.image_view().items()})
    if dpix is not None:
        grads = lonlat.Gradients.empty(g.P, g.M, g.means3D.device, with_conic=True)
        state.backward(g, cam, radii, dpix, grads, D=D, scale_modifier=scale_modifier, R=n)
        torch.cuda.synchronize()
        out["grads"] = grads
    return out


def oracle_stagewise(cu: dict, g_np: scenes.Gaussians, view: scenes.View, dpix_np, bg,
                     D=3, scale_modifier=1.0):
    """Oracle stages fed with the CUDA path's float intermediates."""
    W, H, P = view.width, view.height, g_np.P
    radii = to_np(cu["radii"])
    means2D = to_np(cu["means2D"]).astype(np.float32)
    depths = to_np(cu["depths"]).astype(np.float32)
    tt = to_np(cu["tiles_touched"]).view(np.uint32)
    b = oracle.binning(W, H, radii, means2D, depths, tt, f32=True)
    point_list = to_np(cu["point_list"]).astype(np.uint32)
    ranges = to_np(cu["ranges"]).astype(np.uint32)
    con = to_np(cu["conic_opacity"]).astype(np.float64)
    rgb = to_np(cu["rgb"]).astype(np.float64)
    fw = oracle.render_forward(W, H, ranges, point_list, means2D, con, rgb, bg)
    out = dict(binning=b, forward=fw)
    if dpix_np is not None:
        final_T = to_np(cu["final_T"]).astype(np.float64)
        n_contrib = to_np(cu["n_contrib"]).astype(np.uint32)
        bw = oracle.render_backward(P, W, H, ranges, point_list, means2D, con, rgb, bg, final_T,
                                    n_contrib, dpix_np)
        clamped = np.stack([(to_np(cu["clamp_bits"]) >> k) & 1 for k in range(3)], 1).astype(np.uint8)
        pb = oracle.preprocess_backward(g_np.means3D, radii, g_np.shs, clamped, g_np.scales,
                                        g_np.rotations, view.viewmatrix, view.campos, W, H,
                                        bw["dL_dmean2D"], bw["dL_dconic"], bw["dL_dcolor"], D=D,
                                        scale_modifier=scale_modifier)
        out.update(render_backward=bw, preprocess_backward=pb)
    return out


def normwise_rel(a, b) -> float:
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    den = np.abs(b).max() if b.size else 0.0
    if den == 0.0:
        return float(np.abs(a).max()) if a.size else 0.0
    return float(np.abs(a - b).max() / den)
