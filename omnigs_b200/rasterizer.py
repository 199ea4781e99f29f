"""Python face of the LibTorch autograd layer, mirroring OmniGS include/gaussian_rasterizer.h.

``GaussianRasterizer(settings)(means3D, means2D, opacities, shs=..., scales=..., rotations=...)``
returns ``(color [3,H,W], radii [P])``; ``means2D`` is the zero "viewspace points" tensor whose
``.grad`` receives the screen-space gradient used for densification, as in
src/gaussian_renderer.cpp:184-191.  The autograd node is the C++ torch::autograd::Function.
"""
from __future__ import annotations

import dataclasses

import torch


@dataclasses.dataclass
class GaussianRasterizationSettings:
    image_height: int
    image_width: int
    tanfovx: float
    tanfovy: float
    bg: torch.Tensor
    scale_modifier: float
    viewmatrix: torch.Tensor
    projmatrix: torch.Tensor
    sh_degree: int
    campos: torch.Tensor
    prefiltered: bool = False
    camera_type: int = 3  # Camera::CameraModelType::LONLAT
    render_depth: bool = False


class GaussianRasterizer(torch.nn.Module):
    def __init__(self, raster_settings: GaussianRasterizationSettings):
        super().__init__()
        self.raster_settings = raster_settings

    def mark_visible(self, positions: torch.Tensor) -> torch.Tensor:
        from . import torch_ext
        s = self.raster_settings
        with torch.no_grad():
            return torch_ext().mark_visible(positions, s.viewmatrix, s.projmatrix, s.camera_type)

    def forward(self, means3D, means2D, opacities, shs=None, colors_precomp=None, scales=None,
                rotations=None, cov3D_precomp=None):
        from . import torch_ext
        if (shs is None) == (colors_precomp is None):
            raise RuntimeError("Please provide excatly one of either SHs or precomputed colors!")
        if ((scales is None or rotations is None) and cov3D_precomp is None) or \
                ((scales is not None or rotations is not None) and cov3D_precomp is not None):
            raise RuntimeError("Please provide exactly one of either scale/rotation pair or "
                               "precomputed 3D covariance!")
        empty = means3D.new_empty(0)
        s = self.raster_settings
        color, radii = torch_ext().rasterize(
            means3D, means2D, empty if shs is None else shs,
            empty if colors_precomp is None else colors_precomp, opacities,
            empty if scales is None else scales, empty if rotations is None else rotations,
            empty if cov3D_precomp is None else cov3D_precomp, s.image_height, s.image_width,
            s.tanfovx, s.tanfovy, s.bg, s.scale_modifier, s.viewmatrix, s.projmatrix, s.sh_degree,
            s.campos, s.prefiltered, s.camera_type)
        return color, radii
