"""Seeded synthetic equirectangular scenes.

The reference (liquorleaf/OmniGS) is evaluated on real 360Roam / EgoNeRF captures, which are not
available here.  These generators produce seeded stand-ins with the shapes, sizes and value
distributions of the benchmark configurations:

* means: uniform in volume inside a spherical shell of radius 1-5 m around the origin,
* scales: exp(N(ln 0.02, 0.5)) per axis (already activated, like ``getScalingActivation``),
* rotations: normalised N(0, 1) quaternions in (r, x, y, z) order,
* opacities: sigmoid(N(0, 1)) (already activated),
* SH: degree 3, 16 x 3 coefficients, DC ~ N(0, 0.5), higher bands ~ N(0, 0.05).

Views follow the reference's camera conventions (``src/gaussian_keyframe.cpp:132-162``): the
rasterizer receives ``world_view_transform = Tcw^T`` as a row-major 4x4 tensor, i.e. Tcw stored
column-major, and ``camera_center`` = the camera position in world coordinates.  The lonlat
projection (``cuda_rasterizer/auxiliary.h:236-248``) looks along +z with +x to the right and +y
down, so longitude = atan2(x, z) and latitude = asin(y / r).

Everything is float32 and generated with numpy's PCG64, so a seed gives the same scene on any
machine.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

SH_COEFFS = 16  # degree 3


@dataclasses.dataclass
class Gaussians:
    means3D: np.ndarray    # [P, 3] float32
    scales: np.ndarray     # [P, 3] float32 (activated)
    rotations: np.ndarray  # [P, 4] float32 (normalised, r x y z)
    opacities: np.ndarray  # [P, 1] float32 (activated)
    shs: np.ndarray        # [P, 16, 3] float32

    @property
    def P(self) -> int:
        return int(self.means3D.shape[0])

    def subset(self, idx) -> "Gaussians":
        return Gaussians(*(np.ascontiguousarray(getattr(self, f.name)[idx])
                           for f in dataclasses.fields(self)))


@dataclasses.dataclass
class View:
    width: int
    height: int
    viewmatrix: np.ndarray  # [4, 4] float32, row-major storage of Tcw^T
    campos: np.ndarray      # [3] float32


def _unit_vectors(rng: np.random.Generator, n: int) -> np.ndarray:
    v = rng.standard_normal((n, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    return v


def make_gaussians(P: int, seed: int = 0, pole_fraction: float = 0.0,
                   pole_min_lat_deg: float = 80.0, seam_fraction: float = 0.0,
                   seam_width_deg: float = 5.0) -> Gaussians:
    """Scene of ``P`` Gaussians around a camera at the origin.

    ``pole_fraction`` of the means are placed at |latitude| > ``pole_min_lat_deg`` (in the
    identity camera frame, latitude = asin(y / r)); the pole-heavy precision workload uses 0.3.
    ``seam_fraction`` of the means are placed within ``seam_width_deg`` of longitude +-180 deg
    (the equirect image's left/right edge) at |latitude| < 60 deg, so their splats straddle the
    seam.  Both default to 0, which leaves the generator's draws unchanged.
    """
    rng = np.random.Generator(np.random.PCG64(seed))
    r = np.cbrt(rng.random(P) * (125.0 - 1.0) + 1.0)
    dirs = _unit_vectors(rng, P)
    n_pole = int(round(P * pole_fraction))
    if n_pole > 0:
        # uniform on the two polar caps |lat| > pole_min_lat: sin(lat) uniform in [sin(min), 1]
        s0 = math.sin(math.radians(pole_min_lat_deg))
        sin_lat = rng.uniform(s0, 1.0, n_pole) * rng.choice([-1.0, 1.0], n_pole)
        lon = rng.uniform(-math.pi, math.pi, n_pole)
        cos_lat = np.sqrt(1.0 - sin_lat ** 2)
        pole_dirs = np.stack([cos_lat * np.sin(lon), sin_lat, cos_lat * np.cos(lon)], axis=1)
        sel = rng.permutation(P)[:n_pole]
        dirs[sel] = pole_dirs
    n_seam = int(round(P * seam_fraction))
    if n_seam > 0:
        lon = math.pi + np.radians(rng.uniform(-seam_width_deg, seam_width_deg, n_seam))
        lat = np.radians(rng.uniform(-60.0, 60.0, n_seam))
        seam_dirs = np.stack([np.cos(lat) * np.sin(lon), np.sin(lat), np.cos(lat) * np.cos(lon)], axis=1)
        dirs[rng.permutation(P)[:n_seam]] = seam_dirs
    means = (dirs * r[:, None]).astype(np.float32)
    scales = np.exp(rng.normal(math.log(0.02), 0.5, (P, 3))).astype(np.float32)
    q = rng.standard_normal((P, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    rotations = q.astype(np.float32)
    opacities = (1.0 / (1.0 + np.exp(-rng.standard_normal((P, 1))))).astype(np.float32)
    shs = np.empty((P, SH_COEFFS, 3), dtype=np.float32)
    shs[:, 0, :] = rng.normal(0.0, 0.5, (P, 3))
    shs[:, 1:, :] = rng.normal(0.0, 0.05, (P, SH_COEFFS - 1, 3))
    return Gaussians(means, scales, rotations, opacities, shs)


def rotation_yaw_pitch(yaw: float, pitch: float) -> np.ndarray:
    """Camera-to-world rotation: yaw about +y (down axis), then pitch about the camera x axis."""
    cy, sy = math.cos(yaw), math.sin(yaw)
    cp, sp = math.cos(pitch), math.sin(pitch)
    Ry = np.array([[cy, 0.0, sy], [0.0, 1.0, 0.0], [-sy, 0.0, cy]])
    Rx = np.array([[1.0, 0.0, 0.0], [0.0, cp, -sp], [0.0, sp, cp]])
    return Ry @ Rx


def make_view(width: int, height: int, position=(0.0, 0.0, 0.0), R_wc=None) -> View:
    """Equirectangular view at ``position`` with camera-to-world rotation ``R_wc``."""
    c = np.asarray(position, dtype=np.float64)
    R_wc = np.eye(3) if R_wc is None else np.asarray(R_wc, dtype=np.float64)
    R_cw = R_wc.T
    Tcw = np.eye(4)
    Tcw[:3, :3] = R_cw
    Tcw[:3, 3] = -R_cw @ c
    viewmatrix = np.ascontiguousarray(Tcw.T).astype(np.float32)
    campos = (np.linalg.inv(Tcw.astype(np.float32).astype(np.float64))[:3, 3]).astype(np.float32)
    return View(width, height, viewmatrix, campos)


def identity_view(width: int, height: int) -> View:
    return make_view(width, height)


def random_views(n: int, resolutions, seed: int = 1, cube: float = 2.0,
                 pitch_deg: float = 30.0) -> list[View]:
    """``n`` views with positions uniform in a ``cube``-metre cube centred at the origin,
    uniform yaw and pitch uniform in +-``pitch_deg``; resolutions drawn from ``resolutions``."""
    rng = np.random.Generator(np.random.PCG64(seed))
    views = []
    for _ in range(n):
        w, h = resolutions[int(rng.integers(len(resolutions)))]
        pos = rng.uniform(-cube / 2, cube / 2, 3)
        yaw = rng.uniform(-math.pi, math.pi)
        pitch = math.radians(rng.uniform(-pitch_deg, pitch_deg))
        views.append(make_view(w, h, pos, rotation_yaw_pitch(yaw, pitch)))
    return views


def upstream_grad(width: int, height: int, seed: int = 2) -> np.ndarray:
    """dL/dpixel ~ N(0, 1), layout [3, H, W] like the rendered image."""
    rng = np.random.Generator(np.random.PCG64(seed))
    return rng.standard_normal((3, height, width)).astype(np.float32)


# Benchmark workloads (sizes of the reference's headline configurations).
CONFIG_SMALL = dict(P=10_000, width=512, height=256)        # CPU-runnable case
CONFIG_PLAIN = dict(P=1_000_000, width=2048, height=1024)   # headline single-view case
BATCH_RESOLUTIONS = [(512, 256), (1024, 512), (2048, 1024), (3072, 1536)]
