"""TEST INFRASTRUCTURE ONLY: ctypes wrapper of the FP64 oracle (oracle/oracle.cpp).

Only the test suite, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg use this
module, and only as the checker / CPU baseline.  The product (``omnigs_b200``) never imports it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "lib", "liboracle.so")
_lib = None

P_f32 = ctypes.POINTER(ctypes.c_float)
P_f64 = ctypes.POINTER(ctypes.c_double)
P_i32 = ctypes.POINTER(ctypes.c_int32)
P_u32 = ctypes.POINTER(ctypes.c_uint32)
P_u64 = ctypes.POINTER(ctypes.c_uint64)
P_u8 = ctypes.POINTER(ctypes.c_uint8)
TILE = 16


def build() -> str:
    """Compile the oracle with its Makefile (g++ only) and return the library path."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        L.oracle_higher_msb.restype = ctypes.c_uint32
        L.oracle_num_rendered.restype = ctypes.c_int64
        _lib = L
    return _lib


def _p(a: np.ndarray | None, ptype):
    if a is None:
        return ctypes.cast(None, ptype)
    assert a.flags["C_CONTIGUOUS"], "oracle arrays must be C-contiguous"
    return a.ctypes.data_as(ptype)


def _f32(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float32)


def default_threads() -> int:
    return max(1, os.cpu_count() or 1)


def higher_msb(n: int) -> int:
    return int(lib().oracle_higher_msb(ctypes.c_uint32(n)))


def preprocess(means3D, scales, rotations, opacities, shs, viewmatrix, campos, W, H, D=3,
               scale_modifier=1.0, colors_precomp=None, cov3D_precomp=None, nthreads=None,
               seam_wrap=False):
    """FP64 forward preprocess.  Returns a dict of numpy arrays (doubles for float outputs).
    ``seam_wrap`` counts tiles_touched over the seam-wrapping mode's cyclic tile rects."""
    means3D, scales, rotations, opacities = map(_f32, (means3D, scales, rotations, opacities))
    shs, colors_precomp, cov3D_precomp = map(_f32, (shs, colors_precomp, cov3D_precomp))
    viewmatrix, campos = _f32(viewmatrix), _f32(campos)
    P = means3D.shape[0]
    M = 0 if shs is None else shs.shape[1]
    out = dict(radii=np.zeros(P, np.int32), tiles_touched=np.zeros(P, np.uint32),
               means2D=np.zeros((P, 2)), depths=np.zeros(P), conic_opacity=np.zeros((P, 4)),
               rgb=np.zeros((P, 3)), clamped=np.zeros((P, 3), np.uint8), cov3D=np.zeros((P, 6)))
    lib().oracle_preprocess_seam(
        P, D, M, W, H, _p(means3D, P_f32), _p(scales, P_f32), ctypes.c_float(scale_modifier),
        _p(rotations, P_f32), _p(opacities, P_f32), _p(shs, P_f32), _p(colors_precomp, P_f32),
        _p(cov3D_precomp, P_f32), _p(viewmatrix, P_f32), _p(campos, P_f32),
        _p(out["radii"], P_i32), _p(out["tiles_touched"], P_u32), _p(out["means2D"], P_f64),
        _p(out["depths"], P_f64), _p(out["conic_opacity"], P_f64), _p(out["rgb"], P_f64),
        _p(out["clamped"], P_u8), _p(out["cov3D"], P_f64), 1 if seam_wrap else 0,
        nthreads or default_threads())
    return out


def binning(W, H, radii, means2D, depths, tiles_touched, f32: bool, seam_wrap: bool = False):
    """Duplicate + stable sort + tile ranges.  ``f32=True`` evaluates the tile rects in float
    arithmetic from float32 means2D/depths (bit-exact target for the GPU); ``f32=False`` uses
    doubles (the pure FP64 pipeline).  ``seam_wrap`` uses the seam-wrapping mode's cyclic rects
    with columns taken modulo the grid width.  ``tiles_touched=None`` (float rects only) derives the
    per-Gaussian tile counts from the rects."""
    radii = np.ascontiguousarray(radii, np.int32)
    P = radii.shape[0]
    if tiles_touched is None:  # from the float rects themselves
        assert f32, "tiles_touched is derived from float rects"
        tiles_touched = np.zeros(P, np.uint32)
        m2f = np.ascontiguousarray(means2D, np.float32)
        lib().oracle_tiles_touched_f32(P, W, H, _p(radii, P_i32), _p(m2f, P_f32), 1 if seam_wrap else 0,
                                       _p(tiles_touched, P_u32))
    tiles_touched = np.ascontiguousarray(tiles_touched, np.uint32)
    R = int(lib().oracle_num_rendered(P, _p(tiles_touched, P_u32)))
    gx, gy = (W + TILE - 1) // TILE, (H + TILE - 1) // TILE
    keys = np.zeros(R, np.uint64)
    vals = np.zeros(R, np.uint32)
    ranges = np.zeros((gx * gy, 2), np.uint32)
    if f32:
        m2 = np.ascontiguousarray(means2D, np.float32)
        d = np.ascontiguousarray(depths, np.float32)
        lib().oracle_binning_f32_seam(P, W, H, _p(radii, P_i32), _p(m2, P_f32), _p(d, P_f32),
                                      _p(tiles_touched, P_u32), _p(keys, P_u64), _p(vals, P_u32),
                                      _p(ranges, P_u32), 1 if seam_wrap else 0)
    else:
        m2 = np.ascontiguousarray(means2D, np.float64)
        d = np.ascontiguousarray(depths, np.float64)
        lib().oracle_binning_f64_seam(P, W, H, _p(radii, P_i32), _p(m2, P_f64), _p(d, P_f64),
                                      _p(tiles_touched, P_u32), _p(keys, P_u64), _p(vals, P_u32),
                                      _p(ranges, P_u32), 1 if seam_wrap else 0)
    return dict(num_rendered=R, keys=keys, point_list=vals, ranges=ranges)


def binning_rows(W, H, radii, means2D, depths, row_lo, row_hi):
    """FP64 binning restricted to tile rows [row_lo, row_hi): keys, point list and ranges of those
    rows as the full FP64 binning has them; every other tile's range stays empty."""
    radii = np.ascontiguousarray(radii, np.int32)
    m2 = np.ascontiguousarray(means2D, np.float64)
    d = np.ascontiguousarray(depths, np.float64)
    P = radii.shape[0]
    counts = np.zeros(P, np.uint32)
    lib().oracle_tiles_in_rows_f64(P, W, H, _p(radii, P_i32), _p(m2, P_f64), row_lo, row_hi, _p(counts, P_u32))
    R = int(counts.sum(dtype=np.int64))
    gx, gy = (W + TILE - 1) // TILE, (H + TILE - 1) // TILE
    keys = np.zeros(R, np.uint64)
    vals = np.zeros(R, np.uint32)
    ranges = np.zeros((gx * gy, 2), np.uint32)
    lib().oracle_binning_f64_rows(P, W, H, _p(radii, P_i32), _p(m2, P_f64), _p(d, P_f64), _p(counts, P_u32),
                                  row_lo, row_hi, _p(keys, P_u64), _p(vals, P_u32), _p(ranges, P_u32))
    return dict(num_rendered=R, keys=keys, point_list=vals, ranges=ranges)


def render_forward(W, H, ranges, point_list, means2D, conic_opacity, rgb, bg, nthreads=None,
                   seam_wrap=False):
    """Forward blend; ``seam_wrap`` measures x offsets to the splat copy nearest the centre of
    each pixel's 8-column block."""
    ranges = np.ascontiguousarray(ranges, np.uint32)
    point_list = np.ascontiguousarray(point_list, np.uint32)
    means2D = np.ascontiguousarray(means2D, np.float64)
    conic_opacity = np.ascontiguousarray(conic_opacity, np.float64)
    rgb = np.ascontiguousarray(rgb, np.float64)
    bg = _f32(bg)
    out = np.zeros((3, H, W))
    final_T = np.zeros(H * W)
    n_contrib = np.zeros(H * W, np.uint32)
    lib().oracle_render_forward_seam(W, H, _p(ranges, P_u32), _p(point_list, P_u32), _p(means2D, P_f64),
                                     _p(conic_opacity, P_f64), _p(rgb, P_f64), _p(bg, P_f32),
                                     _p(out, P_f64), _p(final_T, P_f64), _p(n_contrib, P_u32),
                                     1 if seam_wrap else 0, nthreads or default_threads())
    return dict(image=out, final_T=final_T, n_contrib=n_contrib)


def render_backward(P, W, H, ranges, point_list, means2D, conic_opacity, rgb, bg, final_T,
                    n_contrib, dL_dpix, nthreads=None, seam_wrap=False):
    ranges = np.ascontiguousarray(ranges, np.uint32)
    point_list = np.ascontiguousarray(point_list, np.uint32)
    means2D = np.ascontiguousarray(means2D, np.float64)
    conic_opacity = np.ascontiguousarray(conic_opacity, np.float64)
    rgb = np.ascontiguousarray(rgb, np.float64)
    final_T = np.ascontiguousarray(final_T, np.float64)
    n_contrib = np.ascontiguousarray(n_contrib, np.uint32)
    bg, dL_dpix = _f32(bg), _f32(dL_dpix)
    out = dict(dL_dmean2D=np.zeros((P, 3)), dL_dconic=np.zeros((P, 4)), dL_dopacity=np.zeros(P),
               dL_dcolor=np.zeros((P, 3)))
    lib().oracle_render_backward_seam(
        P, W, H, _p(ranges, P_u32), _p(point_list, P_u32), ctypes.c_int64(point_list.shape[0]),
        _p(means2D, P_f64), _p(conic_opacity, P_f64), _p(rgb, P_f64), _p(bg, P_f32),
        _p(final_T, P_f64), _p(n_contrib, P_u32), _p(dL_dpix, P_f32), _p(out["dL_dmean2D"], P_f64),
        _p(out["dL_dconic"], P_f64), _p(out["dL_dopacity"], P_f64), _p(out["dL_dcolor"], P_f64),
        1 if seam_wrap else 0, nthreads or default_threads())
    return out


def preprocess_backward(means3D, radii, shs, clamped, scales, rotations, viewmatrix, campos, W, H,
                        dL_dmean2D, dL_dconic, dL_dcolor, D=3, scale_modifier=1.0,
                        cov3D_precomp=None, nthreads=None):
    means3D, shs, scales, rotations = map(_f32, (means3D, shs, scales, rotations))
    cov3D_precomp, viewmatrix, campos = map(_f32, (cov3D_precomp, viewmatrix, campos))
    radii = np.ascontiguousarray(radii, np.int32)
    clamped = np.ascontiguousarray(clamped, np.uint8)
    dL_dmean2D = np.ascontiguousarray(dL_dmean2D, np.float64)
    dL_dconic = np.ascontiguousarray(dL_dconic, np.float64)
    dL_dcolor = np.ascontiguousarray(dL_dcolor, np.float64)
    P = means3D.shape[0]
    M = 0 if shs is None else shs.shape[1]
    out = dict(dL_dmeans3D=np.zeros((P, 3)), dL_dcov3D=np.zeros((P, 6)),
               dL_dsh=np.zeros((P, M, 3)), dL_dscales=np.zeros((P, 3)),
               dL_drotations=np.zeros((P, 4)))
    lib().oracle_preprocess_backward(
        P, D, M, W, H, _p(means3D, P_f32), _p(radii, P_i32), _p(shs, P_f32), _p(clamped, P_u8),
        _p(scales, P_f32), ctypes.c_float(scale_modifier), _p(rotations, P_f32),
        _p(cov3D_precomp, P_f32), _p(viewmatrix, P_f32), _p(campos, P_f32),
        _p(dL_dmean2D, P_f64), _p(dL_dconic, P_f64), _p(dL_dcolor, P_f64),
        _p(out["dL_dmeans3D"], P_f64), _p(out["dL_dcov3D"], P_f64),
        _p(out["dL_dsh"] if M > 0 else None, P_f64), _p(out["dL_dscales"], P_f64),
        _p(out["dL_drotations"], P_f64), nthreads or default_threads())
    return out


def forward_backward(g, view, dL_dpix, bg=(0.0, 0.0, 0.0), D=3, scale_modifier=1.0,
                     nthreads=None, seam_wrap=False):
    """Whole FP64 pipeline on a scene (``omnigs_b200.scenes.Gaussians``) and a view
    (``seam_wrap``: the seam-wrapping mode in every stage)."""
    W, H = view.width, view.height
    bg = np.asarray(bg, np.float32)
    pre = preprocess(g.means3D, g.scales, g.rotations, g.opacities, g.shs, view.viewmatrix,
                     view.campos, W, H, D=D, scale_modifier=scale_modifier, nthreads=nthreads,
                     seam_wrap=seam_wrap)
    b = binning(W, H, pre["radii"], pre["means2D"], pre["depths"], pre["tiles_touched"], f32=False,
                seam_wrap=seam_wrap)
    fw = render_forward(W, H, b["ranges"], b["point_list"], pre["means2D"], pre["conic_opacity"],
                        pre["rgb"], bg, nthreads=nthreads, seam_wrap=seam_wrap)
    bw = render_backward(g.P, W, H, b["ranges"], b["point_list"], pre["means2D"],
                         pre["conic_opacity"], pre["rgb"], bg, fw["final_T"], fw["n_contrib"],
                         dL_dpix, nthreads=nthreads, seam_wrap=seam_wrap)
    pb = preprocess_backward(g.means3D, pre["radii"], g.shs, pre["clamped"], g.scales, g.rotations,
                             view.viewmatrix, view.campos, W, H, bw["dL_dmean2D"], bw["dL_dconic"],
                             bw["dL_dcolor"], D=D, scale_modifier=scale_modifier, nthreads=nthreads)
    out = dict(pre=pre, binning=b, **fw, **bw, **pb)
    out["dL_dopacity"] = bw["dL_dopacity"].reshape(-1, 1)
    return out
