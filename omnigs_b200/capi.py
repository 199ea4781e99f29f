"""ctypes binding of the C ABI in include/omnigs_b200.h (libomnigs_b200.so).

The functions here take torch CUDA tensors, pass their device pointers and the current CUDA
stream through the C ABI, and raise on a non-zero return code.  There is no CPU path: if the
library is missing this module raises instead of falling back.
"""
from __future__ import annotations

import ctypes
import os

import torch

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libomnigs_b200.so")

OMNIGS_OK = 0
ERR_NAMES = {1: "INVALID_ARGUMENT", 2: "BUFFER_TOO_SMALL", 3: "CUDA", 4: "UNSUPPORTED",
             5: "CAPACITY", 6: "DEVICE"}
STATUS_CAPACITY = 1
STATUS_LOOKBACK = 2
STATUS_OVERFLOW = 4
CAMERA_PINHOLE = 1
CAMERA_LONLAT = 3

_vp = ctypes.c_void_p
_i = ctypes.c_int
_f = ctypes.c_float


class ForwardArgs(ctypes.Structure):
    _fields_ = [("P", _i), ("D", _i), ("M", _i), ("W", _i), ("H", _i),
                ("background", _vp), ("means3D", _vp), ("shs", _vp), ("colors_precomp", _vp),
                ("opacities", _vp), ("scales", _vp), ("scale_modifier", _f), ("rotations", _vp),
                ("cov3D_precomp", _vp), ("viewmatrix", _vp), ("campos", _vp),
                ("out_color", _vp), ("radii", _vp), ("flags", _i)]


class BackwardArgs(ctypes.Structure):
    _fields_ = [("P", _i), ("D", _i), ("M", _i), ("W", _i), ("H", _i), ("R", _i),
                ("background", _vp), ("means3D", _vp), ("shs", _vp), ("colors_precomp", _vp),
                ("scales", _vp), ("scale_modifier", _f), ("rotations", _vp), ("cov3D_precomp", _vp),
                ("viewmatrix", _vp), ("campos", _vp), ("radii", _vp), ("dL_dout_color", _vp),
                ("dL_dmeans2D", _vp), ("dL_dcolors", _vp), ("dL_dopacity", _vp),
                ("dL_dmeans3D", _vp), ("dL_dcov3D", _vp), ("dL_dsh", _vp), ("dL_dscales", _vp),
                ("dL_drotations", _vp), ("dL_dconic", _vp), ("flags", _i)]


STAGES = ["preprocess", "duplicate", "sort", "ranges", "render_forward", "render_backward",
          "preprocess_backward", "other"]


class StageTimes(ctypes.Structure):
    _fields_ = [("ms", ctypes.c_double * 8), ("launches", ctypes.c_uint64 * 8)]


class GeomView(ctypes.Structure):
    _fields_ = [("splat", _vp), ("color", _vp), ("depth", _vp), ("tiles_touched", _vp),
                ("depth_order", _vp)]


class BinningView(ctypes.Structure):
    _fields_ = [("tile_ids", _vp), ("point_list", _vp)]


class ImageView(ctypes.Structure):
    _fields_ = [("final_T", _vp), ("n_contrib", _vp), ("ranges", _vp)]


MAX_BATCH_VIEWS = 32
SH_FP32 = 0
SH_BF16 = 1


class BatchView(ctypes.Structure):
    _fields_ = [("W", _i), ("H", _i), ("out_color", _vp), ("dL_dout_color", _vp)]


class BatchArgs(ctypes.Structure):
    _fields_ = [("P", _i), ("D", _i), ("M", _i), ("V", _i), ("sh_dtype", _i), ("fp64_poles", _i),
                ("means3D", _vp), ("shs", _vp), ("colors_precomp", _vp), ("opacities", _vp),
                ("scales", _vp), ("scale_modifier", _f), ("rotations", _vp), ("cov3D_precomp", _vp),
                ("viewmatrices", _vp), ("campos", _vp), ("backgrounds", _vp),
                ("views", ctypes.POINTER(BatchView)), ("seam_wrap", _i)]


class BatchGrads(ctypes.Structure):
    _fields_ = [("dL_dmeans3D", _vp), ("dL_dsh", _vp), ("dL_dopacity", _vp), ("dL_dscales", _vp),
                ("dL_drotations", _vp), ("dL_dcolors", _vp), ("dL_dcov3D", _vp),
                ("grad_accum", _vp), ("denom", _vp), ("max_radii", _vp)]


class BatchStateView(ctypes.Structure):
    _fields_ = [("radii", _vp), ("splat", _vp), ("color", _vp), ("final_T", _vp),
                ("n_contrib", _vp), ("ranges", _vp),
                ("pixel_base", ctypes.c_int64 * MAX_BATCH_VIEWS),
                ("tile_base", ctypes.c_int64 * MAX_BATCH_VIEWS), ("tile_passes", _i), ("depth", _vp)]


class GaussianParams(ctypes.Structure):
    _fields_ = [("P", _i), ("M", _i), ("xyz", _vp), ("features_dc", _vp), ("features_rest", _vp),
                ("opacity", _vp), ("scaling", _vp), ("rotation", _vp)]


class AdamState(ctypes.Structure):
    _fields_ = [(n, _vp) for n in ("m_xyz", "v_xyz", "m_dc", "v_dc", "m_rest", "v_rest", "m_opacity",
                                   "v_opacity", "m_scaling", "v_scaling", "m_rotation", "v_rotation")]


class Activated(ctypes.Structure):
    _fields_ = [("means3D", _vp), ("shs", _vp), ("shs_bf16", _i), ("opacities", _vp), ("scales", _vp),
                ("rotations", _vp)]


class AdamHyper(ctypes.Structure):
    _fields_ = [("lr", ctypes.c_double * 6), ("beta1", ctypes.c_double), ("beta2", ctypes.c_double),
                ("eps", ctypes.c_double), ("step", ctypes.c_int64)]


class TuneResult(ctypes.Structure):
    _fields_ = [("candidates", _i * 3), ("forward_ms", _f * 3), ("backward_ms", _f * 3),
                ("forward_batch", _i), ("backward_batch", _i)]


# every symbol include/omnigs_b200.h declares
EXPORTED = ["omnigs_version", "omnigs_last_error", "omnigs_lonlat_geom_bytes",
            "omnigs_lonlat_image_bytes", "omnigs_lonlat_image_bytes_flags", "omnigs_lonlat_binning_bytes",
            "omnigs_lonlat_binning_capacity", "omnigs_lonlat_preprocess", "omnigs_lonlat_render",
            "omnigs_lonlat_forward", "omnigs_lonlat_forward_noalloc", "omnigs_lonlat_forward_early_status",
            "omnigs_lonlat_read_status",
            "omnigs_lonlat_backward",
            "omnigs_mark_visible", "omnigs_timing_enable", "omnigs_timing_read",
            "omnigs_kernel_launches", "omnigs_lonlat_geom_view", "omnigs_lonlat_binning_view",
            "omnigs_lonlat_image_view", "omnigs_batch_state_bytes", "omnigs_batch_forward",
            "omnigs_batch_render", "omnigs_batch_backward", "omnigs_batch_read_status",
            "omnigs_batch_state_view", "omnigs_batch_binning_view", "omnigs_l1_dssim_workspace_bytes", "omnigs_l1_dssim",
            "omnigs_activate", "omnigs_adam_step", "omnigs_set_blend_batch", "omnigs_get_blend_batch",
            "omnigs_batch_autotune", "omnigs_debug_lookback_timeout"]

_lib = None


def lib() -> ctypes.CDLL:
    """Load libomnigs_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing; build it with `python -m omnigs_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        L.omnigs_version.restype = ctypes.c_char_p
        L.omnigs_last_error.restype = ctypes.c_char_p
        L.omnigs_lonlat_geom_bytes.restype = ctypes.c_size_t
        L.omnigs_lonlat_geom_bytes.argtypes = [_i]
        L.omnigs_lonlat_image_bytes.restype = ctypes.c_size_t
        L.omnigs_lonlat_image_bytes.argtypes = [_i, _i]
        L.omnigs_lonlat_image_bytes_flags.restype = ctypes.c_size_t
        L.omnigs_lonlat_image_bytes_flags.argtypes = [_i, _i, _i]
        L.omnigs_lonlat_binning_bytes.restype = ctypes.c_size_t
        L.omnigs_lonlat_binning_bytes.argtypes = [ctypes.c_int64]
        L.omnigs_lonlat_binning_capacity.restype = ctypes.c_int64
        L.omnigs_lonlat_binning_capacity.argtypes = [ctypes.c_size_t]
        fw = [ctypes.POINTER(ForwardArgs), _vp, ctypes.c_size_t]
        L.omnigs_lonlat_preprocess.argtypes = fw + [_vp]
        L.omnigs_lonlat_render.argtypes = fw + [_vp, ctypes.c_size_t, _vp, ctypes.c_size_t, _vp]
        L.omnigs_lonlat_forward.argtypes = fw + [_vp, ctypes.c_size_t, _vp, ctypes.c_size_t, _vp]
        L.omnigs_lonlat_forward_noalloc.argtypes = [ctypes.POINTER(ForwardArgs), ctypes.POINTER(_i), _vp]
        L.omnigs_lonlat_forward_early_status.argtypes = fw + [_vp, ctypes.c_size_t, _vp, ctypes.c_size_t,
                                                              ctypes.POINTER(_i), ctypes.POINTER(ctypes.c_uint32),
                                                              _vp]
        L.omnigs_lonlat_read_status.argtypes = [_vp, ctypes.POINTER(_i),
                                                ctypes.POINTER(ctypes.c_uint32), _vp]
        L.omnigs_lonlat_backward.argtypes = [ctypes.POINTER(BackwardArgs), _vp, ctypes.c_size_t,
                                             _vp, ctypes.c_size_t, _vp, ctypes.c_size_t, _vp]
        L.omnigs_mark_visible.argtypes = [_i, _vp, _vp, _i, _vp, _vp]
        L.omnigs_timing_enable.argtypes = [_i]
        L.omnigs_timing_read.argtypes = [ctypes.POINTER(StageTimes)]
        L.omnigs_kernel_launches.restype = ctypes.c_uint64
        L.omnigs_lonlat_geom_view.argtypes = [_vp, _i, ctypes.POINTER(GeomView)]
        L.omnigs_lonlat_binning_view.argtypes = [_vp, ctypes.c_size_t, _i, _i,
                                                 ctypes.POINTER(BinningView)]
        L.omnigs_lonlat_image_view.argtypes = [_vp, _i, _i, ctypes.POINTER(ImageView)]
        ip = ctypes.POINTER(_i)
        L.omnigs_batch_state_bytes.restype = ctypes.c_size_t
        L.omnigs_batch_state_bytes.argtypes = [_i, _i, ip, ip]
        bfw = [ctypes.POINTER(BatchArgs), _vp, ctypes.c_size_t, _vp, ctypes.c_size_t, _vp]
        L.omnigs_batch_forward.argtypes = bfw
        L.omnigs_batch_render.argtypes = bfw
        L.omnigs_batch_backward.argtypes = [ctypes.POINTER(BatchArgs), ctypes.POINTER(BatchGrads), _vp,
                                            ctypes.c_size_t, _vp, ctypes.c_size_t, _vp]
        L.omnigs_batch_read_status.argtypes = [_vp, _i, ctypes.POINTER(ctypes.c_int64),
                                               ctypes.POINTER(ctypes.c_int64),
                                               ctypes.POINTER(ctypes.c_uint32), _vp]
        L.omnigs_batch_state_view.argtypes = [_vp, _i, _i, ip, ip, ctypes.POINTER(BatchStateView)]
        L.omnigs_debug_lookback_timeout.argtypes = fw + [_vp, ctypes.c_size_t, _vp, ctypes.c_size_t, _i,
                                                         ctypes.POINTER(ctypes.c_uint32), _vp]
        L.omnigs_batch_binning_view.argtypes = [_vp, ctypes.c_size_t, _i, _i, ip, ip, ctypes.POINTER(BinningView)]
        L.omnigs_l1_dssim_workspace_bytes.restype = ctypes.c_size_t
        L.omnigs_l1_dssim_workspace_bytes.argtypes = [_i, _i, _i]
        L.omnigs_l1_dssim.argtypes = [_vp, _vp, _i, _i, _i, _i, _f, _vp, _vp, _vp, ctypes.c_size_t, _vp]
        L.omnigs_set_blend_batch.argtypes = [_i, _i]
        L.omnigs_get_blend_batch.argtypes = [ctypes.POINTER(_i), ctypes.POINTER(_i)]
        L.omnigs_batch_autotune.argtypes = [ctypes.POINTER(BatchArgs), _vp, ctypes.c_size_t, _vp, ctypes.c_size_t,
                                            _i, ctypes.POINTER(TuneResult), _vp]
        L.omnigs_activate.argtypes = [ctypes.POINTER(GaussianParams), ctypes.POINTER(Activated), _vp]
        L.omnigs_adam_step.argtypes = [ctypes.POINTER(GaussianParams), ctypes.POINTER(AdamState),
                                       ctypes.POINTER(Activated), _vp, _vp, _vp, _vp, _vp, _vp, _vp]
        _lib = L
    return _lib


class OmnigsError(RuntimeError):
    pass


def check(rc: int, what: str):
    if rc != OMNIGS_OK:
        msg = lib().omnigs_last_error().decode()
        raise OmnigsError(f"{what} failed: {ERR_NAMES.get(rc, rc)}: {msg}")


def ptr(t: torch.Tensor | None):
    if t is None or t.numel() == 0:
        return None
    assert t.is_cuda and t.is_contiguous(), "C-ABI arguments must be contiguous CUDA tensors"
    return t.data_ptr()


def stream_handle(stream: torch.cuda.Stream | None = None):
    s = stream if stream is not None else torch.cuda.current_stream()
    return s.cuda_stream


def geom_bytes(P: int) -> int:
    return int(lib().omnigs_lonlat_geom_bytes(P))


FLAG_RECOMPUTE_T = 1  # OMNIGS_FLAG_RECOMPUTE_T


def image_bytes(W: int, H: int, flags: int = 0) -> int:
    return int(lib().omnigs_lonlat_image_bytes_flags(W, H, flags))


def binning_bytes(capacity: int) -> int:
    return int(lib().omnigs_lonlat_binning_bytes(capacity))


def binning_capacity(nbytes: int) -> int:
    return int(lib().omnigs_lonlat_binning_capacity(nbytes))


def batch_state_bytes(P: int, sizes) -> int:
    """Bytes of the batch state for P Gaussians and views of the given (W, H) sizes (0 if invalid)."""
    V = len(sizes)
    W = (_i * max(V, 1))(*[w for w, _ in sizes])
    H = (_i * max(V, 1))(*[h for _, h in sizes])
    return int(lib().omnigs_batch_state_bytes(P, V, W, H))


def timing_enable(on: bool):
    lib().omnigs_timing_enable(1 if on else 0)


def timing_read() -> dict:
    """{stage: (total_ms, launches)} since the last read (waits for the recorded events)."""
    t = StageTimes()
    check(lib().omnigs_timing_read(ctypes.byref(t)), "omnigs_timing_read")
    return {name: (float(t.ms[i]), int(t.launches[i])) for i, name in enumerate(STAGES)}


def kernel_launches() -> int:
    return int(lib().omnigs_kernel_launches())
