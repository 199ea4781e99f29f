"""omnigs_b200: B200-native (sm_100a) equirectangular differentiable Gaussian rasterizer.

Drop-in replacement for the camera_type = 3 path of OmniGS's rasterizer:

* ``include/omnigs_b200.h`` -- the C ABI (``omnigs_b200/lib/libomnigs_b200.so``);
* ``torch_ext()`` -- the LibTorch layer with the reference's ``RasterizeGaussiansCUDA`` /
  ``RasterizeGaussiansBackwardCUDA`` / ``markVisible`` signatures and its autograd Function;
* ``GaussianRasterizer`` / ``GaussianRasterizationSettings`` -- the Python face of that layer;
* ``lonlat.LonlatState`` -- direct C-ABI driver used by tests and the benchmark.

The compute path is CUDA only: nothing here falls back to a CPU implementation.
"""
from __future__ import annotations

import importlib.util
import os
import sysconfig

from .rasterizer import GaussianRasterizationSettings, GaussianRasterizer  # noqa: F401

_HERE = os.path.dirname(os.path.abspath(__file__))
_ext = None


def set_recompute_transmittance(on: bool) -> None:
    """Transmittance checkpointing for the following LibTorch-layer forwards of this process: no
    per-pixel state is stored and the backward recomputes it (OMNIGS_FLAG_RECOMPUTE_T)."""
    torch_ext().set_recompute_transmittance(bool(on))


def torch_ext():
    """Import the LibTorch extension (omnigs_b200/lib/_omnigs_torch*.so); raises if not built."""
    global _ext
    if _ext is None:
        import torch  # noqa: F401  (loads libtorch / libc10 before the extension)
        path = os.path.join(_HERE, "lib", "_omnigs_torch" + sysconfig.get_config_var("EXT_SUFFIX"))
        if not os.path.exists(path):
            raise ImportError(f"{path} is missing; build it with `python -m omnigs_b200.build`")
        spec = importlib.util.spec_from_file_location("_omnigs_torch", path)
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        _ext = mod
    return _ext
