"""In-tree build of the native libraries.

* ``omnigs_b200/lib/libomnigs_b200.so`` -- the CUDA kernels and the C ABI (include/omnigs_b200.h),
  compiled with nvcc for sm_100a only.  No torch dependency.
* ``omnigs_b200/lib/_omnigs_torch*.so`` -- the LibTorch layer (RasterizeGaussiansCUDA /
  RasterizeGaussiansBackwardCUDA / markVisible with the reference's signatures, the
  torch::autograd::Function) plus its Python bindings, compiled with g++ against the installed
  torch and linked to the C-ABI library.

Both are rebuilt only when a source is newer than the product.  Products stay in the source tree
so that they travel with the repository snapshot.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys
import sysconfig

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB_DIR = os.path.join(HERE, "lib")
OBJ_DIR = os.path.join(LIB_DIR, "obj")
CAPI_LIB = os.path.join(LIB_DIR, "libomnigs_b200.so")
TORCH_EXT = os.path.join(LIB_DIR, "_omnigs_torch" + (sysconfig.get_config_var("EXT_SUFFIX") or ".so"))

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
CUDA_HOME = os.path.dirname(os.path.dirname(NVCC))
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
              "-Xptxas", "-warn-spills"]

CU_SOURCES = ["preprocess.cu", "binning.cu", "render_fwd.cu", "render_bwd.cu",
              "preprocess_bwd.cu", "batch.cu", "train.cu", "capi.cu", "batch_capi.cu", "noalloc.cu"]
HEADERS = glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) + \
    [os.path.join(ROOT, "include", "omnigs_b200.h")]
TORCH_SOURCES = ["torch/rasterize_points.cpp", "torch/gaussian_rasterizer.cpp", "torch/bindings.cpp"]
TORCH_HEADERS = glob.glob(os.path.join(CSRC, "torch", "*.h"))


def _newer(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def build_capi(verbose: bool = False, force: bool = False) -> str:
    from concurrent.futures import ThreadPoolExecutor

    os.makedirs(OBJ_DIR, exist_ok=True)
    objs, jobs = [], []
    for src in CU_SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(OBJ_DIR, src.replace(".cu", ".o"))
        objs.append(obj)
        if force or _newer(obj, [path] + HEADERS):
            jobs.append([NVCC, *ARCH, *NVCC_FLAGS, "-c", path, "-o", obj])
    # one nvcc per source, as many at once as there are cores
    with ThreadPoolExecutor(max_workers=max(1, os.cpu_count() or 1)) as pool:
        for f in [pool.submit(_run, cmd, verbose) for cmd in jobs]:
            f.result()
    if force or _newer(CAPI_LIB, objs):
        _run([NVCC, *ARCH, "-shared", "-o", CAPI_LIB, *objs, "-lcudart"], verbose)
    return CAPI_LIB


def build_torch_ext(verbose: bool = False, force: bool = False) -> str:
    import torch.utils.cpp_extension as ce
    import pybind11

    srcs = [os.path.join(CSRC, s) for s in TORCH_SOURCES]
    deps = srcs + TORCH_HEADERS + [os.path.join(ROOT, "include", "omnigs_b200.h"), CAPI_LIB]
    if not (force or _newer(TORCH_EXT, deps)):
        return TORCH_EXT
    os.makedirs(OBJ_DIR, exist_ok=True)
    incs = ce.include_paths() + [pybind11.get_include(), sysconfig.get_paths()["include"],
                                 os.path.join(CUDA_HOME, "include"), os.path.join(ROOT, "include"),
                                 CSRC]
    import torch
    abi = int(torch._C._GLIBCXX_USE_CXX11_ABI)
    cflags = ["-O2", "-std=c++17", "-fPIC", f"-D_GLIBCXX_USE_CXX11_ABI={abi}",
              "-DTORCH_EXTENSION_NAME=_omnigs_torch", "-DTORCH_API_INCLUDE_EXTENSION_H",
              "-Wno-deprecated-declarations"]
    objs = []
    for src in srcs:
        obj = os.path.join(OBJ_DIR, "torch_" + os.path.basename(src).replace(".cpp", ".o"))
        objs.append(obj)
        if force or _newer(obj, [src] + TORCH_HEADERS + [os.path.join(ROOT, "include", "omnigs_b200.h")]):
            _run(["g++", *cflags, *[f"-I{i}" for i in incs], "-c", src, "-o", obj], verbose)
    libdirs = ce.library_paths() + [os.path.join(CUDA_HOME, "lib64"), LIB_DIR]
    _run(["g++", "-shared", "-o", TORCH_EXT, *objs, *[f"-L{d}" for d in libdirs],
          "-lc10", "-ltorch", "-ltorch_cpu", "-ltorch_python", "-lc10_cuda", "-ltorch_cuda",
          "-lomnigs_b200", "-lcudart", "-Wl,-rpath,$ORIGIN",
          *[f"-Wl,-rpath,{d}" for d in ce.library_paths()]], verbose)
    return TORCH_EXT


def build_all(verbose: bool = False, force: bool = False):
    build_capi(verbose, force)
    build_torch_ext(verbose, force)


if __name__ == "__main__":
    build_all(verbose=True, force="--force" in sys.argv)
