"""The drop-in recipe of INTEGRATION.md, compiled: the reference's own autograd layer
(src/gaussian_rasterizer.cpp and include/gaussian_rasterizer.h, unmodified, read where they lie in
the reference checkout) against this package's rasterize_points.h, linked to this package's
LibTorch layer and C-ABI library with every symbol resolved.

The reference header also includes camera.h (OpenCV) and gaussian_model.h (Sophus, simple-knn,
tinyply); tests/integration holds project-written stand-ins that supply the one enumeration the
autograd layer uses.  A temporary include tree of symbolic links (nothing is copied) puts the
reference's header next to those stand-ins and this package's rasterize_points.h, so its quoted
includes resolve to them.  Skipped where the reference checkout is absent (OMNIGS_REFERENCE,
default /root/reference); runs on the CPU (compile and link only).
"""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.environ.get("OMNIGS_REFERENCE", "/root/reference")
LIB = os.path.join(ROOT, "omnigs_b200", "lib")


@pytest.mark.skipif(not os.path.exists(os.path.join(REF, "src", "gaussian_rasterizer.cpp")),
                    reason="reference checkout not present")
def test_reference_autograd_layer_compiles_and_links_against_this_package(tmp_path):
    import torch
    import torch.utils.cpp_extension as ce

    assert os.path.exists(os.path.join(LIB, "libomnigs_b200.so")), "build the package first (python -m omnigs_b200.build)"
    inc = tmp_path / "include"
    src = tmp_path / "src"
    inc.mkdir()
    src.mkdir()
    links = {
        inc / "gaussian_rasterizer.h": os.path.join(REF, "include", "gaussian_rasterizer.h"),
        inc / "rasterize_points.h": os.path.join(ROOT, "omnigs_b200", "csrc", "torch", "rasterize_points.h"),
        inc / "camera.h": os.path.join(ROOT, "tests", "integration", "camera.h"),
        inc / "gaussian_model.h": os.path.join(ROOT, "tests", "integration", "gaussian_model.h"),
        src / "gaussian_rasterizer.cpp": os.path.join(REF, "src", "gaussian_rasterizer.cpp"),
    }
    for link, target in links.items():
        os.symlink(target, link)
    abi = int(torch._C._GLIBCXX_USE_CXX11_ABI)
    incs = [f"-I{tmp_path}"] + [f"-I{p}" for p in ce.include_paths()] + ["-I/usr/local/cuda/include"]
    flags = ["g++", "-O1", "-std=c++17", "-fPIC", f"-D_GLIBCXX_USE_CXX11_ABI={abi}", "-Wno-deprecated-declarations"]
    # the reference's autograd layer, unmodified
    obj = tmp_path / "gaussian_rasterizer.o"
    r = subprocess.run([*flags, *incs, "-c", str(src / "gaussian_rasterizer.cpp"), "-o", str(obj)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-4000:]
    # this package's LibTorch layer, built as the INTEGRATION.md target builds it
    ours = tmp_path / "rasterize_points.o"
    r = subprocess.run([*flags, f"-I{os.path.join(ROOT, 'include')}",
                        f"-I{os.path.join(ROOT, 'omnigs_b200', 'csrc', 'torch')}",
                        *[f"-I{p}" for p in ce.include_paths()], "-I/usr/local/cuda/include", "-c",
                        os.path.join(ROOT, "omnigs_b200", "csrc", "torch", "rasterize_points.cpp"), "-o", str(ours)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-4000:]
    # link the reference's autograd layer with this package's RasterizeGaussiansCUDA /
    # RasterizeGaussiansBackwardCUDA / markVisible and the C ABI; no symbol may stay undefined
    out = tmp_path / "libreference_autograd_on_omnigs.so"
    libdirs = ce.library_paths() + ["/usr/local/cuda/lib64", LIB]
    ld = ["g++", "-shared", "-o", str(out), str(obj), str(ours), *[f"-L{d}" for d in libdirs],
          "-lc10", "-ltorch", "-ltorch_cpu", "-lc10_cuda", "-ltorch_cuda", "-lomnigs_b200", "-lcudart",
          "-Wl,--no-undefined", f"-Wl,-rpath,{LIB}"]
    r = subprocess.run(ld, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-4000:]
    syms = subprocess.run(["nm", "-DC", "--defined-only", str(out)], capture_output=True, text=True).stdout
    for name in ("GaussianRasterizerFunction::forward", "GaussianRasterizerFunction::backward",
                 "GaussianRasterizer::forward", "RasterizeGaussiansCUDA", "RasterizeGaussiansBackwardCUDA",
                 "markVisible"):
        assert name in syms, name
