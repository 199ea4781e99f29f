// Python bindings of the LibTorch layer (module omnigs_b200.lib._omnigs_torch).  The functions
// keep the reference's argument order; `rasterize` runs the C++ autograd Function so that Python
// autograd differentiates through the same code a LibTorch trainer uses.
#include <torch/extension.h>

#include "gaussian_rasterizer.h"
#include "omnigs_b200.h"
#include "omnigs_settings.h"
#include "rasterize_points.h"

namespace {

std::vector<torch::Tensor> rasterize(torch::Tensor means3D, torch::Tensor means2D, torch::Tensor sh,
                                     torch::Tensor colors_precomp, torch::Tensor opacities, torch::Tensor scales,
                                     torch::Tensor rotations, torch::Tensor cov3Ds_precomp, int image_height,
                                     int image_width, double tanfovx, double tanfovy, torch::Tensor bg,
                                     double scale_modifier, torch::Tensor viewmatrix, torch::Tensor projmatrix,
                                     int sh_degree, torch::Tensor campos, bool prefiltered, int camera_type) {
  omnigs::GaussianRasterizationSettings settings(image_height, image_width, (float)tanfovx, (float)tanfovy, bg,
                                                 (float)scale_modifier, viewmatrix, projmatrix, torch::Tensor(),
                                                 sh_degree, campos, prefiltered, camera_type);
  auto out = omnigs::rasterizeGaussians(means3D, means2D, sh, colors_precomp, opacities, scales, rotations,
                                        cov3Ds_precomp, settings);
  return {out[0], out[1]};
}

}  // namespace

PYBIND11_MODULE(TORCH_EXTENSION_NAME, m) {
  m.doc() = "LibTorch boundary of the omnigs_b200 equirectangular Gaussian rasterizer";
  m.def("rasterize_gaussians_cuda", &RasterizeGaussiansCUDA, "RasterizeGaussiansCUDA (reference signature)",
        py::arg("background"), py::arg("means3D"), py::arg("colors"), py::arg("opacity"), py::arg("scales"),
        py::arg("rotations"), py::arg("scale_modifier"), py::arg("cov3D_precomp"), py::arg("viewmatrix"),
        py::arg("projmatrix"), py::arg("tan_fovx"), py::arg("tan_fovy"), py::arg("image_height"),
        py::arg("image_width"), py::arg("sh"), py::arg("degree"), py::arg("campos"), py::arg("prefiltered"),
        py::arg("camera_type") = 1, py::arg("render_depth") = false);
  m.def("rasterize_gaussians_backward_cuda", &RasterizeGaussiansBackwardCUDA,
        "RasterizeGaussiansBackwardCUDA (reference signature)", py::arg("background"), py::arg("means3D"),
        py::arg("radii"), py::arg("colors"), py::arg("scales"), py::arg("rotations"), py::arg("scale_modifier"),
        py::arg("cov3D_precomp"), py::arg("viewmatrix"), py::arg("projmatrix"), py::arg("tan_fovx"),
        py::arg("tan_fovy"), py::arg("dL_dout_color"), py::arg("sh"), py::arg("degree"), py::arg("campos"),
        py::arg("geomBuffer"), py::arg("R"), py::arg("binningBuffer"), py::arg("imageBuffer"),
        py::arg("camera_type") = 1);
  m.def("mark_visible", &markVisible, "markVisible (reference signature)", py::arg("means3D"),
        py::arg("viewmatrix"), py::arg("projmatrix"), py::arg("camera_type") = 1);
  m.def("rasterize", &rasterize, "GaussianRasterizerFunction::apply (autograd)");
  m.def("version", []() { return std::string(omnigs_version()); });
  m.def("set_recompute_transmittance", &omnigs_torch_set_recompute_transmittance,
        "transmittance checkpointing for the following forwards (omnigs_settings.h)");
  m.def("recompute_transmittance", &omnigs_torch_recompute_transmittance);
}
