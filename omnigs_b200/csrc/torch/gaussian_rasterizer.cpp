// Autograd wrapper (behaviour of OmniGS src/gaussian_rasterizer.cpp:24-223): the forward saves the
// same 14 tensors and 6 scalars, the backward returns the 9 gradients in the reference's order
// (means3D, means2D, sh, colors, opacities, scales, rotations, cov3D, none).
#include "gaussian_rasterizer.h"

#include <stdexcept>

namespace omnigs {

torch::Tensor GaussianRasterizer::markVisibleGaussians(torch::Tensor& positions) {
  torch::NoGradGuard no_grad;
  auto s = raster_settings_;
  return markVisible(positions, s.viewmatrix_, s.projmatrix_, s.camera_type_);
}

torch::autograd::tensor_list GaussianRasterizerFunction::forward(
    torch::autograd::AutogradContext* ctx, torch::Tensor means3D, torch::Tensor means2D, torch::Tensor sh,
    torch::Tensor colors_precomp, torch::Tensor opacities, torch::Tensor scales, torch::Tensor rotations,
    torch::Tensor cov3Ds_precomp, GaussianRasterizationSettings raster_settings) {
  (void)means2D;
  auto result = RasterizeGaussiansCUDA(
      raster_settings.bg_, means3D, colors_precomp, opacities, scales, rotations, raster_settings.scale_modifier_,
      cov3Ds_precomp, raster_settings.viewmatrix_, raster_settings.projmatrix_, raster_settings.tanfovx_,
      raster_settings.tanfovy_, raster_settings.image_height_, raster_settings.image_width_, sh,
      raster_settings.sh_degree_, raster_settings.campos_, raster_settings.prefiltered_,
      raster_settings.camera_type_, raster_settings.render_depth_);
  auto num_rendered = std::get<0>(result);
  auto color = std::get<1>(result);
  auto radii = std::get<2>(result);
  ctx->saved_data["num_rendered"] = num_rendered;
  ctx->saved_data["scale_modifier"] = raster_settings.scale_modifier_;
  ctx->saved_data["tanfovx"] = raster_settings.tanfovx_;
  ctx->saved_data["tanfovy"] = raster_settings.tanfovy_;
  ctx->saved_data["sh_degree"] = raster_settings.sh_degree_;
  ctx->saved_data["camera_type"] = raster_settings.camera_type_;
  ctx->saved_data["image_height"] = raster_settings.image_height_;
  ctx->saved_data["image_width"] = raster_settings.image_width_;
  ctx->save_for_backward({raster_settings.bg_, raster_settings.viewmatrix_, raster_settings.projmatrix_,
                          raster_settings.campos_, colors_precomp, means3D, scales, rotations, cov3Ds_precomp,
                          radii, sh, std::get<3>(result), std::get<4>(result), std::get<5>(result)});
  ctx->mark_non_differentiable({radii});
  return {color, radii};
}

torch::autograd::tensor_list GaussianRasterizerFunction::backward(torch::autograd::AutogradContext* ctx,
                                                                  torch::autograd::tensor_list grad_outputs) {
  const auto num_rendered = ctx->saved_data["num_rendered"].toInt();
  const auto scale_modifier = static_cast<float>(ctx->saved_data["scale_modifier"].toDouble());
  const auto tanfovx = static_cast<float>(ctx->saved_data["tanfovx"].toDouble());
  const auto tanfovy = static_cast<float>(ctx->saved_data["tanfovy"].toDouble());
  const auto sh_degree = ctx->saved_data["sh_degree"].toInt();
  const auto camera_type = ctx->saved_data["camera_type"].toInt();
  auto saved = ctx->get_saved_variables();
  auto grad_out_color = grad_outputs[0];
  if (!grad_out_color.defined())
    grad_out_color = torch::zeros({3, ctx->saved_data["image_height"].toInt(), ctx->saved_data["image_width"].toInt()},
                                  saved[5].options());
  auto r = RasterizeGaussiansBackwardCUDA(saved[0], saved[5], saved[9], saved[4], saved[6], saved[7],
                                          scale_modifier, saved[8], saved[1], saved[2], tanfovx, tanfovy,
                                          grad_out_color.contiguous(), saved[10], sh_degree, saved[3], saved[11],
                                          num_rendered, saved[12], saved[13], camera_type);
  return {std::get<3>(r), std::get<0>(r), std::get<5>(r), std::get<1>(r), std::get<2>(r),
          std::get<6>(r), std::get<7>(r), std::get<4>(r), torch::Tensor()};
}

std::tuple<torch::Tensor, torch::Tensor> GaussianRasterizer::forward(
    torch::Tensor means3D, torch::Tensor means2D, torch::Tensor opacities, bool has_shs, bool has_colors_precomp,
    bool has_scales, bool has_rotations, bool has_cov3D_precomp, torch::Tensor shs, torch::Tensor colors_precomp,
    torch::Tensor scales, torch::Tensor rotations, torch::Tensor cov3D_precomp) {
  auto raster_settings = raster_settings_;
  if ((!has_shs && !has_colors_precomp) || (has_shs && has_colors_precomp))
    throw std::runtime_error("Please provide excatly one of either SHs or precomputed colors!");
  if (((!has_scales || !has_rotations) && !has_cov3D_precomp) ||
      ((has_scales || has_rotations) && has_cov3D_precomp))
    throw std::runtime_error("Please provide exactly one of either scale/rotation pair or precomputed 3D covariance!");
  auto empty = [&]() { return torch::empty({0}, means3D.options()); };
  if (!has_shs) shs = empty();
  if (!has_colors_precomp) colors_precomp = empty();
  if (!has_scales) scales = empty();
  if (!has_rotations) rotations = empty();
  if (!has_cov3D_precomp) cov3D_precomp = empty();
  auto result = rasterizeGaussians(means3D, means2D, shs, colors_precomp, opacities, scales, rotations,
                                   cov3D_precomp, raster_settings);
  return std::make_tuple(result[0], result[1]);
}

}  // namespace omnigs
