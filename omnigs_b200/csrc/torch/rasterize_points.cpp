// LibTorch boundary over the C ABI (mirrors the reference's src/rasterize_points.cu:41-319).
//
// Differences from the reference, none visible in the returned values:
//  * all launches go to the current CUDA stream of the input's device;
//  * the binning buffer is sized from a capacity hint (the previous call's instance count, or a
//    per-Gaussian estimate), so the pipeline runs without the reference's mid-pass device-to-host
//    copy; the one host wait reads num_rendered (which this API returns by value) once the
//    binning has run, while the blend still runs, and only when the hint was too small is the
//    binning stage resized and re-run;
//  * gradient outputs are allocated uninitialised because the backward writes every element;
//  * optional transmittance checkpointing (omnigs_settings.h).
#include "rasterize_points.h"

#include <ATen/cuda/CUDAContext.h>
#include <c10/cuda/CUDAGuard.h>

#include <atomic>
#include <stdexcept>

#include "omnigs_b200.h"
#include "omnigs_settings.h"

namespace {

constexpr int kChannels = 3;  // NUM_CHANNELS, cuda_rasterizer/config.h:25

std::atomic<int64_t> g_capacity_hint{0};
std::atomic<int> g_forward_flags{0};  // OMNIGS_FLAG_* of the next forwards

void check_rc(int rc, const char* what) {
  if (rc != OMNIGS_OK)
    throw std::runtime_error(std::string("[omnigs_b200] ") + what + ": " + omnigs_last_error());
}

// Contiguous float32 view of an optional input, kept alive by the holder; NULL when empty.
struct FloatIn {
  torch::Tensor t;
  const float* ptr = nullptr;
  explicit FloatIn(const torch::Tensor& x) {
    if (x.defined() && x.numel() > 0) {
      TORCH_CHECK(x.is_cuda(), "omnigs_b200: input tensors must be CUDA tensors");
      TORCH_CHECK(x.scalar_type() == torch::kFloat32, "omnigs_b200: input tensors must be float32");
      t = x.contiguous();
      ptr = t.data_ptr<float>();
    }
  }
};

[[noreturn]] void unsupported_camera(int camera_type) {
  if (camera_type == OMNIGS_CAMERA_PINHOLE)
    throw std::runtime_error(
        "[omnigs_b200] camera_type 1 (pinhole) is not provided: this library implements the "
        "equirectangular (camera_type 3) rasterizer");
  throw std::runtime_error("[CudaRasterizer]Invalid camera_type");
}

}  // namespace

void omnigs_torch_set_recompute_transmittance(bool on) { g_forward_flags.store(on ? OMNIGS_FLAG_RECOMPUTE_T : 0); }
bool omnigs_torch_recompute_transmittance() { return (g_forward_flags.load() & OMNIGS_FLAG_RECOMPUTE_T) != 0; }

std::tuple<int, torch::Tensor, torch::Tensor, torch::Tensor, torch::Tensor, torch::Tensor>
RasterizeGaussiansCUDA(const torch::Tensor& background, const torch::Tensor& means3D,
                       const torch::Tensor& colors, const torch::Tensor& opacity,
                       const torch::Tensor& scales, const torch::Tensor& rotations,
                       const float scale_modifier, const torch::Tensor& cov3D_precomp,
                       const torch::Tensor& viewmatrix, const torch::Tensor& projmatrix,
                       const float tan_fovx, const float tan_fovy, const int image_height,
                       const int image_width, const torch::Tensor& sh, const int degree,
                       const torch::Tensor& campos, const bool prefiltered, const int camera_type,
                       const bool render_depth) {
  if (means3D.ndimension() != 2 || means3D.size(1) != 3) {
    AT_ERROR("means3D must have dimensions (num_points, 3)");
  }
  (void)projmatrix; (void)tan_fovx; (void)tan_fovy; (void)prefiltered; (void)render_depth;
  const int P = means3D.size(0);
  const int H = image_height;
  const int W = image_width;
  auto float_opts = means3D.options().dtype(torch::kFloat32);
  torch::Tensor out_color = torch::full({kChannels, H, W}, 0.0, float_opts);
  torch::Tensor radii = torch::full({P}, 0, means3D.options().dtype(torch::kInt32));
  torch::TensorOptions byte_opts = torch::TensorOptions().dtype(torch::kByte).device(means3D.device());
  torch::Tensor geomBuffer = torch::empty({0}, byte_opts);
  torch::Tensor binningBuffer = torch::empty({0}, byte_opts);
  torch::Tensor imgBuffer = torch::empty({0}, byte_opts);

  int rendered = 0;
  if (P != 0) {
    if (camera_type != OMNIGS_CAMERA_LONLAT) unsupported_camera(camera_type);
    TORCH_CHECK(means3D.is_cuda(), "omnigs_b200: means3D must be a CUDA tensor");
    c10::cuda::CUDAGuard guard(means3D.device());
    cudaStream_t stream = at::cuda::getCurrentCUDAStream().stream();
    int M = 0;
    if (sh.size(0) != 0) M = sh.size(1);
    FloatIn bg(background), m3(means3D), shs(sh), col(colors), op(opacity), sc(scales),
        rot(rotations), cov(cov3D_precomp), vm(viewmatrix), cp(campos);
    OmnigsLonlatForwardArgs a{};
    a.P = P;
    a.D = degree;
    a.M = M;
    a.W = W;
    a.H = H;
    a.background = bg.ptr;
    a.means3D = m3.ptr;
    a.shs = shs.ptr;
    a.colors_precomp = col.ptr;
    a.opacities = op.ptr;
    a.scales = sc.ptr;
    a.scale_modifier = scale_modifier;
    a.rotations = rot.ptr;
    a.cov3D_precomp = cov.ptr;
    a.viewmatrix = vm.ptr;
    a.campos = cp.ptr;
    a.out_color = out_color.data_ptr<float>();
    a.radii = radii.data_ptr<int>();
    a.flags = g_forward_flags.load();

    geomBuffer.resize_({(int64_t)omnigs_lonlat_geom_bytes(P)});
    imgBuffer.resize_({(int64_t)omnigs_lonlat_image_bytes_flags(W, H, a.flags)});
    const int64_t capacity = std::max<int64_t>(g_capacity_hint.load(), 4 * (int64_t)P);
    binningBuffer.resize_({(int64_t)omnigs_lonlat_binning_bytes(capacity)});
    auto s = reinterpret_cast<omnigs_stream_t>(stream);
    // returns once the binning has run (num_rendered and the status are final); the blend is still
    // running on the stream, so the caller's next launches overlap it
    uint32_t status = 0;
    check_rc(omnigs_lonlat_forward_early_status(&a, geomBuffer.data_ptr(), geomBuffer.numel(),
                                                binningBuffer.data_ptr(), binningBuffer.numel(),
                                                imgBuffer.data_ptr(), imgBuffer.numel(), &rendered, &status, s),
             "forward");
    if (status & OMNIGS_STATUS_CAPACITY) {
      binningBuffer.resize_({(int64_t)omnigs_lonlat_binning_bytes(rendered)});
      check_rc(omnigs_lonlat_render(&a, geomBuffer.data_ptr(), geomBuffer.numel(), binningBuffer.data_ptr(),
                                    binningBuffer.numel(), imgBuffer.data_ptr(), imgBuffer.numel(), s),
               "render");
      check_rc(omnigs_lonlat_read_status(geomBuffer.data_ptr(), &rendered, &status, s), "read status");
    }
    if (status != 0)
      throw std::runtime_error("[omnigs_b200] forward failed on the device (status bits " +
                               std::to_string(status) + ")");
    const int64_t hint = (int64_t)rendered + rendered / 8 + 1024;
    if (hint > g_capacity_hint.load()) g_capacity_hint.store(hint);
  }
  return std::make_tuple(rendered, out_color, radii, geomBuffer, binningBuffer, imgBuffer);
}

std::tuple<torch::Tensor, torch::Tensor, torch::Tensor, torch::Tensor, torch::Tensor, torch::Tensor,
           torch::Tensor, torch::Tensor>
RasterizeGaussiansBackwardCUDA(const torch::Tensor& background, const torch::Tensor& means3D,
                               const torch::Tensor& radii, const torch::Tensor& colors,
                               const torch::Tensor& scales, const torch::Tensor& rotations,
                               const float scale_modifier, const torch::Tensor& cov3D_precomp,
                               const torch::Tensor& viewmatrix, const torch::Tensor& projmatrix,
                               const float tan_fovx, const float tan_fovy,
                               const torch::Tensor& dL_dout_color, const torch::Tensor& sh,
                               const int degree, const torch::Tensor& campos,
                               const torch::Tensor& geomBuffer, const int R,
                               const torch::Tensor& binningBuffer, const torch::Tensor& imageBuffer,
                               const int camera_type) {
  (void)projmatrix; (void)tan_fovx; (void)tan_fovy;
  const int P = means3D.size(0);
  const int H = dL_dout_color.size(1);
  const int W = dL_dout_color.size(2);
  int M = 0;
  if (sh.size(0) != 0) M = sh.size(1);
  auto o = means3D.options();
  torch::Tensor dL_dmeans3D = torch::empty({P, 3}, o);
  torch::Tensor dL_dmeans2D = torch::empty({P, 3}, o);
  torch::Tensor dL_dcolors = torch::empty({P, kChannels}, o);
  torch::Tensor dL_dopacity = torch::empty({P, 1}, o);
  torch::Tensor dL_dcov3D = torch::empty({P, 6}, o);
  torch::Tensor dL_dsh = torch::empty({P, M, 3}, o);
  torch::Tensor dL_dscales = torch::empty({P, 3}, o);
  torch::Tensor dL_drotations = torch::empty({P, 4}, o);
  if (P != 0) {
    if (camera_type != OMNIGS_CAMERA_LONLAT) unsupported_camera(camera_type);
    c10::cuda::CUDAGuard guard(means3D.device());
    cudaStream_t stream = at::cuda::getCurrentCUDAStream().stream();
    FloatIn bg(background), m3(means3D), shs(sh), col(colors), sc(scales), rot(rotations),
        cov(cov3D_precomp), vm(viewmatrix), cp(campos), dout(dL_dout_color);
    torch::Tensor radii_c = radii.contiguous();
    TORCH_CHECK(radii_c.scalar_type() == torch::kInt32, "omnigs_b200: radii must be int32");
    OmnigsLonlatBackwardArgs a{};
    a.P = P;
    a.D = degree;
    a.M = M;
    a.W = W;
    a.H = H;
    a.R = R;
    a.background = bg.ptr;
    a.means3D = m3.ptr;
    a.shs = shs.ptr;
    a.colors_precomp = col.ptr;
    a.scales = sc.ptr;
    a.scale_modifier = scale_modifier;
    a.rotations = rot.ptr;
    a.cov3D_precomp = cov.ptr;
    a.viewmatrix = vm.ptr;
    a.campos = cp.ptr;
    a.radii = radii_c.data_ptr<int>();
    a.dL_dout_color = dout.ptr;
    a.dL_dmeans2D = dL_dmeans2D.data_ptr<float>();
    a.dL_dcolors = dL_dcolors.data_ptr<float>();
    a.dL_dopacity = dL_dopacity.data_ptr<float>();
    a.dL_dmeans3D = dL_dmeans3D.data_ptr<float>();
    a.dL_dcov3D = dL_dcov3D.data_ptr<float>();
    a.dL_dsh = M > 0 ? dL_dsh.data_ptr<float>() : nullptr;
    a.dL_dscales = dL_dscales.data_ptr<float>();
    a.dL_drotations = dL_drotations.data_ptr<float>();
    a.dL_dconic = nullptr;
    // the forward's mode, from its image buffer: only the checkpointing layout is that small
    a.flags = imageBuffer.numel() < (int64_t)omnigs_lonlat_image_bytes(W, H) ? OMNIGS_FLAG_RECOMPUTE_T : 0;
    // The geometry buffer holds the per-splat gradient accumulators, so it is written here.
    torch::Tensor geom = geomBuffer;
    check_rc(omnigs_lonlat_backward(&a, geom.data_ptr(), geom.numel(), binningBuffer.data_ptr(),
                                    binningBuffer.numel(), imageBuffer.data_ptr(), imageBuffer.numel(),
                                    reinterpret_cast<omnigs_stream_t>(stream)),
             "backward");
  }
  return std::make_tuple(dL_dmeans2D, dL_dcolors, dL_dopacity, dL_dmeans3D, dL_dcov3D, dL_dsh, dL_dscales,
                         dL_drotations);
}

torch::Tensor markVisible(torch::Tensor& means3D, torch::Tensor& viewmatrix, torch::Tensor& projmatrix,
                          const int camera_type) {
  (void)projmatrix;
  const int P = means3D.size(0);
  torch::Tensor present = torch::full({P}, false, means3D.options().dtype(at::kBool));
  if (P != 0) {
    if (camera_type != OMNIGS_CAMERA_LONLAT && camera_type != OMNIGS_CAMERA_PINHOLE)
      throw std::runtime_error("[CudaRasterizer]Invalid camera_type");
    c10::cuda::CUDAGuard guard(means3D.device());
    FloatIn m3(means3D), vm(viewmatrix);
    check_rc(omnigs_mark_visible(P, m3.ptr, vm.ptr, camera_type,
                                 reinterpret_cast<uint8_t*>(present.data_ptr<bool>()),
                                 reinterpret_cast<omnigs_stream_t>(at::cuda::getCurrentCUDAStream().stream())),
             "markVisible");
  }
  return present;
}
