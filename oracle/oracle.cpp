// TEST INFRASTRUCTURE ONLY -- the FP64 oracle.
//
// A multithreaded FP64 CPU restatement of OmniGS's equirectangular ("lonlat", camera_type = 3)
// differentiable Gaussian tile rasterizer.  It is the checker for the CUDA path and the timed CPU
// baseline; the product never links, loads or calls it.  Every stage follows the reference's
// control flow, thresholds and epsilons, in double precision:
//
//   preprocess      cuda_rasterizer/forward.cu:592-703 (+ computeCov3D :194-228,
//                   computeCov2DLonlat :130-189, computeColorFromSH :30-83, auxiliary.h:198-248)
//   binning         cuda_rasterizer/rasterizer_impl.cu:94-167, 622-679 (inclusive scan,
//                   duplicateWithKeys, stable radix sort over bits [0, 32 + getHigherMsb(tiles)),
//                   identifyTileRanges)
//   forward blend   cuda_rasterizer/forward.cu:346-467
//   backward blend  cuda_rasterizer/backward.cu:672-843
//   bwd preprocess  cuda_rasterizer/backward.cu:297-485 (computeCov2DLonLatCUDA), :613-669
//                   (preprocessLonLatCUDA), :30-151 (SH), :489-552 (computeCov3D)
//
// Constants that the reference writes as float literals (0.04f, 1e-7f, 0.3f, 0.1f, 0.99f,
// 1/255, 1e-4) are used at their float values so the thresholds are the reference's thresholds.
// The glm expressions of the reference are restated with a small column-major double matrix type
// (DMat3 below) so each formula can be read against its source line.
//
// Parity pin: checked stage by stage against the reference CUDA rasterizer itself (rebuilt from its
// own sources for sm_100a by oracle/ref/Makefile and run on a B200), each stage fed with the
// reference's float intermediates: tests/test_oracle_vs_reference_gpu.py.

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <numeric>
#include <thread>
#include <vector>

namespace {

constexpr double kNearR2 = (double)0.04f;              // auxiliary.h:208
constexpr double kEps = (double)0.0000001f;            // auxiliary.h:238, forward.cu:148-152
constexpr double kLowPass = (double)0.3f;              // forward.cu:185-186
constexpr double kEigFloor = (double)0.1f;             // forward.cu:672
constexpr double kAlphaMax = (double)0.99f;            // forward.cu:436
constexpr double kAlphaMin = (double)(1.0f / 255.0f);  // forward.cu:437
constexpr double kTMin = (double)0.0001f;              // forward.cu:440
constexpr int kTile = 16;                              // config.h:26-27

const double SH_C0 = 0.28209479177387814;              // auxiliary.h:32-49
const double SH_C1 = 0.4886025119029199;
const double SH_C2[5] = {1.0925484305920792, -1.0925484305920792, 0.31539156525252005,
                         -1.0925484305920792, 0.5462742152960396};
const double SH_C3[7] = {-0.5900435899266435, 2.890611442640554, -0.4570457994644658,
                         0.3731763325901154, -0.4570457994644658, 1.445305721320277,
                         -0.5900435899266435};

struct D3 {
  double x, y, z;
};
inline D3 operator+(D3 a, D3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline D3 operator-(D3 a, D3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline D3 operator*(double s, D3 a) { return {s * a.x, s * a.y, s * a.z}; }
inline double dot(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

// Column-major 3x3 matrix with glm's indexing: m[col][row].
struct DMat3 {
  double m[3][3];
};
inline DMat3 mat_cols(double a0, double a1, double a2, double a3, double a4, double a5, double a6,
                      double a7, double a8) {
  DMat3 r;
  r.m[0][0] = a0; r.m[0][1] = a1; r.m[0][2] = a2;
  r.m[1][0] = a3; r.m[1][1] = a4; r.m[1][2] = a5;
  r.m[2][0] = a6; r.m[2][1] = a7; r.m[2][2] = a8;
  return r;
}
inline DMat3 mul(const DMat3& a, const DMat3& b) {
  DMat3 r;
  for (int c = 0; c < 3; ++c)
    for (int row = 0; row < 3; ++row)
      r.m[c][row] = a.m[0][row] * b.m[c][0] + a.m[1][row] * b.m[c][1] + a.m[2][row] * b.m[c][2];
  return r;
}
inline DMat3 transpose(const DMat3& a) {
  DMat3 r;
  for (int c = 0; c < 3; ++c)
    for (int row = 0; row < 3; ++row) r.m[c][row] = a.m[row][c];
  return r;
}

// transformPoint4x3 / transformVec4x3Transpose, auxiliary.h:85-124 (matrix = Tcw column-major).
inline D3 xform_point(const float* m, D3 p) {
  return {m[0] * p.x + m[4] * p.y + m[8] * p.z + m[12], m[1] * p.x + m[5] * p.y + m[9] * p.z + m[13],
          m[2] * p.x + m[6] * p.y + m[10] * p.z + m[14]};
}
inline D3 xform_vec_T(const float* m, D3 p) {
  return {m[0] * p.x + m[1] * p.y + m[2] * p.z, m[4] * p.x + m[5] * p.y + m[6] * p.z,
          m[8] * p.x + m[9] * p.y + m[10] * p.z};
}
inline DMat3 view_rot_glm(const float* v) {  // forward.cu:169-172
  return mat_cols(v[0], v[4], v[8], v[1], v[5], v[9], v[2], v[6], v[10]);
}

template <class F>
void parallel_for(int64_t n, int nthreads, F&& f) {
  if (n <= 0) return;
  if (nthreads <= 1 || n < 64) {
    for (int64_t i = 0; i < n; ++i) f(i);
    return;
  }
  std::atomic<int64_t> next{0};
  const int64_t chunk = std::max<int64_t>(1, n / ((int64_t)nthreads * 32));
  std::vector<std::thread> pool;
  for (int t = 0; t < nthreads; ++t)
    pool.emplace_back([&] {
      for (;;) {
        int64_t s = next.fetch_add(chunk);
        if (s >= n) break;
        int64_t e = std::min(n, s + chunk);
        for (int64_t i = s; i < e; ++i) f(i);
      }
    });
  for (auto& th : pool) th.join();
}

// CUDA's float->int conversion in device code (cvt.rzi.s32): truncate, saturate, NaN -> 0.
inline int to_int_sat(double v) {
  if (std::isnan(v)) return 0;
  if (v >= 2147483647.0) return 2147483647;
  if (v <= -2147483648.0) return (int)-2147483648LL;
  return (int)v;
}

// getRect, auxiliary.h:56-66 (the lonlat path clamps; getRectCyclic is not called, forward.cu:680).
template <class T>
inline void get_rect(T px, T py, int max_radius, int gx, int gy, int rmin[2], int rmax[2]) {
  const T r = (T)max_radius;
  const T b = (T)kTile;
  rmin[0] = std::min(gx, std::max(0, to_int_sat((double)((px - r) / b))));
  rmin[1] = std::min(gy, std::max(0, to_int_sat((double)((py - r) / b))));
  rmax[0] = std::min(gx, std::max(0, to_int_sat((double)((px + r + b - (T)1) / b))));
  rmax[1] = std::min(gy, std::max(0, to_int_sat((double)((py + r + b - (T)1) / b))));
}

// Seam-wrapping mode (an extension beyond the reference's lonlat path, which clamps): the tile
// column range of getRectCyclic (auxiliary.h:68-83: x may start at -gx and end at 2 gx, columns
// outside [0, gx) wrap modulo gx), with two choices of this package stated here as the mode's
// semantics: the left edge is floor((x - r) / 16) rather than the truncation towards zero, so a
// splat reaching less than one tile past x = 0 still gets the wrapped column, and the range is
// capped at one image width (gx columns), so no tile holds a splat twice.  Rows clamp as getRect.
template <class T>
inline void get_rect_cyclic(T px, T py, int max_radius, int gx, int gy, int rmin[2], int rmax[2]) {
  const T r = (T)max_radius;
  const T b = (T)kTile;
  rmin[0] = std::min(gx, std::max(-gx, to_int_sat(std::floor((double)((px - r) / b)))));
  rmin[1] = std::min(gy, std::max(0, to_int_sat((double)((py - r) / b))));
  rmax[0] = std::min(2 * gx, std::max(0, to_int_sat((double)((px + r + b - (T)1) / b))));
  rmax[1] = std::min(gy, std::max(0, to_int_sat((double)((py + r + b - (T)1) / b))));
  if (rmax[0] < rmin[0]) rmax[0] = rmin[0];
  if (rmax[0] - rmin[0] > gx) rmax[0] = rmin[0] + gx;
}

template <class T>
inline void tile_rect(bool seam_wrap, T px, T py, int max_radius, int gx, int gy, int rmin[2], int rmax[2]) {
  if (seam_wrap)
    get_rect_cyclic<T>(px, py, max_radius, gx, gy, rmin, rmax);
  else
    get_rect<T>(px, py, max_radius, gx, gy, rmin, rmax);
}

// x offset of a splat centre from a pixel column: the plain difference (the reference), or in
// seam-wrapping mode the difference to the centre's copy (shifted by a multiple of the image
// width) nearest the centre of the pixel's block of 8 columns (columns 8k .. 8k + 7, centre
// 8k + 3.5).  The mode defines the copy per 8-column block, not per pixel: a splat wider than
// half the image reaches a block's pixels from one copy only, the one nearest the block.
inline double seam_dx(bool seam_wrap, double mx, double px, int W) {
  if (seam_wrap) {
    const double block_centre = std::floor(px / 8.0) * 8.0 + 3.5;
    mx -= W * std::nearbyint((mx - block_centre) / W);
  }
  return mx - px;
}

// getHigherMsb, rasterizer_impl.cu:47-62.
uint32_t higher_msb(uint32_t n) {
  uint32_t msb = sizeof(n) * 4;
  uint32_t step = msb;
  while (step > 1) {
    step /= 2;
    if (n >> msb)
      msb += step;
    else
      msb -= step;
  }
  if (n >> msb) msb++;
  return msb;
}

// computeCov3D, forward.cu:194-228 (quaternion (r, x, y, z) is not normalised).
void cov3d(const float* s, double mod, const float* q, double out[6]) {
  DMat3 S = mat_cols(1, 0, 0, 0, 1, 0, 0, 0, 1);
  S.m[0][0] = mod * s[0];
  S.m[1][1] = mod * s[1];
  S.m[2][2] = mod * s[2];
  const double r = q[0], x = q[1], y = q[2], z = q[3];
  DMat3 R = mat_cols(1. - 2. * (y * y + z * z), 2. * (x * y - r * z), 2. * (x * z + r * y),
                     2. * (x * y + r * z), 1. - 2. * (x * x + z * z), 2. * (y * z - r * x),
                     2. * (x * z - r * y), 2. * (y * z + r * x), 1. - 2. * (x * x + y * y));
  DMat3 M = mul(S, R);
  DMat3 Sig = mul(transpose(M), M);
  out[0] = Sig.m[0][0]; out[1] = Sig.m[0][1]; out[2] = Sig.m[0][2];
  out[3] = Sig.m[1][1]; out[4] = Sig.m[1][2]; out[5] = Sig.m[2][2];
}

struct LonlatJac {
  double dpx_dtx, dpx_dtz, dpy_dtx, dpy_dty, dpy_dtz;
};

// The lonlat Jacobian of (px, py) w.r.t. the camera-space mean, forward.cu:147-162.
LonlatJac lonlat_jacobian(D3 t, int width, int height) {
  const double trxztrxz = t.x * t.x + t.z * t.z;
  const double trxztrxz_inv = 1.0 / (trxztrxz + kEps);
  const double trxz = std::sqrt(trxztrxz);
  const double trxz_inv = 1.0 / (trxz + kEps);
  const double trtr = trxztrxz + t.y * t.y;
  const double trtr_inv = 1.0 / (trtr + kEps);
  const double W_div_2pi = width * 0.5 / M_PI;
  const double H_div_pi = height / M_PI;
  LonlatJac j;
  j.dpx_dtx = W_div_2pi * t.z * trxztrxz_inv;
  j.dpx_dtz = -W_div_2pi * t.x * trxztrxz_inv;
  j.dpy_dtx = -H_div_pi * t.x * t.y * trxz_inv * trtr_inv;
  j.dpy_dty = H_div_pi * trxz * trtr_inv;
  j.dpy_dtz = -H_div_pi * t.z * t.y * trxz_inv * trtr_inv;
  return j;
}

// computeCov2DLonlat, forward.cu:130-189: cov = T^T Vrk^T T with T = W J, plus the 0.3 low-pass.
void cov2d_lonlat(D3 mean, int width, int height, const double* c3, const float* view, double out[3],
                  DMat3* T_out = nullptr) {
  const D3 t = xform_point(view, mean);
  const LonlatJac j = lonlat_jacobian(t, width, height);
  DMat3 J = mat_cols(j.dpx_dtx, 0.0, j.dpx_dtz, j.dpy_dtx, j.dpy_dty, j.dpy_dtz, 0.0, 0.0, 0.0);
  DMat3 W = view_rot_glm(view);
  DMat3 T = mul(W, J);
  DMat3 Vrk = mat_cols(c3[0], c3[1], c3[2], c3[1], c3[3], c3[4], c3[2], c3[4], c3[5]);
  DMat3 cov = mul(mul(transpose(T), transpose(Vrk)), T);
  cov.m[0][0] += kLowPass;
  cov.m[1][1] += kLowPass;
  out[0] = cov.m[0][0];
  out[1] = cov.m[0][1];
  out[2] = cov.m[1][1];
  if (T_out) *T_out = T;
}

// computeColorFromSH, forward.cu:30-83.  Returns the clamped colour and the clamp flags.
D3 sh_to_rgb(int deg, int max_coeffs, D3 pos, D3 campos, const float* shs_g, uint8_t clamped[3]) {
  D3 dir = pos - campos;
  const double len = std::sqrt(dot(dir, dir));
  dir = {dir.x / len, dir.y / len, dir.z / len};
  auto sh = [&](int k) { return D3{shs_g[3 * k], shs_g[3 * k + 1], shs_g[3 * k + 2]}; };
  (void)max_coeffs;
  D3 result = SH_C0 * sh(0);
  if (deg > 0) {
    const double x = dir.x, y = dir.y, z = dir.z;
    result = result - (SH_C1 * y) * sh(1) + (SH_C1 * z) * sh(2) - (SH_C1 * x) * sh(3);
    if (deg > 1) {
      const double xx = x * x, yy = y * y, zz = z * z, xy = x * y, yz = y * z, xz = x * z;
      result = result + (SH_C2[0] * xy) * sh(4) + (SH_C2[1] * yz) * sh(5) +
               (SH_C2[2] * (2.0 * zz - xx - yy)) * sh(6) + (SH_C2[3] * xz) * sh(7) +
               (SH_C2[4] * (xx - yy)) * sh(8);
      if (deg > 2) {
        result = result + (SH_C3[0] * y * (3.0 * xx - yy)) * sh(9) + (SH_C3[1] * xy * z) * sh(10) +
                 (SH_C3[2] * y * (4.0 * zz - xx - yy)) * sh(11) +
                 (SH_C3[3] * z * (2.0 * zz - 3.0 * xx - 3.0 * yy)) * sh(12) +
                 (SH_C3[4] * x * (4.0 * zz - xx - yy)) * sh(13) + (SH_C3[5] * z * (xx - yy)) * sh(14) +
                 (SH_C3[6] * x * (xx - 3.0 * yy)) * sh(15);
      }
    }
  }
  result = {result.x + 0.5, result.y + 0.5, result.z + 0.5};
  clamped[0] = result.x < 0;
  clamped[1] = result.y < 0;
  clamped[2] = result.z < 0;
  return {std::max(result.x, 0.0), std::max(result.y, 0.0), std::max(result.z, 0.0)};
}

}  // namespace

extern "C" {

int oracle_abi_version() { return 1; }

uint32_t oracle_higher_msb(uint32_t n) { return higher_msb(n); }

// Forward preprocess (forward.cu:592-703) in FP64.  Outputs: radii [P] (0 = culled), tiles_touched
// [P], means2D [P,2] (pixels), depths [P] (radial distance r, forward.cu:697), conic_opacity [P,4],
// rgb [P,3], clamped [P,3], cov3D [P,6].
// seam_wrap selects the cyclic tile rect of the seam-wrapping mode (get_rect_cyclic).
void oracle_preprocess_seam(int P, int D, int M, int W, int H, const float* means3D, const float* scales,
                            float scale_modifier, const float* rotations, const float* opacities,
                            const float* shs, const float* colors_precomp, const float* cov3D_precomp,
                            const float* viewmatrix, const float* campos, int* radii,
                            uint32_t* tiles_touched, double* means2D, double* depths,
                            double* conic_opacity, double* rgb, uint8_t* clamped, double* cov3D_out,
                            int seam_wrap, int nthreads) {
  const int gx = (W + kTile - 1) / kTile, gy = (H + kTile - 1) / kTile;
  const D3 cam = {campos[0], campos[1], campos[2]};
  parallel_for(P, nthreads, [&](int64_t i) {
    radii[i] = 0;
    tiles_touched[i] = 0;
    const D3 p = {means3D[3 * i], means3D[3 * i + 1], means3D[3 * i + 2]};
    const D3 t = xform_point(viewmatrix, p);  // too_close, auxiliary.h:198-220
    const double rr = t.x * t.x + t.y * t.y + t.z * t.z;
    if (rr <= kNearR2) return;
    const double r = std::sqrt(rr);
    const double inv_r = 1.0 / (r + kEps);  // point3ToLonlatScreen, auxiliary.h:236-248
    const double lon = std::atan2(t.x, t.z);
    const double lat = std::asin(t.y * inv_r);
    const double sx = lon / M_PI, sy = lat * 2.0 / M_PI;
    double c3[6];
    if (cov3D_precomp)
      for (int k = 0; k < 6; ++k) c3[k] = cov3D_precomp[6 * i + k];
    else
      cov3d(scales + 3 * i, scale_modifier, rotations + 4 * i, c3);
    for (int k = 0; k < 6; ++k) cov3D_out[6 * i + k] = c3[k];
    double cov[3];
    cov2d_lonlat(p, W, H, c3, viewmatrix, cov);
    const double det = cov[0] * cov[2] - cov[1] * cov[1];
    if (det == 0.0) return;
    const double det_inv = 1.0 / det;
    const double conic[3] = {cov[2] * det_inv, -cov[1] * det_inv, cov[0] * det_inv};
    const double mid = 0.5 * (cov[0] + cov[2]);
    const double l1 = mid + std::sqrt(std::max(kEigFloor, mid * mid - det));
    const double l2 = mid - std::sqrt(std::max(kEigFloor, mid * mid - det));
    const double my_radius = std::ceil(3.0 * std::sqrt(std::max(l1, l2)));
    const double px = ((sx + 1.0) * W - 1.0) * 0.5;  // ndc2Pix, auxiliary.h:51-54
    const double py = ((sy + 1.0) * H - 1.0) * 0.5;
    const int ir = to_int_sat(my_radius);
    int rmin[2], rmax[2];
    tile_rect<double>(seam_wrap != 0, px, py, ir, gx, gy, rmin, rmax);
    const int64_t area = (int64_t)(rmax[0] - rmin[0]) * (rmax[1] - rmin[1]);
    if (area == 0) return;
    if (colors_precomp == nullptr) {
      uint8_t cl[3];
      D3 c = sh_to_rgb(D, M, p, cam, shs + (int64_t)i * M * 3, cl);
      rgb[3 * i] = c.x; rgb[3 * i + 1] = c.y; rgb[3 * i + 2] = c.z;
      for (int k = 0; k < 3; ++k) clamped[3 * i + k] = cl[k];
    } else {
      for (int k = 0; k < 3; ++k) {
        rgb[3 * i + k] = colors_precomp[3 * i + k];
        clamped[3 * i + k] = 0;
      }
    }
    depths[i] = r;
    radii[i] = ir;
    means2D[2 * i] = px;
    means2D[2 * i + 1] = py;
    conic_opacity[4 * i] = conic[0];
    conic_opacity[4 * i + 1] = conic[1];
    conic_opacity[4 * i + 2] = conic[2];
    conic_opacity[4 * i + 3] = opacities[i];
    tiles_touched[i] = (uint32_t)area;
  });
}

void oracle_preprocess(int P, int D, int M, int W, int H, const float* means3D, const float* scales,
                       float scale_modifier, const float* rotations, const float* opacities,
                       const float* shs, const float* colors_precomp, const float* cov3D_precomp,
                       const float* viewmatrix, const float* campos, int* radii,
                       uint32_t* tiles_touched, double* means2D, double* depths,
                       double* conic_opacity, double* rgb, uint8_t* clamped, double* cov3D_out,
                       int nthreads) {
  oracle_preprocess_seam(P, D, M, W, H, means3D, scales, scale_modifier, rotations, opacities, shs,
                         colors_precomp, cov3D_precomp, viewmatrix, campos, radii, tiles_touched, means2D,
                         depths, conic_opacity, rgb, clamped, cov3D_out, 0, nthreads);
}

// Total instances = inclusive scan's last element (rasterizer_impl.cu:622-628).
int64_t oracle_num_rendered(int P, const uint32_t* tiles_touched) {
  int64_t s = 0;
  for (int i = 0; i < P; ++i) s += tiles_touched[i];
  return s;
}

}  // extern "C"

namespace {
template <class T>
void binning_impl(int P, int W, int H, const int* radii, const T* means2D, const float* depth32,
                  const uint32_t* tiles_touched, uint64_t* keys_out, uint32_t* vals_out,
                  uint32_t* ranges, bool seam_wrap, int row_lo = 0, int row_hi = 1 << 30) {
  const int gx = (W + kTile - 1) / kTile, gy = (H + kTile - 1) / kTile;
  const int64_t tiles = (int64_t)gx * gy;
  std::vector<uint64_t> offs(P + 1, 0);
  for (int i = 0; i < P; ++i) offs[i + 1] = offs[i] + tiles_touched[i];
  const int64_t R = (int64_t)offs[P];
  std::vector<uint64_t> keys(R);
  std::vector<uint32_t> vals(R);
  // duplicateWithKeys, rasterizer_impl.cu:94-140 (unsorted order: by Gaussian, then row, column)
  for (int i = 0; i < P; ++i) {
    if (!(radii[i] > 0)) continue;
    int rmin[2], rmax[2];
    tile_rect<T>(seam_wrap, means2D[2 * i], means2D[2 * i + 1], radii[i], gx, gy, rmin, rmax);
    uint64_t off = offs[i];
    uint32_t dbits;
    std::memcpy(&dbits, &depth32[i], 4);
    for (int y = std::max(rmin[1], row_lo); y < std::min(rmax[1], row_hi); ++y)
      for (int x = rmin[0]; x < rmax[0]; ++x) {
        const int col = ((x % gx) + gx) % gx;  // x itself unless the seam wraps
        uint64_t key = (uint32_t)(y * gx + col);
        key <<= 32;
        key |= dbits;
        keys[off] = key;
        vals[off] = (uint32_t)i;
        off++;
      }
  }
  // Stable ascending sort by key over bits [0, 32 + getHigherMsb(tiles)) (rasterizer_impl.cu:651-661).
  // Tile ids are < 2^bit, so no key bit lies outside the sorted range and the result is the
  // unique stable order: by key, ties in unsorted order.
  const uint32_t bit = higher_msb((uint32_t)tiles);
  const uint64_t mask = (32 + bit >= 64) ? ~0ull : ((1ull << (32 + bit)) - 1);
  std::vector<uint32_t> order(R);
  std::iota(order.begin(), order.end(), 0u);
  std::sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) {
    const uint64_t ka = keys[a] & mask, kb = keys[b] & mask;
    return ka < kb || (ka == kb && a < b);
  });
  for (int64_t s = 0; s < R; ++s) {
    keys_out[s] = keys[order[s]];
    vals_out[s] = vals[order[s]];
  }
  // identifyTileRanges, rasterizer_impl.cu:145-167, after the zeroing memset at :664.
  std::fill(ranges, ranges + 2 * tiles, 0u);
  for (int64_t s = 0; s < R; ++s) {
    const uint32_t cur = (uint32_t)(keys_out[s] >> 32);
    if (s == 0)
      ranges[2 * cur] = 0;
    else {
      const uint32_t prev = (uint32_t)(keys_out[s - 1] >> 32);
      if (cur != prev) {
        ranges[2 * prev + 1] = (uint32_t)s;
        ranges[2 * cur] = (uint32_t)s;
      }
    }
    if (s == R - 1) ranges[2 * cur + 1] = (uint32_t)R;
  }
}
}  // namespace

extern "C" {

// Binning from FP32 preprocess outputs (means2D float [P,2], depths float [P]) with the getRect
// arithmetic in float, i.e. exactly what the reference computes from the same inputs.
void oracle_binning_f32(int P, int W, int H, const int* radii, const float* means2D,
                        const float* depths, const uint32_t* tiles_touched, uint64_t* keys,
                        uint32_t* vals, uint32_t* ranges) {
  binning_impl<float>(P, W, H, radii, means2D, depths, tiles_touched, keys, vals, ranges, false);
}

// Tiles touched per Gaussian from its float rect (clamped, or cyclic when seam_wrap != 0): the
// preprocess's tiles_touched for callers that hold only radii and means2D.
void oracle_tiles_touched_f32(int P, int W, int H, const int* radii, const float* means2D, int seam_wrap,
                              uint32_t* tiles_touched) {
  const int gx = (W + kTile - 1) / kTile, gy = (H + kTile - 1) / kTile;
  for (int i = 0; i < P; ++i) {
    tiles_touched[i] = 0;
    if (!(radii[i] > 0)) continue;
    int rmin[2], rmax[2];
    tile_rect<float>(seam_wrap != 0, means2D[2 * i], means2D[2 * i + 1], radii[i], gx, gy, rmin, rmax);
    tiles_touched[i] = (uint32_t)((rmax[0] - rmin[0]) * (rmax[1] - rmin[1]));
  }
}

// The same with the seam-wrapping mode's cyclic rects (seam_wrap != 0).
void oracle_binning_f32_seam(int P, int W, int H, const int* radii, const float* means2D,
                             const float* depths, const uint32_t* tiles_touched, uint64_t* keys,
                             uint32_t* vals, uint32_t* ranges, int seam_wrap) {
  binning_impl<float>(P, W, H, radii, means2D, depths, tiles_touched, keys, vals, ranges, seam_wrap != 0);
}

// Binning from the FP64 preprocess (rects in double; the key's depth bits are float(r)),
// seam_wrap != 0 for the seam-wrapping mode's cyclic rects.
void oracle_binning_f64_seam(int P, int W, int H, const int* radii, const double* means2D,
                             const double* depths, const uint32_t* tiles_touched, uint64_t* keys,
                             uint32_t* vals, uint32_t* ranges, int seam_wrap) {
  std::vector<float> d32(P);
  for (int i = 0; i < P; ++i) d32[i] = (float)depths[i];
  binning_impl<double>(P, W, H, radii, means2D, d32.data(), tiles_touched, keys, vals, ranges, seam_wrap != 0);
}

void oracle_binning_f64(int P, int W, int H, const int* radii, const double* means2D,
                        const double* depths, const uint32_t* tiles_touched, uint64_t* keys,
                        uint32_t* vals, uint32_t* ranges) {
  oracle_binning_f64_seam(P, W, H, radii, means2D, depths, tiles_touched, keys, vals, ranges, 0);
}

// Per-Gaussian instance counts restricted to tile rows [row_lo, row_hi) of the FP64 rects (for
// oracle_binning_f64_rows).
void oracle_tiles_in_rows_f64(int P, int W, int H, const int* radii, const double* means2D, int row_lo, int row_hi,
                              uint32_t* counts) {
  const int gx = (W + kTile - 1) / kTile, gy = (H + kTile - 1) / kTile;
  for (int i = 0; i < P; ++i) {
    counts[i] = 0;
    if (!(radii[i] > 0)) continue;
    int rmin[2], rmax[2];
    get_rect<double>(means2D[2 * i], means2D[2 * i + 1], radii[i], gx, gy, rmin, rmax);
    const int rows = std::min(rmax[1], row_hi) - std::max(rmin[1], row_lo);
    if (rows > 0) counts[i] = (uint32_t)(rows * (rmax[0] - rmin[0]));
  }
}

// Binning of the FP64 pipeline restricted to tile rows [row_lo, row_hi): the instances, sorted
// list and ranges of those rows exactly as the full binning has them (other tiles stay empty),
// for checking rows of a scene too large to bin whole on the CPU.  counts from
// oracle_tiles_in_rows_f64.
void oracle_binning_f64_rows(int P, int W, int H, const int* radii, const double* means2D, const double* depths,
                             const uint32_t* counts, int row_lo, int row_hi, uint64_t* keys, uint32_t* vals,
                             uint32_t* ranges) {
  std::vector<float> d32(P);
  for (int i = 0; i < P; ++i) d32[i] = (float)depths[i];
  binning_impl<double>(P, W, H, radii, means2D, d32.data(), counts, keys, vals, ranges, false, row_lo, row_hi);
}

// Forward blend, forward.cu:346-467.  out_color [3,H,W], final_T [H*W], n_contrib [H*W].
// seam_wrap != 0: x offsets to the splat's copy nearest the pixel's 8-column block (seam_dx).
void oracle_render_forward_seam(int W, int H, const uint32_t* ranges, const uint32_t* point_list,
                                const double* means2D, const double* conic_opacity, const double* rgb,
                                const float* bg, double* out_color, double* final_T,
                                uint32_t* n_contrib, int seam_wrap, int nthreads) {
  const int gx = (W + kTile - 1) / kTile, gy = (H + kTile - 1) / kTile;
  parallel_for((int64_t)gx * gy, nthreads, [&](int64_t tile) {
    const int tx = (int)(tile % gx), ty = (int)(tile / gx);
    const uint32_t r0 = ranges[2 * tile], r1 = ranges[2 * tile + 1];
    for (int py = ty * kTile; py < std::min(H, (ty + 1) * kTile); ++py)
      for (int px = tx * kTile; px < std::min(W, (tx + 1) * kTile); ++px) {
        double T = 1.0, C[3] = {0, 0, 0};
        uint32_t contributor = 0, last = 0;
        for (uint32_t s = r0; s < r1; ++s) {
          contributor++;
          const uint32_t g = point_list[s];
          const double dx = seam_dx(seam_wrap != 0, means2D[2 * g], px, W), dy = means2D[2 * g + 1] - py;
          const double* co = conic_opacity + 4 * (int64_t)g;
          const double power = -0.5 * (co[0] * dx * dx + co[2] * dy * dy) - co[1] * dx * dy;
          if (power > 0.0) continue;
          const double alpha = std::min(kAlphaMax, co[3] * std::exp(power));
          if (alpha < kAlphaMin) continue;
          const double test_T = T * (1 - alpha);
          if (test_T < kTMin) break;  // done: this Gaussian is not blended
          for (int ch = 0; ch < 3; ++ch) C[ch] += rgb[3 * (int64_t)g + ch] * alpha * T;
          T = test_T;
          last = contributor;
        }
        const int64_t pix = (int64_t)py * W + px;
        final_T[pix] = T;
        n_contrib[pix] = last;
        for (int ch = 0; ch < 3; ++ch) out_color[(int64_t)ch * H * W + pix] = C[ch] + T * bg[ch];
      }
  });
}

void oracle_render_forward(int W, int H, const uint32_t* ranges, const uint32_t* point_list,
                           const double* means2D, const double* conic_opacity, const double* rgb,
                           const float* bg, double* out_color, double* final_T,
                           uint32_t* n_contrib, int nthreads) {
  oracle_render_forward_seam(W, H, ranges, point_list, means2D, conic_opacity, rgb, bg, out_color, final_T,
                             n_contrib, 0, nthreads);
}

// Backward blend, backward.cu:672-843.  Gradients are accumulated per sorted instance (each
// instance belongs to one tile, so tiles run in parallel without races) and then summed per
// Gaussian in instance order, which makes the oracle deterministic.
// Outputs (zeroed here): dL_dmean2D [P,3], dL_dconic [P,4] (x, y, -, w), dL_dopacity [P],
// dL_dcolor [P,3].
// seam_wrap != 0: x offsets to the splat's copy nearest the pixel's 8-column block (seam_dx); the offset's
// derivative with respect to the centre is 1 for every copy, so the formulas are unchanged.
void oracle_render_backward_seam(int P, int W, int H, const uint32_t* ranges, const uint32_t* point_list,
                                 int64_t R, const double* means2D, const double* conic_opacity,
                                 const double* rgb, const float* bg, const double* final_T,
                                 const uint32_t* n_contrib, const float* dL_dpix, double* dL_dmean2D,
                                 double* dL_dconic, double* dL_dopacity, double* dL_dcolor,
                                 int seam_wrap, int nthreads) {
  const int gx = (W + kTile - 1) / kTile, gy = (H + kTile - 1) / kTile;
  std::vector<double> inst((size_t)R * 9, 0.0);
  const double ddelx_dx = 0.5 * W, ddely_dy = 0.5 * H;
  parallel_for((int64_t)gx * gy, nthreads, [&](int64_t tile) {
    const int tx = (int)(tile % gx), ty = (int)(tile / gx);
    const uint32_t r0 = ranges[2 * tile];
    for (int py = ty * kTile; py < std::min(H, (ty + 1) * kTile); ++py)
      for (int px = tx * kTile; px < std::min(W, (tx + 1) * kTile); ++px) {
        const int64_t pix = (int64_t)py * W + px;
        const double T_final = final_T[pix];
        double T = T_final;
        const uint32_t last = n_contrib[pix];
        double dpix[3], accum[3] = {0, 0, 0}, last_color[3] = {0, 0, 0}, last_alpha = 0;
        for (int ch = 0; ch < 3; ++ch) dpix[ch] = dL_dpix[(int64_t)ch * H * W + pix];
        const double bg_dot = bg[0] * dpix[0] + bg[1] * dpix[1] + bg[2] * dpix[2];
        for (int64_t k = (int64_t)last - 1; k >= 0; --k) {
          const uint32_t s = r0 + (uint32_t)k;
          const uint32_t g = point_list[s];
          const double dx = seam_dx(seam_wrap != 0, means2D[2 * g], px, W), dy = means2D[2 * g + 1] - py;
          const double* co = conic_opacity + 4 * (int64_t)g;
          const double power = -0.5 * (co[0] * dx * dx + co[2] * dy * dy) - co[1] * dx * dy;
          if (power > 0.0) continue;
          const double G = std::exp(power);
          const double alpha = std::min(kAlphaMax, co[3] * G);
          if (alpha < kAlphaMin) continue;
          T = T / (1.0 - alpha);
          const double dchannel_dcolor = alpha * T;
          double* acc = &inst[(size_t)s * 9];
          double dL_dalpha = 0.0;
          for (int ch = 0; ch < 3; ++ch) {
            const double c = rgb[3 * (int64_t)g + ch];
            accum[ch] = last_alpha * last_color[ch] + (1.0 - last_alpha) * accum[ch];
            last_color[ch] = c;
            dL_dalpha += (c - accum[ch]) * dpix[ch];
            acc[6 + ch] += dchannel_dcolor * dpix[ch];
          }
          dL_dalpha *= T;
          last_alpha = alpha;
          dL_dalpha += (-T_final / (1.0 - alpha)) * bg_dot;
          const double dL_dG = co[3] * dL_dalpha;
          const double gdx = G * dx, gdy = G * dy;
          const double dG_ddelx = -gdx * co[0] - gdy * co[1];
          const double dG_ddely = -gdy * co[2] - gdx * co[1];
          acc[0] += dL_dG * dG_ddelx * ddelx_dx;
          acc[1] += dL_dG * dG_ddely * ddely_dy;
          acc[2] += -0.5 * gdx * dx * dL_dG;
          acc[3] += -0.5 * gdx * dy * dL_dG;
          acc[4] += -0.5 * gdy * dy * dL_dG;
          acc[5] += G * dL_dalpha;
        }
      }
  });
  std::fill(dL_dmean2D, dL_dmean2D + 3 * (int64_t)P, 0.0);
  std::fill(dL_dconic, dL_dconic + 4 * (int64_t)P, 0.0);
  std::fill(dL_dopacity, dL_dopacity + P, 0.0);
  std::fill(dL_dcolor, dL_dcolor + 3 * (int64_t)P, 0.0);
  for (int64_t s = 0; s < R; ++s) {
    const uint32_t g = point_list[s];
    const double* a = &inst[(size_t)s * 9];
    dL_dmean2D[3 * (int64_t)g] += a[0];
    dL_dmean2D[3 * (int64_t)g + 1] += a[1];
    dL_dconic[4 * (int64_t)g] += a[2];
    dL_dconic[4 * (int64_t)g + 1] += a[3];
    dL_dconic[4 * (int64_t)g + 3] += a[4];
    dL_dopacity[g] += a[5];
    for (int ch = 0; ch < 3; ++ch) dL_dcolor[3 * (int64_t)g + ch] += a[6 + ch];
  }
}

void oracle_render_backward(int P, int W, int H, const uint32_t* ranges, const uint32_t* point_list,
                            int64_t R, const double* means2D, const double* conic_opacity,
                            const double* rgb, const float* bg, const double* final_T,
                            const uint32_t* n_contrib, const float* dL_dpix, double* dL_dmean2D,
                            double* dL_dconic, double* dL_dopacity, double* dL_dcolor,
                            int nthreads) {
  oracle_render_backward_seam(P, W, H, ranges, point_list, R, means2D, conic_opacity, rgb, bg, final_T, n_contrib,
                              dL_dpix, dL_dmean2D, dL_dconic, dL_dopacity, dL_dcolor, 0, nthreads);
}

// Backward preprocess: computeCov2DLonLatCUDA (backward.cu:297-485) + preprocessLonLatCUDA
// (:613-669) with its SH (:30-151) and cov3D (:489-552) parts.  All outputs are written for every
// Gaussian (zero where radii <= 0).  dL_dsh may be null when M == 0.
void oracle_preprocess_backward(int P, int D, int M, int W, int H, const float* means3D,
                                const int* radii, const float* shs, const uint8_t* clamped,
                                const float* scales, float scale_modifier, const float* rotations,
                                const float* cov3D_precomp, const float* viewmatrix,
                                const float* campos, const double* dL_dmean2D,
                                const double* dL_dconic, const double* dL_dcolor,
                                double* dL_dmeans3D, double* dL_dcov3D, double* dL_dsh,
                                double* dL_dscales, double* dL_drots, int nthreads) {
  const D3 cam = {campos[0], campos[1], campos[2]};
  parallel_for(P, nthreads, [&](int64_t i) {
    for (int k = 0; k < 3; ++k) dL_dmeans3D[3 * i + k] = 0;
    for (int k = 0; k < 6; ++k) dL_dcov3D[6 * i + k] = 0;
    if (dL_dsh)
      for (int k = 0; k < 3 * M; ++k) dL_dsh[(int64_t)i * 3 * M + k] = 0;
    for (int k = 0; k < 3; ++k) dL_dscales[3 * i + k] = 0;
    for (int k = 0; k < 4; ++k) dL_drots[4 * i + k] = 0;
    if (!(radii[i] > 0)) return;
    const D3 mean = {means3D[3 * i], means3D[3 * i + 1], means3D[3 * i + 2]};
    double c3[6];
    if (cov3D_precomp)
      for (int k = 0; k < 6; ++k) c3[k] = cov3D_precomp[6 * i + k];
    else
      cov3d(scales + 3 * i, scale_modifier, rotations + 4 * i, c3);

    // ---- computeCov2DLonLatCUDA ----
    const double dcx = dL_dconic[4 * i], dcy = dL_dconic[4 * i + 1], dcz = dL_dconic[4 * i + 3];
    const D3 t = xform_point(viewmatrix, mean);
    const double txtx = t.x * t.x, tyty = t.y * t.y, tztz = t.z * t.z, txtytz = t.x * t.y * t.z;
    const double trxztrxz = txtx + tztz;
    const double trxztrxz_inv = 1.0 / (trxztrxz + kEps);
    const double trxz4_inv = trxztrxz_inv * trxztrxz_inv;
    const double trxz = std::sqrt(trxztrxz);
    const double trxz_inv = 1.0 / (trxz + kEps);
    const double trtr = trxztrxz + tyty;
    const double trtr_inv = 1.0 / (trtr + kEps);
    const double trtr2_inv = trtr_inv * trtr_inv;
    const double trxz_trtr2_inv = trxz_inv * trtr2_inv;
    const double trxz3_trtr2_inv = trxztrxz_inv * trxz_trtr2_inv;
    const double tyty_minus_trxztrxz = tyty - trxztrxz;
    const double W_div_2pi = W * 0.5 / M_PI, H_div_pi = H / M_PI;
    const LonlatJac j = lonlat_jacobian(t, W, H);
    DMat3 Jm = mat_cols(j.dpx_dtx, 0.0, j.dpx_dtz, j.dpy_dtx, j.dpy_dty, j.dpy_dtz, 0.0, 0.0, 0.0);
    DMat3 Wm = view_rot_glm(viewmatrix);
    DMat3 Vrk = mat_cols(c3[0], c3[1], c3[2], c3[1], c3[3], c3[4], c3[2], c3[4], c3[5]);
    DMat3 T = mul(Wm, Jm);
    DMat3 cov2D = mul(mul(transpose(T), transpose(Vrk)), T);
    const double a = cov2D.m[0][0] + kLowPass, b = cov2D.m[0][1], c = cov2D.m[1][1] + kLowPass;
    const double denom = a * c - b * b;
    double dL_da = 0, dL_db = 0, dL_dc = 0;
    const double denom2inv = 1.0 / ((denom * denom) + kEps);
    double* dcov = dL_dcov3D + 6 * i;
    if (denom2inv != 0) {
      dL_da = denom2inv * (-c * c * dcx + 2 * b * c * dcy + (denom - a * c) * dcz);
      dL_dc = denom2inv * (-a * a * dcz + 2 * a * b * dcy + (denom - a * c) * dcx);
      dL_db = denom2inv * 2 * (b * c * dcx - (denom + 2 * b * b) * dcy + a * b * dcz);
      const auto& Tm = T.m;
      dcov[0] = (Tm[0][0] * Tm[0][0] * dL_da + Tm[0][0] * Tm[1][0] * dL_db + Tm[1][0] * Tm[1][0] * dL_dc);
      dcov[3] = (Tm[0][1] * Tm[0][1] * dL_da + Tm[0][1] * Tm[1][1] * dL_db + Tm[1][1] * Tm[1][1] * dL_dc);
      dcov[5] = (Tm[0][2] * Tm[0][2] * dL_da + Tm[0][2] * Tm[1][2] * dL_db + Tm[1][2] * Tm[1][2] * dL_dc);
      dcov[1] = 2 * Tm[0][0] * Tm[0][1] * dL_da + (Tm[0][0] * Tm[1][1] + Tm[0][1] * Tm[1][0]) * dL_db +
                2 * Tm[1][0] * Tm[1][1] * dL_dc;
      dcov[2] = 2 * Tm[0][0] * Tm[0][2] * dL_da + (Tm[0][0] * Tm[1][2] + Tm[0][2] * Tm[1][0]) * dL_db +
                2 * Tm[1][0] * Tm[1][2] * dL_dc;
      dcov[4] = 2 * Tm[0][2] * Tm[0][1] * dL_da + (Tm[0][1] * Tm[1][2] + Tm[0][2] * Tm[1][1]) * dL_db +
                2 * Tm[1][1] * Tm[1][2] * dL_dc;
    }
    const auto& Tm = T.m;
    const auto& V = Vrk.m;
    auto rowdot = [&](int ti, int vj) {
      return Tm[ti][0] * V[vj][0] + Tm[ti][1] * V[vj][1] + Tm[ti][2] * V[vj][2];
    };
    double dL_dT0[3], dL_dT1[3];
    for (int jj = 0; jj < 3; ++jj) {
      dL_dT0[jj] = 2 * rowdot(0, jj) * dL_da + rowdot(1, jj) * dL_db;
      dL_dT1[jj] = 2 * rowdot(1, jj) * dL_dc + rowdot(0, jj) * dL_db;
    }
    const auto& Wg = Wm.m;
    const double dL_dJ00 = Wg[0][0] * dL_dT0[0] + Wg[0][1] * dL_dT0[1] + Wg[0][2] * dL_dT0[2];
    const double dL_dJ02 = Wg[2][0] * dL_dT0[0] + Wg[2][1] * dL_dT0[1] + Wg[2][2] * dL_dT0[2];
    const double dL_dJ10 = Wg[0][0] * dL_dT1[0] + Wg[0][1] * dL_dT1[1] + Wg[0][2] * dL_dT1[2];
    const double dL_dJ11 = Wg[1][0] * dL_dT1[0] + Wg[1][1] * dL_dT1[1] + Wg[1][2] * dL_dT1[2];
    const double dL_dJ12 = Wg[2][0] * dL_dT1[0] + Wg[2][1] * dL_dT1[1] + Wg[2][2] * dL_dT1[2];
    // second derivatives of the lonlat map, backward.cu:455-475 (supp.pdf eqs. 43ff)
    const double temp1 = H_div_pi * tyty_minus_trxztrxz * trxz_trtr2_inv;
    const double temp2 = H_div_pi * txtytz * (trtr + 2.0 * trxztrxz) * trxz3_trtr2_inv;
    const double temp3 = W_div_2pi * (txtx - tztz) * trxz4_inv;
    const double temp4 = W_div_2pi * 2.0 * t.x * t.z * trxz4_inv;
    const double temp5 = H_div_pi * t.y * trxz3_trtr2_inv;
    const double dL_dtx = -dL_dJ00 * temp4 + dL_dJ02 * temp3 +
                          dL_dJ10 * temp5 * (2.0 * txtx * trxztrxz - tztz * trtr) +
                          dL_dJ11 * t.x * temp1 + dL_dJ12 * temp2;
    const double dL_dty = dL_dJ10 * t.x * temp1 - dL_dJ11 * H_div_pi * 2.0 * trxz * t.y * trtr2_inv +
                          dL_dJ12 * t.z * temp1;
    const double dL_dtz = dL_dJ00 * temp3 + dL_dJ02 * temp4 + dL_dJ10 * temp2 + dL_dJ11 * t.z * temp1 +
                          dL_dJ12 * temp5 * (2.0 * tztz * trxztrxz - txtx * trtr);
    D3 dmean = xform_vec_T(viewmatrix, {dL_dtx, dL_dty, dL_dtz});

    // ---- preprocessLonLatCUDA: the screen-space mean path ----
    const double dL_dpx = dL_dmean2D[3 * i] * (2.0 / W);
    const double dL_dpy = dL_dmean2D[3 * i + 1] * (2.0 / H);
    const D3 dL_dt2 = {dL_dpx * j.dpx_dtx + dL_dpy * j.dpy_dtx, dL_dpy * j.dpy_dty,
                       dL_dpx * j.dpx_dtz + dL_dpy * j.dpy_dtz};
    dmean = dmean + xform_vec_T(viewmatrix, dL_dt2);

    // ---- computeColorFromSH backward ----
    if (shs && dL_dsh) {
      const D3 dir_orig = mean - cam;
      const double len = std::sqrt(dot(dir_orig, dir_orig));
      const D3 dir = {dir_orig.x / len, dir_orig.y / len, dir_orig.z / len};
      const float* shg = shs + (int64_t)i * M * 3;
      auto sh = [&](int k) { return D3{shg[3 * k], shg[3 * k + 1], shg[3 * k + 2]}; };
      D3 dRGB = {dL_dcolor[3 * i], dL_dcolor[3 * i + 1], dL_dcolor[3 * i + 2]};
      if (clamped[3 * i]) dRGB.x = 0;
      if (clamped[3 * i + 1]) dRGB.y = 0;
      if (clamped[3 * i + 2]) dRGB.z = 0;
      double* dsh = dL_dsh + (int64_t)i * M * 3;
      auto put = [&](int k, double w) {
        dsh[3 * k] = w * dRGB.x; dsh[3 * k + 1] = w * dRGB.y; dsh[3 * k + 2] = w * dRGB.z;
      };
      D3 dx = {0, 0, 0}, dy = {0, 0, 0}, dz = {0, 0, 0};
      const double x = dir.x, y = dir.y, z = dir.z;
      put(0, SH_C0);
      if (D > 0) {
        put(1, -SH_C1 * y); put(2, SH_C1 * z); put(3, -SH_C1 * x);
        dx = (-SH_C1) * sh(3);
        dy = (-SH_C1) * sh(1);
        dz = SH_C1 * sh(2);
        if (D > 1) {
          const double xx = x * x, yy = y * y, zz = z * z, xy = x * y, yz = y * z, xz = x * z;
          put(4, SH_C2[0] * xy); put(5, SH_C2[1] * yz); put(6, SH_C2[2] * (2. * zz - xx - yy));
          put(7, SH_C2[3] * xz); put(8, SH_C2[4] * (xx - yy));
          dx = dx + (SH_C2[0] * y) * sh(4) + (SH_C2[2] * 2. * -x) * sh(6) + (SH_C2[3] * z) * sh(7) +
               (SH_C2[4] * 2. * x) * sh(8);
          dy = dy + (SH_C2[0] * x) * sh(4) + (SH_C2[1] * z) * sh(5) + (SH_C2[2] * 2. * -y) * sh(6) +
               (SH_C2[4] * 2. * -y) * sh(8);
          dz = dz + (SH_C2[1] * y) * sh(5) + (SH_C2[2] * 2. * 2. * z) * sh(6) + (SH_C2[3] * x) * sh(7);
          if (D > 2) {
            put(9, SH_C3[0] * y * (3. * xx - yy)); put(10, SH_C3[1] * xy * z);
            put(11, SH_C3[2] * y * (4. * zz - xx - yy)); put(12, SH_C3[3] * z * (2. * zz - 3. * xx - 3. * yy));
            put(13, SH_C3[4] * x * (4. * zz - xx - yy)); put(14, SH_C3[5] * z * (xx - yy));
            put(15, SH_C3[6] * x * (xx - 3. * yy));
            dx = dx + (SH_C3[0] * 3. * 2. * xy) * sh(9) + (SH_C3[1] * yz) * sh(10) +
                 (SH_C3[2] * -2. * xy) * sh(11) + (SH_C3[3] * -3. * 2. * xz) * sh(12) +
                 (SH_C3[4] * (-3. * xx + 4. * zz - yy)) * sh(13) + (SH_C3[5] * 2. * xz) * sh(14) +
                 (SH_C3[6] * 3. * (xx - yy)) * sh(15);
            dy = dy + (SH_C3[0] * 3. * (xx - yy)) * sh(9) + (SH_C3[1] * xz) * sh(10) +
                 (SH_C3[2] * (-3. * yy + 4. * zz - xx)) * sh(11) + (SH_C3[3] * -3. * 2. * yz) * sh(12) +
                 (SH_C3[4] * -2. * xy) * sh(13) + (SH_C3[5] * -2. * yz) * sh(14) +
                 (SH_C3[6] * -3. * 2. * xy) * sh(15);
            dz = dz + (SH_C3[1] * xy) * sh(10) + (SH_C3[2] * 4. * 2. * yz) * sh(11) +
                 (SH_C3[3] * 3. * (2. * zz - xx - yy)) * sh(12) + (SH_C3[4] * 4. * 2. * xz) * sh(13) +
                 (SH_C3[5] * (xx - yy)) * sh(14);
          }
        }
      }
      const D3 dL_ddir = {dot(dx, dRGB), dot(dy, dRGB), dot(dz, dRGB)};
      // dnormvdv, auxiliary.h:134-144
      const D3 v = dir_orig;
      const double sum2 = dot(v, v);
      const double invsum32 = 1.0 / std::sqrt(sum2 * sum2 * sum2);
      const D3 dn = {((sum2 - v.x * v.x) * dL_ddir.x - v.y * v.x * dL_ddir.y - v.z * v.x * dL_ddir.z) * invsum32,
                     (-v.x * v.y * dL_ddir.x + (sum2 - v.y * v.y) * dL_ddir.y - v.z * v.y * dL_ddir.z) * invsum32,
                     (-v.x * v.z * dL_ddir.x - v.y * v.z * dL_ddir.y + (sum2 - v.z * v.z) * dL_ddir.z) * invsum32};
      dmean = dmean + dn;
    }
    dL_dmeans3D[3 * i] = dmean.x;
    dL_dmeans3D[3 * i + 1] = dmean.y;
    dL_dmeans3D[3 * i + 2] = dmean.z;

    // ---- computeCov3D backward ----
    if (scales) {
      const float* q = rotations + 4 * i;
      const double r = q[0], x = q[1], y = q[2], z = q[3];
      DMat3 R = mat_cols(1. - 2. * (y * y + z * z), 2. * (x * y - r * z), 2. * (x * z + r * y),
                         2. * (x * y + r * z), 1. - 2. * (x * x + z * z), 2. * (y * z - r * x),
                         2. * (x * z - r * y), 2. * (y * z + r * x), 1. - 2. * (x * x + y * y));
      DMat3 S = mat_cols(1, 0, 0, 0, 1, 0, 0, 0, 1);
      const double s[3] = {scale_modifier * (double)scales[3 * i], scale_modifier * (double)scales[3 * i + 1],
                           scale_modifier * (double)scales[3 * i + 2]};
      S.m[0][0] = s[0]; S.m[1][1] = s[1]; S.m[2][2] = s[2];
      DMat3 Mm = mul(S, R);
      const double* dc = dcov;
      DMat3 dSig = mat_cols(dc[0], 0.5 * dc[1], 0.5 * dc[2], 0.5 * dc[1], dc[3], 0.5 * dc[4], 0.5 * dc[2],
                            0.5 * dc[4], dc[5]);
      DMat3 twoM = Mm;
      for (int cc = 0; cc < 3; ++cc)
        for (int rr = 0; rr < 3; ++rr) twoM.m[cc][rr] *= 2.0;
      DMat3 dM = mul(twoM, dSig);
      DMat3 Rt = transpose(R), dMt = transpose(dM);
      for (int k = 0; k < 3; ++k)
        dL_dscales[3 * i + k] = Rt.m[k][0] * dMt.m[k][0] + Rt.m[k][1] * dMt.m[k][1] + Rt.m[k][2] * dMt.m[k][2];
      for (int k = 0; k < 3; ++k)
        for (int rr = 0; rr < 3; ++rr) dMt.m[k][rr] *= s[k];
      const auto& G = dMt.m;
      double* dq = dL_drots + 4 * i;
      dq[0] = 2 * z * (G[0][1] - G[1][0]) + 2 * y * (G[2][0] - G[0][2]) + 2 * x * (G[1][2] - G[2][1]);
      dq[1] = 2 * y * (G[1][0] + G[0][1]) + 2 * z * (G[2][0] + G[0][2]) + 2 * r * (G[1][2] - G[2][1]) -
              4 * x * (G[2][2] + G[1][1]);
      dq[2] = 2 * x * (G[1][0] + G[0][1]) + 2 * r * (G[2][0] - G[0][2]) + 2 * z * (G[1][2] + G[2][1]) -
              4 * y * (G[2][2] + G[0][0]);
      dq[3] = 2 * r * (G[0][1] - G[1][0]) + 2 * x * (G[2][0] + G[0][2]) + 2 * y * (G[1][2] + G[2][1]) -
              4 * z * (G[1][1] + G[0][0]);
    }
  });
}

}  // extern "C"
