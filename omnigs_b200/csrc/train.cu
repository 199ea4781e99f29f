// Train-step kernels around the rasterizer: the L1 + D-SSIM photometric loss with its image
// gradient, and the Adam step of the Gaussian parameters fused with their activations.
//
// Loss (include/loss_utils.h:30-131, as used at src/gaussian_mapper.cpp:384-409):
//   L = (1 - lambda) mean|img - gt| + lambda (1 - mean SSIM(img, gt)),
// SSIM with the 11x11 Gaussian window (sigma 1.5, zero padding 5, per channel), C1 = 0.01^2,
// C2 = 0.03^2.  The window is separable, so every 2D convolution runs as a horizontal then a
// vertical 11-tap pass in shared memory.  The gradient follows from
//   dSSIM/dimg(p) = 1/N [ (w * A)(p) + 2 img(p) (w * B)(p) + gt(p) (w * Cm)(p) ]
// with per-pixel A = dS/dmu1, B = dS/d(w * img^2), Cm = dS/d(w * img gt) (the window is
// symmetric, so the adjoint convolution is the same convolution).  Kernel 1 computes the local
// statistics, S and A, B, Cm (written to a workspace) and per-block FP64 sums; kernel 2
// convolves A, B, Cm back and writes dL/dimg; kernel 3 writes the three loss values.
//
// Adam (torch::optim::Adam as configured at src/gaussian_model.cpp:485-518: per-group learning
// rates, betas (0.9, 0.999), eps 1e-15, no weight decay) of the raw parameters xyz, f_dc, f_rest,
// opacity (pre-sigmoid), scaling (log) and rotation (unnormalised), given the rasterizer's
// gradients with respect to the activated values (gaussian_model.cpp:54-77): the activation
// backward (exp, sigmoid, L2 normalisation, SH split) is fused into the step, and the kernel
// writes the activated values for the next forward (SH as FP32 or BF16).  The step counter and
// learning rates are read from device memory, so a captured CUDA graph replays across steps.
#include <algorithm>
#include <cmath>
#include <cuda_bf16.h>

#include "../../include/omnigs_b200.h"
#include "capi_internal.h"
#include "device_util.cuh"

namespace omnigs {
namespace {

constexpr int kWin = 11, kHalf = 5;
constexpr int kLossTileW = 32, kLossTileH = 16;
constexpr int kLossThreads = kLossTileW * kLossTileH / 2;  // each thread owns two output pixels
constexpr double kC1 = 0.01 * 0.01, kC2 = 0.03 * 0.03;

struct LossParams {
  const float* img;   // [C][H][W]
  const float* gt;
  float* dimg;        // [C][H][W] gradient; rows >= `rows` are set to 0
  float* ws;          // [3][C][rows][W]: A, B, Cm
  double* sums;       // [2 * blocks]: per-block sum |img - gt|, sum S
  float* loss;        // [3]: loss, l1, ssim
  int C, H, W, rows;
  float lambda;
  float w[kWin];
};

// Register segment of the sliding 11-tap windows: kSeg outputs from kSeg + 10 loads, so shared
// memory is read ~1.8 times per output instead of 11 times.
constexpr int kSeg = 8;

// Block sums of (a, b) into partials[2 * block] (no contended atomics; loss_finalize adds them).
__device__ __forceinline__ void block_sum2(double a, double b, double* partials) {
  __shared__ double s_red[2][kLossThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_xor_sync(kFullMask, a, o);
    b += __shfl_xor_sync(kFullMask, b, o);
  }
  if (lane == 0) {
    s_red[0][warp] = a;
    s_red[1][warp] = b;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double ta = 0.0, tb = 0.0;
    for (int k = 0; k < kLossThreads / 32; ++k) {
      ta += s_red[0][k];
      tb += s_red[1][k];
    }
    const size_t blk = ((size_t)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
    partials[2 * blk] = ta;
    partials[2 * blk + 1] = tb;
  }
}

// Separable 11-tap convolution with zero padding of a [rows][W] plane region, by column strips: a
// block walks down kStripChunks chunks of 16 output rows of a 32-column strip, each pass sliding
// the window along register segments, and keeps the horizontal pass's last 10 rows for the next
// chunk, so each input row is loaded and filtered horizontally once per strip (a 16x32 tile with
// its own 26-row window re-read 10 halo rows: 0.228 -> 0.213 ms per 2048x1024x3 loss, identical
// results).
// `src(ok, y, x, v)` gives the NQ inputs at (y, x) (zeros when !ok, i.e. outside [0, rows) x
// [0, W)), `out(y, x, v)` receives the NQ convolved values of an output pixel; `s_in` holds up to
// 16 input rows (later the vertical results), `s_tmp` the horizontal results of input rows
// y0 - 5 .. y0 + 20 of the current chunk.
constexpr int kStripChunks = 4;
constexpr int kStripRows = kStripChunks * kLossTileH;

template <int NQ, class Src, class Out>
__device__ __forceinline__ void conv_strip(int x0, int ystart, int rows, int W, const float* w,
                                           float (*s_in)[kLossTileH][kLossTileW + 2 * kHalf],
                                           float (*s_tmp)[kLossTileH + 2 * kHalf][kLossTileW], Src src, Out out) {
  constexpr int IW = kLossTileW + 2 * kHalf;
  constexpr int kRowsPerPass = kLossThreads / kLossTileW;
  constexpr int kHSegs = kLossTileW / kSeg, kVSegs = kLossTileH / kSeg;
  const int lx = threadIdx.x % kLossTileW, ly = threadIdx.x / kLossTileW;
  // input rows [ya, ya + n) (with the x halo) into s_in rows [0, n), their horizontal pass into
  // s_tmp rows [dst, dst + n)
  auto load_and_filter = [&](int ya, int n, int dst) {
    for (int ty = ly; ty < n; ty += kRowsPerPass) {
      for (int tx = lx; tx < IW; tx += kLossTileW) {
        const int y = ya + ty, x = x0 + tx - kHalf;
        const bool ok = y >= 0 && y < rows && x >= 0 && x < W;
        float v[NQ];
        src(ok, y, x, v);
#pragma unroll
        for (int q = 0; q < NQ; ++q) s_in[q][ty][tx] = v[q];
      }
    }
    __syncthreads();
    for (int t = threadIdx.x; t < NQ * n * kHSegs; t += kLossThreads) {
      const int q = t / (n * kHSegs), rem = t - q * (n * kHSegs);
      const int ty = rem / kHSegs, xs = (rem - ty * kHSegs) * kSeg;
      float r[kSeg + kWin - 1];
#pragma unroll
      for (int k = 0; k < kSeg + kWin - 1; ++k) r[k] = s_in[q][ty][xs + k];
#pragma unroll
      for (int j = 0; j < kSeg; ++j) {
        float acc = 0.f;
#pragma unroll
        for (int k = 0; k < kWin; ++k) acc = fmaf(w[k], r[j + k], acc);
        s_tmp[q][dst + ty][xs + j] = acc;
      }
    }
    __syncthreads();
  };

  load_and_filter(ystart - kHalf, 2 * kHalf, 0);  // rows ystart - 5 .. ystart + 4
  for (int ch = 0; ch < kStripChunks; ++ch) {
    const int y0 = ystart + ch * kLossTileH;
    if (y0 >= rows) break;  // block-uniform
    load_and_filter(y0 + kHalf, kLossTileH, 2 * kHalf);  // rows y0 + 5 .. y0 + 20
    // vertical pass of the chunk's 16 output rows into s_in
    for (int t = threadIdx.x; t < NQ * kLossTileW * kVSegs; t += kLossThreads) {
      const int q = t / (kLossTileW * kVSegs), rem = t - q * (kLossTileW * kVSegs);
      const int ys = (rem / kLossTileW) * kSeg, tx = rem % kLossTileW;
      float r[kSeg + kWin - 1];
#pragma unroll
      for (int k = 0; k < kSeg + kWin - 1; ++k) r[k] = s_tmp[q][ys + k][tx];
#pragma unroll
      for (int j = 0; j < kSeg; ++j) {
        float acc = 0.f;
#pragma unroll
        for (int k = 0; k < kWin; ++k) acc = fmaf(w[k], r[j + k], acc);
        s_in[q][ys + j][tx] = acc;
      }
    }
    __syncthreads();
    // outputs of the chunk; meanwhile the horizontal rows the next chunk shares move to the front
    for (int ty = ly; ty < kLossTileH; ty += kRowsPerPass) {
      float v[NQ];
#pragma unroll
      for (int q = 0; q < NQ; ++q) v[q] = s_in[q][ty][lx];
      const int y = y0 + ty, x = x0 + lx;
      if (y < rows && x < W) out(y, x, v);
    }
    for (int t = threadIdx.x; t < NQ * 2 * kHalf * kLossTileW; t += kLossThreads) {
      const int q = t / (2 * kHalf * kLossTileW), rem = t - q * (2 * kHalf * kLossTileW);
      const int r = rem / kLossTileW, x = rem - r * kLossTileW;
      s_tmp[q][r][x] = s_tmp[q][kLossTileH + r][x];
    }
    __syncthreads();
  }
}

// Kernel 1: local statistics of one 32-column strip of kStripRows rows of one channel (blockIdx.z).
__global__ void __launch_bounds__(kLossThreads) ssim_stats_kernel(const __grid_constant__ LossParams p) {
  __shared__ float s_in[5][kLossTileH][kLossTileW + 2 * kHalf];
  __shared__ float s_tmp[5][kLossTileH + 2 * kHalf][kLossTileW];
  const int c = blockIdx.z;
  const int x0 = blockIdx.x * kLossTileW, ystart = blockIdx.y * kStripRows;
  const size_t plane = (size_t)p.H * p.W;
  const float* a = p.img + c * plane;
  const float* b = p.gt + c * plane;
  const size_t ws_plane = (size_t)p.rows * p.W;
  float* A = p.ws + c * ws_plane;
  float* B = p.ws + (p.C + c) * ws_plane;
  float* Cm = p.ws + (2 * p.C + c) * ws_plane;
  double l1 = 0.0, ssum = 0.0;
  auto src = [&](bool ok, int y, int x, float v[5]) {
    const float u = ok ? a[(size_t)y * p.W + x] : 0.f;
    const float g = ok ? b[(size_t)y * p.W + x] : 0.f;
    v[0] = u;
    v[1] = g;
    v[2] = u * u;
    v[3] = g * g;
    v[4] = u * g;
  };
  auto out = [&](int y, int x, const float m[5]) {
    const float mu1 = m[0], mu2 = m[1];
    const float mu1_sq = mu1 * mu1, mu2_sq = mu2 * mu2, mu1_mu2 = mu1 * mu2;
    const float s1 = m[2] - mu1_sq, s2 = m[3] - mu2_sq, s12 = m[4] - mu1_mu2;
    const float a1 = 2.f * mu1_mu2 + (float)kC1, a2 = 2.f * s12 + (float)kC2;
    const float b1 = mu1_sq + mu2_sq + (float)kC1, b2 = s1 + s2 + (float)kC2;
    const float inv = 1.f / (b1 * b2);
    const float S = a1 * a2 * inv;
    const size_t o = (size_t)y * p.W + x;
    // dS/dmu1, dS/d(w * img^2), dS/d(w * img gt) with mu2 and the gt moments fixed
    A[o] = 2.f * mu2 * (a2 - a1) * inv - 2.f * mu1 * S * (1.f / b1 - 1.f / b2);
    B[o] = -S / b2;
    Cm[o] = 2.f * a1 * inv;
    ssum += (double)S;
    l1 += (double)fabsf(a[o] - b[o]);
  };
  conv_strip<5>(x0, ystart, p.rows, p.W, p.w, s_in, s_tmp, src, out);
  block_sum2(l1, ssum, p.sums);
}

// Kernel 2: dL/dimg of one 32-column strip of kStripRows rows of one channel.
__global__ void __launch_bounds__(kLossThreads) ssim_grad_kernel(const __grid_constant__ LossParams p) {
  __shared__ float s_in[3][kLossTileH][kLossTileW + 2 * kHalf];
  __shared__ float s_tmp[3][kLossTileH + 2 * kHalf][kLossTileW];
  const int c = blockIdx.z;
  const int x0 = blockIdx.x * kLossTileW, ystart = blockIdx.y * kStripRows;
  const size_t plane = (size_t)p.H * p.W;
  const float* a = p.img + c * plane;
  const float* b = p.gt + c * plane;
  float* d = p.dimg + c * plane;
  const size_t ws_plane = (size_t)p.rows * p.W;
  const float* A = p.ws + c * ws_plane;
  const float* B = p.ws + (p.C + c) * ws_plane;
  const float* Cm = p.ws + (2 * p.C + c) * ws_plane;
  const float invN = (float)(1.0 / ((double)p.C * p.rows * p.W));
  const float k_l1 = (1.f - p.lambda) * invN, k_ssim = -p.lambda * invN;
  auto src = [&](bool ok, int y, int x, float v[3]) {
    const size_t o = (size_t)y * p.W + x;
    v[0] = ok ? A[o] : 0.f;
    v[1] = ok ? B[o] : 0.f;
    v[2] = ok ? Cm[o] : 0.f;
  };
  auto out = [&](int y, int x, const float m[3]) {
    const size_t o = (size_t)y * p.W + x;
    const float u = a[o], g = b[o];
    const float diff = u - g;
    const float sgn = diff > 0.f ? 1.f : (diff < 0.f ? -1.f : 0.f);
    const float dssim = m[0] + 2.f * u * m[1] + g * m[2];
    d[o] = k_l1 * sgn + k_ssim * dssim;
  };
  conv_strip<3>(x0, ystart, p.rows, p.W, p.w, s_in, s_tmp, src, out);
  // rows below `rows` are not part of the loss
  if (blockIdx.y == gridDim.y - 1) {
    for (int i = threadIdx.x; i < (p.H - p.rows) * kLossTileW; i += blockDim.x) {
      const int y = p.rows + i / kLossTileW, x = x0 + i % kLossTileW;
      if (x < p.W) d[(size_t)y * p.W + x] = 0.f;
    }
  }
}

__global__ void __launch_bounds__(1024) loss_finalize_kernel(const double* partials, int blocks, float* loss,
                                                              double invN, float lambda) {
  __shared__ double s_red[2][32];
  double a = 0.0, b = 0.0;
  for (int i = threadIdx.x; i < blocks; i += blockDim.x) {
    a += partials[2 * i];
    b += partials[2 * i + 1];
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_xor_sync(kFullMask, a, o);
    b += __shfl_xor_sync(kFullMask, b, o);
  }
  if (lane == 0) {
    s_red[0][warp] = a;
    s_red[1][warp] = b;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double ta = 0.0, tb = 0.0;
    for (int k = 0; k < (int)(blockDim.x / 32); ++k) {
      ta += s_red[0][k];
      tb += s_red[1][k];
    }
    const double l1 = ta * invN, ssim = tb * invN;
    loss[0] = (float)((1.0 - lambda) * l1 + lambda * (1.0 - ssim));
    loss[1] = (float)l1;
    loss[2] = (float)ssim;
  }
}

// ---------------------------------------------------------------- Adam ------------------------
struct AdamParams {
  OmnigsGaussianParams prm;
  OmnigsAdamState st;
  OmnigsActivated act;
  const float* dL_dmeans3D;
  const float* dL_dsh;
  const float* dL_dopacity;
  const float* dL_dscales;
  const float* dL_drotations;
  const OmnigsAdamHyper* hyper;  // device
};

struct AdamScalars {
  float step_size, bc2_sqrt, beta1, one_minus_beta1, beta2, one_minus_beta2, eps;
};

// The float coefficients torch::optim::Adam applies (its double options rounded once).
__device__ __forceinline__ AdamScalars adam_scalars(const OmnigsAdamHyper& h, int group) {
  const double t = (double)h.step;
  AdamScalars s;
  const double bc1 = 1.0 - pow(h.beta1, t), bc2 = 1.0 - pow(h.beta2, t);
  s.step_size = (float)(h.lr[group] / bc1);
  s.bc2_sqrt = (float)sqrt(bc2);
  s.beta1 = (float)h.beta1;
  s.one_minus_beta1 = (float)(1.0 - h.beta1);
  s.beta2 = (float)h.beta2;
  s.one_minus_beta2 = (float)(1.0 - h.beta2);
  s.eps = (float)h.eps;
  return s;
}

// One Adam update of one parameter value (torch::optim::Adam: exp_avg = b1 m + (1 - b1) g,
// exp_avg_sq = b2 v + (1 - b2) g^2, p -= step_size m / (sqrt(v) / sqrt(bc2) + eps)).
__device__ __forceinline__ float adam_update(float& p, float& m, float& v, float g, const AdamScalars& s) {
  m = __fmaf_rn(s.one_minus_beta1, g, __fmul_rn(m, s.beta1));
  v = __fmaf_rn(__fmul_rn(s.one_minus_beta2, g), g, __fmul_rn(v, s.beta2));
  const float denom = __fadd_rn(__fdiv_rn(sqrtf(v), s.bc2_sqrt), s.eps);
  p = __fsub_rn(p, __fmul_rn(s.step_size, __fdiv_rn(m, denom)));
  return p;
}

__global__ void __launch_bounds__(256) adam_gaussian_kernel(const __grid_constant__ AdamParams p) {
  __shared__ AdamScalars s_sc[6];
  const int P = p.prm.P, M = p.prm.M;
  const int64_t rest_n = (int64_t)P * (M - 1) * 3;
  if (threadIdx.x < 6) s_sc[threadIdx.x] = adam_scalars(*p.hyper, threadIdx.x);
  __syncthreads();
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  // per-Gaussian groups: xyz, f_dc, opacity, scaling, rotation
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < P; i += stride) {
    const int g = (int)i;
    {  // xyz (group 0): the activated mean is the parameter itself
      const AdamScalars& s = s_sc[0];
      for (int k = 0; k < 3; ++k) {
        const float v = adam_update(p.prm.xyz[3 * g + k], p.st.m_xyz[3 * g + k], p.st.v_xyz[3 * g + k],
                                    p.dL_dmeans3D[3 * g + k], s);
        if (p.act.means3D != p.prm.xyz) p.act.means3D[3 * g + k] = v;
      }
    }
    {  // f_dc (group 1) = SH coefficient 0
      const AdamScalars& s = s_sc[1];
      for (int k = 0; k < 3; ++k) {
        const float v = adam_update(p.prm.features_dc[3 * g + k], p.st.m_dc[3 * g + k], p.st.v_dc[3 * g + k],
                                    p.dL_dsh[(size_t)g * M * 3 + k], s);
        if (p.act.shs_bf16)
          reinterpret_cast<__nv_bfloat16*>(p.act.shs)[(size_t)g * M * 3 + k] = __float2bfloat16_rn(v);
        else
          static_cast<float*>(p.act.shs)[(size_t)g * M * 3 + k] = v;
      }
    }
    {  // opacity (group 3), sigmoid
      const AdamScalars& s = s_sc[3];
      const float o = p.act.opacities[g];  // sigmoid of the current parameter (previous forward)
      const float grad = p.dL_dopacity[g] * o * (1.f - o);
      const float v = adam_update(p.prm.opacity[g], p.st.m_opacity[g], p.st.v_opacity[g], grad, s);
      p.act.opacities[g] = 1.f / (1.f + expf(-v));
    }
    {  // scaling (group 4), exp
      const AdamScalars& s = s_sc[4];
      for (int k = 0; k < 3; ++k) {
        const float e = p.act.scales[3 * g + k];  // exp of the current parameter
        const float v = adam_update(p.prm.scaling[3 * g + k], p.st.m_scaling[3 * g + k], p.st.v_scaling[3 * g + k],
                                    p.dL_dscales[3 * g + k] * e, s);
        p.act.scales[3 * g + k] = expf(v);
      }
    }
    {  // rotation (group 5), L2 normalisation (F.normalize, eps 1e-12)
      const AdamScalars& s = s_sc[5];
      float r[4], gr[4];
      for (int k = 0; k < 4; ++k) {
        r[k] = p.prm.rotation[4 * g + k];
        gr[k] = p.dL_drotations[4 * g + k];
      }
      const float n = fmaxf(sqrtf(r[0] * r[0] + r[1] * r[1] + r[2] * r[2] + r[3] * r[3]), 1e-12f);
      const float inv = 1.f / n;
      const float yg = (r[0] * gr[0] + r[1] * gr[1] + r[2] * gr[2] + r[3] * gr[3]) * inv;  // y . g
      float nr[4];
      for (int k = 0; k < 4; ++k) {
        const float dr = (gr[k] - r[k] * inv * yg) * inv;
        nr[k] = adam_update(p.prm.rotation[4 * g + k], p.st.m_rotation[4 * g + k], p.st.v_rotation[4 * g + k], dr, s);
      }
      const float n2 = fmaxf(sqrtf(nr[0] * nr[0] + nr[1] * nr[1] + nr[2] * nr[2] + nr[3] * nr[3]), 1e-12f);
      for (int k = 0; k < 4; ++k) p.act.rotations[4 * g + k] = nr[k] / n2;
    }
  }
  // f_rest (group 2), elementwise (element e of Gaussian g's (M - 1) x 3 rest coefficients; rest_n <
  // 2^32 is checked on the host, so 32-bit index arithmetic suffices).  Each thread loads
  // kAdamUnroll elements before updating any, so that many loads are in flight per thread.
  constexpr int kAdamUnroll = 4;
  const uint32_t per = (uint32_t)(M - 1) * 3u;
  // e / per as a multiply-high by ceil(2^32 / per): for every 32-bit e the estimate is the quotient
  // or one more, and one comparison settles it
  const uint32_t per_magic = per ? (uint32_t)((0x100000000ull + per - 1) / per) : 0u;
  const AdamScalars& s = s_sc[2];
  for (int64_t base = (int64_t)blockIdx.x * blockDim.x * kAdamUnroll + threadIdx.x; base < rest_n;
       base += stride * kAdamUnroll) {
    float pv[kAdamUnroll], mv[kAdamUnroll], vv[kAdamUnroll], gv[kAdamUnroll];
    size_t sh_idx[kAdamUnroll];
#pragma unroll
    for (int u = 0; u < kAdamUnroll; ++u) {
      const int64_t e = base + (int64_t)u * blockDim.x;
      if (e < rest_n) {
        uint32_t g = __umulhi((uint32_t)e, per_magic);
        if ((uint64_t)g * per > (uint64_t)e) --g;
        const uint32_t r = (uint32_t)e - g * per;
        sh_idx[u] = (size_t)g * M * 3 + 3 + r;
        pv[u] = p.prm.features_rest[e];
        mv[u] = p.st.m_rest[e];
        vv[u] = p.st.v_rest[e];
        gv[u] = p.dL_dsh[sh_idx[u]];
      }
    }
#pragma unroll
    for (int u = 0; u < kAdamUnroll; ++u) {
      const int64_t e = base + (int64_t)u * blockDim.x;
      if (e < rest_n) {
        const float v = adam_update(pv[u], mv[u], vv[u], gv[u], s);
        p.prm.features_rest[e] = pv[u];
        p.st.m_rest[e] = mv[u];
        p.st.v_rest[e] = vv[u];
        if (p.act.shs_bf16)
          reinterpret_cast<__nv_bfloat16*>(p.act.shs)[sh_idx[u]] = __float2bfloat16_rn(v);
        else
          static_cast<float*>(p.act.shs)[sh_idx[u]] = v;
      }
    }
  }
}

// Activated values from the raw parameters (the first forward of a training run).
__global__ void __launch_bounds__(256) activate_kernel(const OmnigsGaussianParams prm, const OmnigsActivated act) {
  const int P = prm.P, M = prm.M;
  const int64_t rest_n = (int64_t)P * (M - 1) * 3;
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  auto put_sh = [&](size_t idx, float v) {
    if (act.shs_bf16)
      reinterpret_cast<__nv_bfloat16*>(act.shs)[idx] = __float2bfloat16_rn(v);
    else
      static_cast<float*>(act.shs)[idx] = v;
  };
  if (i < P) {
    const int g = (int)i;
    for (int k = 0; k < 3; ++k) {
      if (act.means3D != prm.xyz) act.means3D[3 * g + k] = prm.xyz[3 * g + k];
      put_sh((size_t)g * M * 3 + k, prm.features_dc[3 * g + k]);
      act.scales[3 * g + k] = expf(prm.scaling[3 * g + k]);
    }
    act.opacities[g] = 1.f / (1.f + expf(-prm.opacity[g]));
    float r[4];
    for (int k = 0; k < 4; ++k) r[k] = prm.rotation[4 * g + k];
    const float n = fmaxf(sqrtf(r[0] * r[0] + r[1] * r[1] + r[2] * r[2] + r[3] * r[3]), 1e-12f);
    for (int k = 0; k < 4; ++k) act.rotations[4 * g + k] = r[k] / n;
  } else if (i - P < rest_n) {
    const uint32_t e = (uint32_t)(i - P);
    const uint32_t per = (uint32_t)(M - 1) * 3u;
    const uint32_t g = e / per, r = e - g * per;
    put_sh((size_t)g * M * 3 + 3 + r, prm.features_rest[e]);
  }
}

int validate_params(const OmnigsGaussianParams* prm, const OmnigsActivated* act) {
  if (prm == nullptr || act == nullptr) return fail(OMNIGS_ERR_INVALID_ARGUMENT, "parameters are NULL");
  if (prm->P < 0 || prm->M < 1 || prm->M > 16)
    return fail(OMNIGS_ERR_INVALID_ARGUMENT, "P must be >= 0 and M (SH coefficients) in [1, 16]");
  if ((int64_t)prm->P * (prm->M - 1) * 3 >= (int64_t(1) << 32))
    return fail(OMNIGS_ERR_INVALID_ARGUMENT, "P * (M - 1) * 3 must be below 2^32");
  if (prm->P == 0) return OMNIGS_OK;
  if (!prm->xyz || !prm->features_dc || (prm->M > 1 && !prm->features_rest) || !prm->opacity || !prm->scaling ||
      !prm->rotation || !act->means3D || !act->shs || !act->opacities || !act->scales || !act->rotations)
    return fail(OMNIGS_ERR_INVALID_ARGUMENT, "a parameter or activated-value array is NULL");
  return OMNIGS_OK;
}

}  // namespace
}  // namespace omnigs

using namespace omnigs;

extern "C" {

size_t omnigs_l1_dssim_workspace_bytes(int C, int H, int W) {
  if (C <= 0 || H <= 0 || W <= 0) return 0;
  const size_t blocks = (size_t)C * ((W + kLossTileW - 1) / kLossTileW) * ((H + kLossTileH - 1) / kLossTileH);
  return align_up(sizeof(double) * 2 * blocks) + sizeof(float) * 3 * (size_t)C * H * W;
}

int omnigs_l1_dssim(const float* image, const float* gt, int C, int H, int W, int rows, float lambda_dssim,
                    float* dL_dimage, float* loss, void* workspace, size_t workspace_bytes, omnigs_stream_t stream) {
  g_last_error.clear();
  if (image == nullptr || gt == nullptr || dL_dimage == nullptr || loss == nullptr || workspace == nullptr)
    return fail(OMNIGS_ERR_INVALID_ARGUMENT, "image, gt, dL_dimage, loss and workspace are required");
  if (C <= 0 || H <= 0 || W <= 0 || rows <= 0 || rows > H || (int64_t)H * W > (int64_t(1) << 28))
    return fail(OMNIGS_ERR_INVALID_ARGUMENT, "image size must be positive with 0 < rows <= H");
  if (!(lambda_dssim >= 0.f && lambda_dssim <= 1.f))
    return fail(OMNIGS_ERR_INVALID_ARGUMENT, "lambda_dssim must be in [0, 1]");
  if (workspace_bytes < omnigs_l1_dssim_workspace_bytes(C, H, W))
    return fail(OMNIGS_ERR_BUFFER_TOO_SMALL, "workspace smaller than omnigs_l1_dssim_workspace_bytes()");
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  LossParams p{};
  p.img = image;
  p.gt = gt;
  p.dimg = dL_dimage;
  const dim3 grid((W + kLossTileW - 1) / kLossTileW, (rows + kLossTileH - 1) / kLossTileH, C);
  const size_t max_blocks = (size_t)C * ((W + kLossTileW - 1) / kLossTileW) * ((H + kLossTileH - 1) / kLossTileH);
  p.sums = static_cast<double*>(workspace);
  p.ws = reinterpret_cast<float*>(static_cast<unsigned char*>(workspace) + align_up(sizeof(double) * 2 * max_blocks));
  p.loss = loss;
  p.C = C;
  p.H = H;
  p.W = W;
  p.rows = rows;
  p.lambda = lambda_dssim;
  // the reference's window: exp(-x^2 / (2 sigma^2)) in float, normalised (loss_utils.h:54-68)
  float sum = 0.f;
  for (int k = 0; k < kWin; ++k) {
    const int t = k - kWin / 2;
    p.w[k] = std::exp(-(float)(t * t) / (2.0f * 1.5f * 1.5f));
    sum += p.w[k];
  }
  for (int k = 0; k < kWin; ++k) p.w[k] /= sum;
  const dim3 strip_grid(grid.x, (rows + kStripRows - 1) / kStripRows, C);
  const int blocks = (int)(strip_grid.x * strip_grid.y * strip_grid.z);
  staged(OMNIGS_STAGE_OTHER, 3, s, [&] {
    ssim_stats_kernel<<<strip_grid, kLossThreads, 0, s>>>(p);
    ssim_grad_kernel<<<strip_grid, kLossThreads, 0, s>>>(p);
    loss_finalize_kernel<<<1, 1024, 0, s>>>(p.sums, blocks, loss, 1.0 / ((double)C * rows * W), lambda_dssim);
  });
  return check_launch("l1 + d-ssim");
}

int omnigs_activate(const OmnigsGaussianParams* prm, const OmnigsActivated* act, omnigs_stream_t stream) {
  g_last_error.clear();
  if (int rc = validate_params(prm, act)) return rc;
  if (prm->P == 0) return OMNIGS_OK;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const int64_t n = (int64_t)prm->P + (int64_t)prm->P * (prm->M - 1) * 3;
  staged(OMNIGS_STAGE_OTHER, 1, s,
         [&] { activate_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(*prm, *act); });
  return check_launch("activate");
}

int omnigs_adam_step(const OmnigsGaussianParams* prm, const OmnigsAdamState* st, const OmnigsActivated* act,
                     const float* dL_dmeans3D, const float* dL_dsh, const float* dL_dopacity, const float* dL_dscales,
                     const float* dL_drotations, const OmnigsAdamHyper* hyper, omnigs_stream_t stream) {
  g_last_error.clear();
  if (int rc = validate_params(prm, act)) return rc;
  if (st == nullptr || hyper == nullptr) return fail(OMNIGS_ERR_INVALID_ARGUMENT, "Adam state and hyper are required");
  if (prm->P == 0) return OMNIGS_OK;
  if (!dL_dmeans3D || !dL_dsh || !dL_dopacity || !dL_dscales || !dL_drotations || !st->m_xyz || !st->v_xyz ||
      !st->m_dc || !st->v_dc || (prm->M > 1 && (!st->m_rest || !st->v_rest)) || !st->m_opacity || !st->v_opacity ||
      !st->m_scaling || !st->v_scaling || !st->m_rotation || !st->v_rotation)
    return fail(OMNIGS_ERR_INVALID_ARGUMENT, "a gradient or Adam moment array is NULL");
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  AdamParams p{};
  p.prm = *prm;
  p.st = *st;
  p.act = *act;
  p.dL_dmeans3D = dL_dmeans3D;
  p.dL_dsh = dL_dsh;
  p.dL_dopacity = dL_dopacity;
  p.dL_dscales = dL_dscales;
  p.dL_drotations = dL_drotations;
  p.hyper = hyper;
  const int64_t n = (int64_t)prm->P + (int64_t)prm->P * (prm->M - 1) * 3;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const unsigned blocks = (unsigned)std::min<int64_t>((n + 255) / 256, (int64_t)sms * 8);
  staged(OMNIGS_STAGE_OTHER, 1, s, [&] { adam_gaussian_kernel<<<blocks, 256, 0, s>>>(p); });
  return check_launch("adam step");
}

}  // extern "C"
