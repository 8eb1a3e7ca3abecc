// k_tonemap.cu -- detail-preserving tone map and highlight micro-contrast.
//
// Detail-preserving tone map: core/libraw_wrapper.cpp:1389-1471 with the
// separable box filter box_filter_normalized (:45-116).  The reference's box
// filter is a sliding running sum whose float rounding depends on the scan
// order, so it is reproduced exactly: one thread owns one row (horizontal
// pass) or one column (vertical pass) and walks it in the reference's order.
// Columns are coalesced across the warp; rows are walked through L1.
//
// Micro-contrast: core/cpu_accelerator.cpp:3074-3319.  The 9x9 Gaussian
// (sigma 5/3.7, clamp-to-edge) is a non-separable 81-tap sum in (ky, kx)
// order; it runs out of a shared-memory halo tile with the reference's tap
// order.  The global max of the local standard deviation needs a grid-wide
// reduction, so the stage is two kernels: statistics (+ atomic max), then the
// per-pixel enhancement.
#include <cmath>

#include "lre_internal.h"
#include "stencil.cuh"

namespace lre {

namespace {

__device__ __forceinline__ float aces_tm(float x) {
  const float a = 2.51f, b = 0.03f, c = 2.43f, d = 0.59f, e = 0.14f;
  return (x * (a * x + b)) / (x * (c * x + d) + e);
}

// -------------------------------------------------------- detail tone map
// Horizontal running box sums of two planes at once.  mode 0: the planes are
// derived from RGB (guide = max(0, maxRGB), guide^2); mode 1: plain planes.
__global__ void k_box_rows2(const float* __restrict__ rgb, const float* __restrict__ p0, const float* __restrict__ p1,
                            float* __restrict__ t0, float* __restrict__ t1, int W, int H, int R, int mode) {
  int y = blockIdx.x * blockDim.x + threadIdx.x;
  if (y >= H) return;
  const size_t row = (size_t)y * W;
  auto val = [&](int x, float& a, float& b) {
    if (mode == 0) {
      const float* p = rgb + (row + x) * 3;
      float g = smax(0.0f, smax(p[0], smax(p[1], p[2])));
      a = g;
      b = g * g;
    } else {
      a = p0[row + x];
      b = p1[row + x];
    }
  };
  float s0 = 0.f, s1 = 0.f;
  const int first_right = min(W - 1, R);
  for (int x = 0; x <= first_right; x++) {
    float a, b;
    val(x, a, b);
    s0 += a;
    s1 += b;
  }
  for (int x = 0; x < W; x++) {
    const int left = x > R ? x - R : 0;
    const int right = min(W - 1, x + R);
    const float cnt = (float)(right - left + 1);
    t0[row + x] = s0 / cnt;
    t1[row + x] = s1 / cnt;
    const int remove_x = x >= R ? x - R : W;
    const int add_x = x + R + 1;
    if (remove_x < W) {
      float a, b;
      val(remove_x, a, b);
      s0 -= a;
      s1 -= b;
    }
    if (add_x < W) {
      float a, b;
      val(add_x, a, b);
      s0 += a;
      s1 += b;
    }
  }
}

// Vertical running box sums of two planes; `emit(x, y, m0, m1)` consumes the
// means.  mode 0: produce a, b of the guided filter; mode 1: final apply.
__global__ void k_box_cols2(const float* __restrict__ t0, const float* __restrict__ t1, int W, int H, int R, int mode,
                            float* __restrict__ a_out, float* __restrict__ b_out, const float* __restrict__ rgb_in,
                            float* __restrict__ rgb_out) {
  int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= W) return;
  const float eps = 0.0025f, edge0 = 0.55f, edge1 = 0.90f;
  float s0 = 0.f, s1 = 0.f;
  const int first_bottom = min(H - 1, R);
  for (int y = 0; y <= first_bottom; y++) {
    s0 += t0[(size_t)y * W + x];
    s1 += t1[(size_t)y * W + x];
  }
  for (int y = 0; y < H; y++) {
    const int top = y > R ? y - R : 0;
    const int bottom = min(H - 1, y + R);
    const float cnt = (float)(bottom - top + 1);
    const float m0 = s0 / cnt, m1 = s1 / cnt;
    const size_t i = (size_t)y * W + x;
    if (mode == 0) {
      // m0 = mean(guide), m1 = mean(guide^2)  (core/libraw_wrapper.cpp:1431-1436)
      const float var = smax(0.0f, m1 - m0 * m0);
      const float a = var / (var + eps);
      a_out[i] = a;
      b_out[i] = m0 * (1.0f - a);
    } else {
      // m0 = mean(a), m1 = mean(b)  (core/libraw_wrapper.cpp:1442-1465)
      const float* p = rgb_in + i * 3;
      const float r = p[0], g = p[1], bl = p[2];
      const float guide = smax(0.0f, smax(r, smax(g, bl)));
      const float base = smax(1e-6f, m0 * guide + m1);
      const float mapped = aces_tm(base);
      float gain = sclamp(mapped / base, 0.0f, 1.0f);
      float w = (base - edge0) / (edge1 - edge0);
      w = sclamp(w, 0.0f, 1.0f);
      w = w * w * (3.0f - 2.0f * w);
      float* q = rgb_out + i * 3;
      if (w <= 0.0f) {
        q[0] = r;
        q[1] = g;
        q[2] = bl;
      } else {
        gain = 1.0f + (gain - 1.0f) * w;
        q[0] = r * gain;
        q[1] = g * gain;
        q[2] = bl * gain;
      }
    }
    const int remove_y = y >= R ? y - R : H;
    const int add_y = y + R + 1;
    if (remove_y < H) {
      s0 -= t0[(size_t)remove_y * W + x];
      s1 -= t1[(size_t)remove_y * W + x];
    }
    if (add_y < H) {
      s0 += t0[(size_t)add_y * W + x];
      s1 += t1[(size_t)add_y * W + x];
    }
  }
}

// -------------------------------------------------------- micro-contrast
constexpr int MC_T = 32;
constexpr int MC_R = 4;
constexpr int MC_E = MC_T + 2 * MC_R;

struct McTaps {
  float w[81];
};

// local mean and local std of each channel; atomic max of the std.
__global__ void __launch_bounds__(256) k_mc_stats(const float* __restrict__ in, int W, int H, McTaps taps,
                                                  float* __restrict__ mean3, float* __restrict__ std3, float* d_max) {
  __shared__ float s[3][MC_E * MC_E];
  const int x0 = blockIdx.x * MC_T, y0 = blockIdx.y * MC_T;
  for (int i = threadIdx.x; i < MC_E * MC_E; i += blockDim.x) {
    int gy = min(max(y0 - MC_R + i / MC_E, 0), H - 1);
    int gx = min(max(x0 - MC_R + i % MC_E, 0), W - 1);
    const float* p = in + ((size_t)gy * W + gx) * 3;
    s[0][i] = p[0];
    s[1][i] = p[1];
    s[2][i] = p[2];
  }
  __syncthreads();
  float local_max = 0.f;
  for (int i = threadIdx.x; i < MC_T * MC_T; i += blockDim.x) {
    int ly = i / MC_T, lx = i % MC_T;
    int y = y0 + ly, x = x0 + lx;
    if (x >= W || y >= H) continue;
    float m[3] = {0.f, 0.f, 0.f}, q[3] = {0.f, 0.f, 0.f};
    for (int ky = 0; ky < 9; ky++)
      for (int kx = 0; kx < 9; kx++) {
        const float wgt = taps.w[ky * 9 + kx];
        const int si = (ly + ky) * MC_E + (lx + kx);
#pragma unroll
        for (int c = 0; c < 3; c++) {
          const float v = s[c][si];
          m[c] += v * wgt;
          q[c] += (v * v) * wgt;
        }
      }
    const size_t o = ((size_t)y * W + x) * 3;
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const float var = q[c] - m[c] * m[c];
      const float sd = sqrtf(smax(var, 0.f));
      mean3[o + c] = m[c];
      std3[o + c] = sd;
      local_max = smax(local_max, sd);
    }
  }
  block_max_atomic(local_max, d_max);
}

__global__ void k_mc_apply(const float* in, float* out, const float* __restrict__ mean3,
                           const float* __restrict__ std3, const float* __restrict__ mask, size_t n, float threshold,
                           float strength, float target, const float* d_max) {
  const float max_std = *d_max;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const float* p = in + i * 3;
    const float I0 = p[0], I1 = p[1], I2 = p[2];
    float rgb[3];
    const float Iv[3] = {I0, I1, I2};
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const float m = mean3[i * 3 + c];
      const float contrast = std3[i * 3 + c] / max_std;
      const float ef = (contrast < target) ? strength * (target - contrast) / target : 0.f;
      const float hf = Iv[c] - m;
      const float ehf = hf * (1.f + ef);
      rgb[c] = m + ehf;
    }
    float r = rgb[0], g = rgb[1], b = rgb[2];
    float* q = out + i * 3;
    if (mask) {
      const float w = sclamp(mask[i], 0.f, 1.f);
      const float maxc = smax(r, smax(g, b));
      if (maxc > 1.f) {
        const float scale = 1.f / maxc;
        r *= scale;
        g *= scale;
        b *= scale;
      }
      q[0] = I0 + (r - I0) * w;
      q[1] = I1 + (g - I1) * w;
      q[2] = I2 + (b - I2) * w;
    } else if (I1 >= threshold) {
      const float maxc = smax(r, smax(g, b));
      if (maxc > 1.f) {
        const float scale = 1.f / maxc;
        r *= scale;
        g *= scale;
        b *= scale;
      }
      q[0] = r;
      q[1] = g;
      q[2] = b;
    } else {
      q[0] = I0;
      q[1] = I1;
      q[2] = I2;
    }
  }
}

McTaps make_mc_taps() {
  // create_gaussian_kernel(9, 5/3.7) of core/cpu_accelerator.cpp:3077-3098,
  // evaluated with the host libm exactly as the reference does.
  McTaps t{};
  const float sigma = 5.f / 3.7f;
  const int size = 9, center = size / 2;
  float k[9][9];
  float sum = 0.0f;
  for (int i = 0; i < size; i++)
    for (int j = 0; j < size; j++) {
      float x = (float)(i - center);
      float y = (float)(j - center);
      k[i][j] = std::exp(-(x * x + y * y) / (2.0f * sigma * sigma));
      sum += k[i][j];
    }
  for (int i = 0; i < size; i++)
    for (int j = 0; j < size; j++) k[i][j] /= sum;
  for (int ky = 0; ky < 9; ky++)
    for (int kx = 0; kx < 9; kx++) t.w[ky * 9 + kx] = k[ky][kx];
  return t;
}

}  // namespace

size_t ws_bytes_detail_tonemap(size_t w, size_t h) { return 4 * ((w * h * 4 + 255) & ~size_t(255)); }
size_t ws_bytes_micro_contrast(size_t w, size_t h) { return 2 * ((w * h * 12 + 255) & ~size_t(255)) + 256; }

lre_status launch_detail_tonemap(Context* c, const float* in, float* out, size_t w, size_t h) {
  const int W = (int)w, H = (int)h, R = 12;
  const size_t plane = w * h;
  float* t0 = reinterpret_cast<float*>(c->ws.take(plane * 4));
  float* t1 = reinterpret_cast<float*>(c->ws.take(plane * 4));
  float* pa = reinterpret_cast<float*>(c->ws.take(plane * 4));
  float* pb = reinterpret_cast<float*>(c->ws.take(plane * 4));
  if (!t0 || !t1 || !pa || !pb) return fail(c, LRE_ERR_OUT_OF_MEMORY, "detail_tonemap: workspace too small");
  const int tb = 64;
  k_box_rows2<<<(H + tb - 1) / tb, tb, 0, c->stream>>>(in, nullptr, nullptr, t0, t1, W, H, R, 0);
  k_box_cols2<<<(W + tb - 1) / tb, tb, 0, c->stream>>>(t0, t1, W, H, R, 0, pa, pb, nullptr, nullptr);
  k_box_rows2<<<(H + tb - 1) / tb, tb, 0, c->stream>>>(nullptr, pa, pb, t0, t1, W, H, R, 1);
  k_box_cols2<<<(W + tb - 1) / tb, tb, 0, c->stream>>>(t0, t1, W, H, R, 1, nullptr, nullptr, in, out);
  count_launch(c, 4);
  return check_launch(c, "detail_tonemap");
}

lre_status launch_micro_contrast(Context* c, const float* in, float* out, size_t w, size_t h, float threshold,
                                 float strength, float target, const float* mask) {
  const int W = (int)w, H = (int)h;
  float* mean3 = reinterpret_cast<float*>(c->ws.take(w * h * 12));
  float* std3 = reinterpret_cast<float*>(c->ws.take(w * h * 12));
  float* dmax = reinterpret_cast<float*>(c->ws.take(sizeof(float)));
  if (!mean3 || !std3 || !dmax) return fail(c, LRE_ERR_OUT_OF_MEMORY, "enhance_micro_contrast: workspace too small");
  static const McTaps taps = make_mc_taps();
  LRE_CUDA_TRY(c, cudaMemsetAsync(dmax, 0, sizeof(float), c->stream));
  dim3 grid((W + MC_T - 1) / MC_T, (H + MC_T - 1) / MC_T);
  k_mc_stats<<<grid, 256, 0, c->stream>>>(in, W, H, taps, mean3, std3, dmax);
  k_mc_apply<<<grid_for(w * h, 256, c->sm_count * 8), 256, 0, c->stream>>>(in, out, mean3, std3, mask, w * h,
                                                                            threshold, strength, target, dmax);
  count_launch(c, 2);
  return check_launch(c, "enhance_micro_contrast");
}

}  // namespace lre
