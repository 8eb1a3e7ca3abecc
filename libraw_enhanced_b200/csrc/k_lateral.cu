// k_lateral.cu -- lateral chromatic-aberration registration: pyramidal
// Lucas-Kanade of R and B against G per cell, confidence gate, 3x3 cell
// smoothing, bilinear remap.
//
// Semantics: core/cpu_accelerator.cpp:3496-3673 (ca_register_lateral) with
// downsample_2x_box (:3369-3384), lk_estimate_level (:3390-3471),
// smooth_3x3_cells (:3474-3492) and bilinear_sample_plane (:3328-3346).
//
// Device plan: planar split + 2x box pyramid (one kernel per level); per
// level ONE launch estimates every cell of both channels, one CTA per
// (cell, channel): the CTA sweeps the cell's pixels, reduces the 2x2 normal
// equations in double with warp shuffles, and thread 0 solves and broadcasts
// the step, so all LK iterations of a cell stay on chip.  Gate + smoothing
// run in one small kernel; the remap is a streaming kernel.
#include <algorithm>
#include <cmath>

#include "lre_internal.h"
#include "stencil.cuh"

namespace lre {

namespace {

constexpr int LK_THREADS = 256;

__global__ void k_split_planes(const float* __restrict__ rgb, float* __restrict__ R, float* __restrict__ G,
                               float* __restrict__ B, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    R[i] = rgb[i * 3 + 0];
    G[i] = rgb[i * 3 + 1];
    B[i] = rgb[i * 3 + 2];
  }
}

struct Planes3 {
  const float* in[3];
  float* out[3];
};

__global__ void k_downsample3(Planes3 p, int W, int H, int W2, int H2) {
  size_t n = (size_t)W2 * H2;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    int y = (int)(i / W2), x = (int)(i % W2);
    int y0 = 2 * y, y1 = min(y0 + 1, H - 1);
    int x0 = 2 * x, x1 = min(x0 + 1, W - 1);
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const float* in = p.in[c];
      p.out[c][i] = 0.25f * (in[(size_t)y0 * W + x0] + in[(size_t)y0 * W + x1] + in[(size_t)y1 * W + x0] +
                             in[(size_t)y1 * W + x1]);
    }
  }
}

__device__ __forceinline__ float bilinear_plane(const float* __restrict__ plane, int W, int H, float x, float y) {
  if (x < 0.f) x = 0.f;
  if (y < 0.f) y = 0.f;
  if (x > (float)(W - 1)) x = (float)(W - 1);
  if (y > (float)(H - 1)) y = (float)(H - 1);
  const int x0 = (int)x;
  const int y0 = (int)y;
  const int x1 = min(x0 + 1, W - 1);
  const int y1 = min(y0 + 1, H - 1);
  const float fx = x - (float)x0;
  const float fy = y - (float)y0;
  const float v00 = plane[(size_t)y0 * W + x0];
  const float v01 = plane[(size_t)y0 * W + x1];
  const float v10 = plane[(size_t)y1 * W + x0];
  const float v11 = plane[(size_t)y1 * W + x1];
  return (v00 * (1.f - fx) + v01 * fx) * (1.f - fy) + (v10 * (1.f - fx) + v11 * fx) * fy;
}

struct LkMaps {
  float* dx[2];
  float* dy[2];
  float* conf[2];
};

// One CTA per (cell, channel).  blockIdx.x = cell, blockIdx.y = channel
// (0: R, 1: B).
__global__ void __launch_bounds__(LK_THREADS) k_lk_level(const float* __restrict__ G, const float* __restrict__ Rt,
                                                         const float* __restrict__ Bt, int W, int H, int map_w,
                                                         int map_h, int max_iterations, float max_shift,
                                                         float scale_down, float scale_up, LkMaps maps) {
  __shared__ double red[5][LK_THREADS / 32];
  __shared__ float s_acc[2];
  __shared__ int s_done;
  const int ch = blockIdx.y;
  const float* T = ch == 0 ? Rt : Bt;
  const int cell = blockIdx.x;
  const int cy = cell / map_w, cx = cell % map_w;
  const float cell_w_f = (float)W / (float)map_w;
  const float cell_h_f = (float)H / (float)map_h;
  const size_t x0 = (size_t)(cx * cell_w_f);
  const size_t y0 = (size_t)(cy * cell_h_f);
  size_t x1 = (size_t)((cx + 1) * cell_w_f);
  size_t y1 = (size_t)((cy + 1) * cell_h_f);
  x1 = x1 < (size_t)W ? x1 : (size_t)W;
  y1 = y1 < (size_t)H ? y1 : (size_t)H;
  float* dxm = maps.dx[ch];
  float* dym = maps.dy[ch];
  float* cfm = maps.conf[ch];
  float accum_dx = dxm[cell] * scale_down;
  float accum_dy = dym[cell] * scale_down;
  if (x1 <= x0 + 4 || y1 <= y0 + 4) {
    if (threadIdx.x == 0) {
      dxm[cell] = accum_dx * scale_up;
      dym[cell] = accum_dy * scale_up;
    }
    return;
  }
  const int iw = (int)(x1 - x0) - 2, ih = (int)(y1 - y0) - 2;  // interior extent
  const int npx = iw * ih;
  float min_eig_final = 0.f;
  for (int iter = 0; iter < max_iterations; iter++) {
    double A00 = 0.0, A01 = 0.0, A11 = 0.0, bx = 0.0, by = 0.0;
    for (int k = threadIdx.x; k < npx; k += blockDim.x) {
      const int y = (int)y0 + 1 + k / iw;
      const int x = (int)x0 + 1 + k % iw;
      const size_t i = (size_t)y * W + x;
      const float gx = G[i + 1] - G[i - 1];
      const float gy = G[i + W] - G[i - W];
      const float t_warp = bilinear_plane(T, W, H, (float)x + accum_dx, (float)y + accum_dy);
      const float err = t_warp - G[i];
      A00 += (double)gx * gx;
      A01 += (double)gx * gy;
      A11 += (double)gy * gy;
      bx -= (double)gx * err;
      by -= (double)gy * err;
    }
    A00 = warp_sum_d(A00);
    A01 = warp_sum_d(A01);
    A11 = warp_sum_d(A11);
    bx = warp_sum_d(bx);
    by = warp_sum_d(by);
    const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) {
      red[0][wid] = A00;
      red[1][wid] = A01;
      red[2][wid] = A11;
      red[3][wid] = bx;
      red[4][wid] = by;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      double s[5] = {0, 0, 0, 0, 0};
      for (int w = 0; w < LK_THREADS / 32; w++)
        for (int q = 0; q < 5; q++) s[q] += red[q][w];
      int done = 0;
      if (npx < 32) {
        done = 1;
      } else {
        const double det = s[0] * s[2] - s[1] * s[1];
        const double trace = s[0] + s[2];
        const double disc = fmax(0.0, trace * trace - 4.0 * det);
        const double sq = sqrt(disc);
        min_eig_final = (float)(0.5 * (trace - sq));
        if (det <= 1e-12) {
          done = 1;
        } else {
          const double inv = 1.0 / det;
          const double step_x = inv * (s[2] * s[3] - s[1] * s[4]);
          const double step_y = inv * (-s[1] * s[3] + s[0] * s[4]);
          accum_dx += (float)step_x;
          accum_dy += (float)step_y;
          if (accum_dx > max_shift) accum_dx = max_shift;
          if (accum_dx < -max_shift) accum_dx = -max_shift;
          if (accum_dy > max_shift) accum_dy = max_shift;
          if (accum_dy < -max_shift) accum_dy = -max_shift;
          if (fabs(step_x) < 0.005 && fabs(step_y) < 0.005) done = 1;
        }
      }
      s_acc[0] = accum_dx;
      s_acc[1] = accum_dy;
      s_done = done;
    }
    __syncthreads();
    accum_dx = s_acc[0];
    accum_dy = s_acc[1];
    const int done = s_done;
    __syncthreads();
    if (done) break;
  }
  if (threadIdx.x == 0) {
    dxm[cell] = accum_dx * scale_up;
    dym[cell] = accum_dy * scale_up;
    cfm[cell] = fmaxf(0.f, min_eig_final);
  }
}

// Confidence gate (relative to the strongest cell) and one 3x3 smoothing
// pass of each map.  One CTA; `tmp` holds 4 * n floats.
__global__ void k_lk_gate_smooth(LkMaps maps, int map_w, int map_h, float min_conf, float* tmp) {
  __shared__ float s_max[2][32];
  const int n = map_w * map_h;
  for (int ch = 0; ch < 2; ch++) {
    float m = 0.f;
    for (int i = threadIdx.x; i < n; i += blockDim.x) m = smax(m, maps.conf[ch][i]);
    m = warp_max(m);
    if ((threadIdx.x & 31) == 0) s_max[ch][threadIdx.x >> 5] = m;
  }
  __syncthreads();
  for (int ch = 0; ch < 2; ch++) {
    float maxc = 0.f;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) maxc = smax(maxc, s_max[ch][w]);
    if (maxc <= 0.f) continue;
    const float thr = maxc * min_conf;
    for (int i = threadIdx.x; i < n; i += blockDim.x)
      if (maps.conf[ch][i] < thr) {
        maps.dx[ch][i] = 0.f;
        maps.dy[ch][i] = 0.f;
      }
  }
  __syncthreads();
  float* m4[4] = {maps.dx[0], maps.dy[0], maps.dx[1], maps.dy[1]};
  for (int q = 0; q < 4; q++) {
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      const int cy = i / map_w, cx = i % map_w;
      float acc = 0.f;
      int cnt = 0;
      for (int dy = -1; dy <= 1; dy++)
        for (int dx = -1; dx <= 1; dx++) {
          const int yy = cy + dy, xx = cx + dx;
          if (yy < 0 || yy >= map_h || xx < 0 || xx >= map_w) continue;
          acc += m4[q][yy * map_w + xx];
          cnt++;
        }
      tmp[q * n + i] = cnt > 0 ? acc / (float)cnt : 0.f;
    }
  }
  __syncthreads();
  for (int q = 0; q < 4; q++)
    for (int i = threadIdx.x; i < n; i += blockDim.x) m4[q][i] = tmp[q * n + i];
}

struct ShiftMaps {
  const float* dx;
  const float* dy;
};

__device__ __forceinline__ void sample_shift(ShiftMaps m, int map_w, int map_h, float cell, float clamp_shift, float px,
                                             float py, float& out_dx, float& out_dy) {
  const float gx_f = (px / cell) - 0.5f;
  const float gy_f = (py / cell) - 0.5f;
  int gx0 = (int)floorf(gx_f);
  int gy0 = (int)floorf(gy_f);
  if (gx0 < 0) gx0 = 0;
  if (gy0 < 0) gy0 = 0;
  if (gx0 >= map_w - 1) gx0 = map_w - 2;
  if (gy0 >= map_h - 1) gy0 = map_h - 2;
  if (gx0 < 0) gx0 = 0;
  if (gy0 < 0) gy0 = 0;
  const float fx = sclamp(gx_f - gx0, 0.f, 1.f);
  const float fy = sclamp(gy_f - gy0, 0.f, 1.f);
  const int gx1 = min(gx0 + 1, map_w - 1);
  const int gy1 = min(gy0 + 1, map_h - 1);
  const float dx = (m.dx[gy0 * map_w + gx0] * (1.f - fx) + m.dx[gy0 * map_w + gx1] * fx) * (1.f - fy) +
                   (m.dx[gy1 * map_w + gx0] * (1.f - fx) + m.dx[gy1 * map_w + gx1] * fx) * fy;
  const float dy = (m.dy[gy0 * map_w + gx0] * (1.f - fx) + m.dy[gy0 * map_w + gx1] * fx) * (1.f - fy) +
                   (m.dy[gy1 * map_w + gx0] * (1.f - fx) + m.dy[gy1 * map_w + gx1] * fx) * fy;
  out_dx = sclamp(dx, -clamp_shift, clamp_shift);
  out_dy = sclamp(dy, -clamp_shift, clamp_shift);
}

__global__ void k_lk_remap(const float* __restrict__ R0, const float* __restrict__ G0, const float* __restrict__ B0,
                           float* __restrict__ dst, int W, int H, ShiftMaps mr, ShiftMaps mb, int map_w, int map_h,
                           float cell, float clamp_shift) {
  // (32 x 8) threads, 2D grid-stride: no 64-bit index division per pixel
  for (int y = blockIdx.y * blockDim.y + threadIdx.y; y < H; y += gridDim.y * blockDim.y)
  for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < W; x += gridDim.x * blockDim.x) {
    const size_t i = (size_t)y * W + x;
    float drx, dry, dbx, dby;
    sample_shift(mr, map_w, map_h, cell, clamp_shift, (float)x, (float)y, drx, dry);
    sample_shift(mb, map_w, map_h, cell, clamp_shift, (float)x, (float)y, dbx, dby);
    const float r_new = bilinear_plane(R0, W, H, (float)x + drx, (float)y + dry);
    const float b_new = bilinear_plane(B0, W, H, (float)x + dbx, (float)y + dby);
    dst[i * 3 + 0] = r_new;
    dst[i * 3 + 1] = G0[i];
    dst[i * 3 + 2] = b_new;
  }
}

__global__ void k_zero(float* p, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) p[i] = 0.f;
}

int effective_levels(size_t W0, size_t H0, int levels) {
  int e = levels;
  while (e > 1 && ((W0 >> (e - 1)) < 32 || (H0 >> (e - 1)) < 32)) e--;
  return e;
}

}  // namespace

size_t ws_bytes_lateral(size_t w, size_t h, int cell, int levels, bool in_place) {
  (void)in_place;
  if (cell < 16) cell = 16;
  if (levels < 1) levels = 1;
  size_t total = 0;
  size_t lw = w, lh = h;
  for (int l = 0; l < levels; l++) {
    total += 3 * (((lw * lh * 4) + 255) & ~size_t(255));
    lw /= 2;
    lh /= 2;
  }
  size_t mw = std::max<size_t>(2, (w + cell - 1) / cell), mh = std::max<size_t>(2, (h + cell - 1) / cell);
  total += 10 * (((mw * mh * 4) + 255) & ~size_t(255));
  return total + 4096;
}

lre_status launch_lateral_ca(Context* c, const float* in, float* out, size_t w, size_t h, int cell, int iters,
                             float max_shift, float min_conf, int levels) {
  if (cell < 16) cell = 16;
  if (iters < 1) iters = 1;
  if (levels < 1) levels = 1;
  const int eff = effective_levels(w, h, levels);
  std::vector<float*> Rl(eff), Gl(eff), Bl(eff);
  std::vector<int> Wl(eff), Hl(eff);
  Wl[0] = (int)w;
  Hl[0] = (int)h;
  for (int l = 1; l < eff; l++) {
    Wl[l] = Wl[l - 1] / 2;
    Hl[l] = Hl[l - 1] / 2;
  }
  for (int l = 0; l < eff; l++) {
    size_t n = (size_t)Wl[l] * Hl[l];
    Rl[l] = reinterpret_cast<float*>(c->ws.take(n * 4));
    Gl[l] = reinterpret_cast<float*>(c->ws.take(n * 4));
    Bl[l] = reinterpret_cast<float*>(c->ws.take(n * 4));
    if (!Rl[l] || !Gl[l] || !Bl[l]) return fail(c, LRE_ERR_OUT_OF_MEMORY, "ca_register_lateral: workspace too small");
  }
  const int map_w = (int)std::max<size_t>(2, (w + cell - 1) / cell);
  const int map_h = (int)std::max<size_t>(2, (h + cell - 1) / cell);
  const size_t ncell = (size_t)map_w * map_h;
  LkMaps maps;
  float* mapmem = reinterpret_cast<float*>(c->ws.take(10 * ncell * 4));
  if (!mapmem) return fail(c, LRE_ERR_OUT_OF_MEMORY, "ca_register_lateral: workspace too small");
  maps.dx[0] = mapmem;
  maps.dy[0] = mapmem + ncell;
  maps.conf[0] = mapmem + 2 * ncell;
  maps.dx[1] = mapmem + 3 * ncell;
  maps.dy[1] = mapmem + 4 * ncell;
  maps.conf[1] = mapmem + 5 * ncell;
  float* tmp = mapmem + 6 * ncell;

  k_split_planes<<<grid_for(w * h, 256, c->sm_count * 8), 256, 0, c->stream>>>(in, Rl[0], Gl[0], Bl[0], w * h);
  k_zero<<<grid_for(6 * ncell, 256, 64), 256, 0, c->stream>>>(mapmem, 6 * ncell);
  count_launch(c, 2);
  for (int l = 1; l < eff; l++) {
    Planes3 p{{Rl[l - 1], Gl[l - 1], Bl[l - 1]}, {Rl[l], Gl[l], Bl[l]}};
    k_downsample3<<<grid_for((size_t)Wl[l] * Hl[l], 256, c->sm_count * 8), 256, 0, c->stream>>>(p, Wl[l - 1], Hl[l - 1],
                                                                                                Wl[l], Hl[l]);
    count_launch(c);
  }
  for (int L = eff - 1; L >= 0; L--) {
    const float scale_down = 1.f / (float)(1 << L);
    const float level_max_shift = max_shift * scale_down + (float)(1 << L) * 0.5f;
    const float scale_up = (float)(1 << L);
    dim3 grid((unsigned)ncell, 2);
    k_lk_level<<<grid, LK_THREADS, 0, c->stream>>>(Gl[L], Rl[L], Bl[L], Wl[L], Hl[L], map_w, map_h, iters,
                                                   level_max_shift, scale_down, scale_up, maps);
    count_launch(c);
  }
  k_lk_gate_smooth<<<1, 1024, 0, c->stream>>>(maps, map_w, map_h, min_conf, tmp);
  const float clamp_shift = max_shift * (float)(1 << (eff - 1));
  k_lk_remap<<<dim3((unsigned)std::min<size_t>((w + 31) / 32, 1024), (unsigned)std::min<size_t>((h + 7) / 8, 8192)),
               dim3(32, 8), 0, c->stream>>>(
      Rl[0], Gl[0], Bl[0], out, (int)w, (int)h, ShiftMaps{maps.dx[0], maps.dy[0]}, ShiftMaps{maps.dx[1], maps.dy[1]},
      map_w, map_h, (float)cell, clamp_shift);
  count_launch(c, 2);
  return check_launch(c, "ca_register_lateral");
}

}  // namespace lre
