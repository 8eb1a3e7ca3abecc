// k_linear.cu -- bilinear Bayer demosaic (CPUAccelerator::demosaic_bayer_linear,
// core/cpu_accelerator.cpp:74-156; GPUAccelerator::demosaic_bayer_linear,
// core/gpu_accelerator.h:29-32).
//
// Every site's own colour is its sample / maximum; in the interior each
// missing colour is the mean of that colour's diagonal neighbours, or, when
// no diagonal neighbour has it, of the 8-neighbourhood's samples of it (each
// sample divided by maximum before summing, as the reference does); then the
// 1-px frame is filled by the LibRaw border interpolation.  One thread per
// pixel; the interior reads only the mosaic, so there is no ordering.
#include <algorithm>

#include "common.cuh"
#include "lre_internal.h"

namespace lre {

namespace {

__device__ __forceinline__ float lin_raw(const float* __restrict__ raw, int cstride, int x, int y, int W, unsigned c) {
  const size_t i = (size_t)y * W + x;
  return cstride == 1 ? raw[i] : raw[i * 3 + c];
}

// (32 x 8) threads per block, grid-strided over rows; along x a block
// covers 64 columns and each thread takes two of them of the same parity in
// two half-passes, so a warp's lanes see one Bayer colour at a time and take
// the same branches.
__global__ void __launch_bounds__(256) k_bayer_linear(const float* __restrict__ raw, int cstride,
                                                      float* __restrict__ rgb, int W, int H, uint32_t filters,
                                                      float maximum) {
  for (int row = blockIdx.y * blockDim.y + threadIdx.y; row < H; row += gridDim.y * blockDim.y)
  for (int half = 0; half < 2; half++)
  for (int col = 2 * (blockIdx.x * blockDim.x + threadIdx.x) + half; col < W; col += 2 * gridDim.x * blockDim.x) {
    const size_t i = (size_t)row * W + col;
    const unsigned color = fcol3((unsigned)row, (unsigned)col, filters);
    float* o = rgb + i * 3;
    o[color] = lin_raw(raw, cstride, col, row, W, color) / maximum;
    if (row < 1 || row >= H - 1 || col < 1 || col >= W - 1) continue;
    for (unsigned c = 0; c < 3; c++) {
      if (c == color) continue;
      float sum = 0.0f;
      int count = 0;
      for (int dy = -1; dy <= 1; dy += 2)
        for (int dx = -1; dx <= 1; dx += 2) {
          const int ny = row + dy, nx = col + dx;
          if (fcol3((unsigned)ny, (unsigned)nx, filters) == c) {
            sum += lin_raw(raw, cstride, nx, ny, W, c) / maximum;
            count++;
          }
        }
      if (count == 0) {
        for (int dy = -1; dy <= 1; dy++)
          for (int dx = -1; dx <= 1; dx++) {
            if (dy == 0 && dx == 0) continue;
            const int ny = row + dy, nx = col + dx;
            if (fcol3((unsigned)ny, (unsigned)nx, filters) == c) {
              sum += lin_raw(raw, cstride, nx, ny, W, c) / maximum;
              count++;
            }
          }
      }
      if (count > 0) o[c] = sum / count;
    }
  }
}

}  // namespace

lre_status launch_bayer_linear(Context* c, const float* raw, int raw_c_stride, float* rgb, size_t w, size_t h,
                               uint32_t filters, float maximum_value) {
  const dim3 blk(32, 8);
  const dim3 grd((unsigned)std::min<size_t>((w + 63) / 64, 1024), (unsigned)std::min<size_t>((h + 7) / 8, 8192));
  k_bayer_linear<<<grd, blk, 0, c->stream>>>(raw, raw_c_stride, rgb, (int)w, (int)h, filters, maximum_value);
  count_launch(c);
  LRE_TRY(check_launch(c, "demosaic_bayer_linear"));
  return launch_border_interp(c, rgb, w, h, filters, 1);
}

}  // namespace lre
