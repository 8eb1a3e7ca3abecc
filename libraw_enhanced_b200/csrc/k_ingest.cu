// k_ingest.cu -- on-device raw ingest: the LibRaw-side steps between the
// decoded raw_image and the demosaic, so a frame crosses PCIe as its 16-bit
// CFA samples (2 B/px) instead of a float mosaic.
//
// Steps and their reference (all bit-exact integer work up to the WB multiply):
//   raw2image        core/libraw_wrapper.cpp:2299-2438 (copy_bayer_image
//                    standard path, copy_xtrans_image), into uint16[4] pixels
//   black level      core/libraw_wrapper.cpp:401-491 (k_pointwise.cu)
//   green matching   core/libraw_wrapper.cpp:496-585
//   white balance    core/cpu_accelerator.cpp:2789-2869, written as the dense
//                    float mosaic the demosaic kernels read
//   adjust_maximum   core/libraw_wrapper.cpp:1010-1087
// then the develop chain (pipeline.cu) with the adopted maximum.
#include <cmath>
#include <cstring>

#include "common.cuh"
#include "lre_internal.h"

namespace lre {

namespace {

struct XtPat36 {
  char p[36];
};

__device__ __forceinline__ unsigned ingest_fcol(unsigned row, unsigned col, uint32_t filters, const XtPat36& xt) {
  return filters == LRE_FILTERS_XTRANS ? (unsigned)xt.p[((row + 6) % 6) * 6 + (col + 6) % 6]
                                       : fcol_native(row, col, filters);
}

// One thread per image4 pixel; with shrink the 2x2 source cell is written in
// the reference's row-major order (later samples overwrite earlier ones).
__global__ void k_raw2image(const uint16_t* __restrict__ raw, int raw_width, int raw_height, size_t pitch_px,
                            int top, int left, int width, int height, int shrink, uint32_t filters, XtPat36 xt,
                            ushort4* __restrict__ image4, int iwidth, int iheight) {
  const size_t n = (size_t)iwidth * iheight;
  const bool is_xt = filters == LRE_FILTERS_XTRANS;
  const int row_lim = min(height, raw_height - top), col_lim = min(width, raw_width - left);
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
    const int dy = (int)(q / iwidth), dx = (int)(q % iwidth);
    unsigned short v[4] = {0, 0, 0, 0};
    const int span = 1 << shrink;
    for (int sy = 0; sy < span; sy++) {
      const int row = (dy << shrink) + sy;
      if (row >= row_lim) break;
      for (int sx = 0; sx < span; sx++) {
        const int col = (dx << shrink) + sx;
        if (col >= col_lim) break;
        const size_t src_row = (size_t)(row + top), src_col = (size_t)(col + left);
        const size_t src = is_xt ? src_row * (size_t)raw_width + src_col : src_row * pitch_px + src_col;
        const unsigned short val = raw[src];
        const unsigned c = ingest_fcol((unsigned)row, (unsigned)col, filters, xt);
        v[c] = val;
        if (!is_xt && c == 3) v[1] = val;
      }
    }
    image4[q] = make_ushort4(v[0], v[1], v[2], v[3]);
  }
}

// Fuji SuperCCD honeycomb raw2image (core/libraw_wrapper.cpp:2342-2392).
// The reference scatters raw (row, col) onto the 45-degree frame; here one
// thread owns one image4 pixel and inverts the map for each frame site
// (r, c) that lands on it (one site, or the 2x2 cell when shrinking):
//   fuji_layout: r + c = fuji_width - 1 + row,  col = c - (row + 1) / 2
//   otherwise:   c - r = col - fuji_width + 1,   row = c - (col + 1) / 2
// Where several samples land on one pixel, the one latest in the
// reference's row-major (row, col) scan wins, per channel.
__global__ void k_raw2image_fuji(const uint16_t* __restrict__ raw, int raw_width, int raw_height, size_t pitch_px,
                                 int top, int left, int width, int height, int shrink, uint32_t filters,
                                 int fuji_width, int fuji_layout, ushort4* __restrict__ image4, int iwidth,
                                 int iheight) {
  const size_t n = (size_t)iwidth * iheight;
  const int copy_rows = max(0, raw_height - top * 2);
  const int copy_cols = fuji_width << (fuji_layout ? 0 : 1);
  const int span = 1 << shrink;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
    const int R = (int)(q / iwidth), Cc = (int)(q % iwidth);
    unsigned short v[4] = {0, 0, 0, 0};
    long long key[4] = {-1, -1, -1, -1};
    for (int sy = 0; sy < span; sy++) {
      const int r = (R << shrink) + sy;
      if (r >= height) break;
      for (int sx = 0; sx < span; sx++) {
        const int c = (Cc << shrink) + sx;
        if (c >= width) break;
        int row, col;
        if (fuji_layout) {
          row = r + c - fuji_width + 1;
          if (row < 0) continue;
          col = c - ((row + 1) >> 1);
        } else {
          col = c - r + fuji_width - 1;
          if (col < 0) continue;
          row = c - ((col + 1) >> 1);
        }
        if (row < 0 || row >= copy_rows || col < 0 || col >= copy_cols) continue;
        const int src_row = row + top, src_col = col + left;
        if (src_row >= raw_height || src_col >= raw_width) continue;
        const long long k = (long long)row * copy_cols + col;
        const unsigned short val = raw[(size_t)src_row * pitch_px + src_col];
        const unsigned ch = fcol_native((unsigned)r, (unsigned)c, filters);
        if (k > key[ch]) {
          key[ch] = k;
          v[ch] = val;
        }
        if (ch == 3 && k > key[1]) {
          key[1] = k;
          v[1] = val;
        }
      }
    }
    image4[q] = make_ushort4(v[0], v[1], v[2], v[3]);
  }
}

// The Fuji rotate (core/libraw_wrapper.cpp:1709-1750): one thread per output
// pixel; the sample position in double then float, the bilinear weights in
// float, as the reference computes them.
__global__ void k_fuji_rotate(const float* __restrict__ rgb, size_t w, size_t h, int fuji_width, float* __restrict__ out,
                              size_t wide, size_t high) {
  const double step = sqrt(0.5);
  const size_t n = wide * high;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
    const size_t row = q / wide, col = q % wide;
    const float r = (float)(fuji_width + ((double)row - (double)col) * step);
    const float c = (float)(((double)row + (double)col) * step);
    const size_t ur = (size_t)r, uc = (size_t)c;
    float* dst = out + q * 3;
    if (ur >= h - 1 || uc >= w - 1) {
      dst[0] = dst[1] = dst[2] = 0.f;
      continue;
    }
    const float fr = r - (float)ur, fc = c - (float)uc;
    const float* p00 = rgb + (ur * w + uc) * 3;
    const float* p01 = rgb + (ur * w + uc + 1) * 3;
    const float* p10 = rgb + ((ur + 1) * w + uc) * 3;
    const float* p11 = rgb + ((ur + 1) * w + uc + 1) * 3;
#pragma unroll
    for (int ch = 0; ch < 3; ++ch) {
      const float top = p00[ch] * (1.0f - fc) + p01[ch] * fc;
      const float bottom = p10[ch] * (1.0f - fc) + p11[ch] * fc;
      dst[ch] = top * (1.0f - fr) + bottom * fr;
    }
  }
}

// One thread per G2 candidate (rows 3, 5, ..., columns 2, 4, ...), reading
// the pre-matching copy, writing channel 3 of the image.
__global__ void k_green_matching(const ushort4* __restrict__ img, ushort4* __restrict__ out, int width, int height,
                                 int maximum) {
  const int margin = 3;
  const float thr = 0.01f;
  const int nj = (height - margin - 3 + 1) / 2, ni = (width - margin - 2 + 1) / 2;
  if (nj <= 0 || ni <= 0) return;
  const size_t n = (size_t)nj * ni;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
    const int j = 3 + 2 * (int)(q / ni), i = 2 + 2 * (int)(q % ni);
    if (j - 1 < 0 || j + 1 >= height || i - 1 < 0 || i + 1 >= width || j - 2 < 0 || j + 2 >= height || i - 2 < 0 ||
        i + 2 >= width)
      continue;
    const int o1_1 = img[(size_t)(j - 1) * width + i - 1].y;
    const int o1_2 = img[(size_t)(j - 1) * width + i + 1].y;
    const int o1_3 = img[(size_t)(j + 1) * width + i - 1].y;
    const int o1_4 = img[(size_t)(j + 1) * width + i + 1].y;
    const int o2_1 = img[(size_t)(j - 2) * width + i].w;
    const int o2_2 = img[(size_t)(j + 2) * width + i].w;
    const int o2_3 = img[(size_t)j * width + i - 2].w;
    const int o2_4 = img[(size_t)j * width + i + 2].w;
    const double m1 = (o1_1 + o1_2 + o1_3 + o1_4) / 4.0;
    const double m2 = (o2_1 + o2_2 + o2_3 + o2_4) / 4.0;
    const double c1 = (abs(o1_1 - o1_2) + abs(o1_1 - o1_3) + abs(o1_1 - o1_4) + abs(o1_2 - o1_3) + abs(o1_3 - o1_4) +
                       abs(o1_2 - o1_4)) / 6.0;
    const double c2 = (abs(o2_1 - o2_2) + abs(o2_1 - o2_3) + abs(o2_1 - o2_4) + abs(o2_2 - o2_3) + abs(o2_3 - o2_4) +
                       abs(o2_2 - o2_4)) / 6.0;
    const size_t at = (size_t)j * width + i;
    const int g2 = img[at].w;
    if ((g2 < maximum * 0.95) && (c1 < maximum * thr) && (c2 < maximum * thr) && (m2 > 0.1)) {
      const float correction = g2 * m1 / m2;
      out[at].w = correction > maximum ? (unsigned short)maximum : (unsigned short)correction;
    }
  }
}

// White balance into the dense mosaic: each site's own sample times its
// channel's multiplier (what apply_white_balance stores in the site's
// channel of the sparse buffer).
__global__ void k_wb_dense(const ushort4* __restrict__ raw4, float* __restrict__ dense, int w, int h, float4 wb,
                           uint32_t filters, XtPat36 xt) {
  const size_t n = (size_t)w * h;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const unsigned row = (unsigned)(i / w), col = (unsigned)(i % w);
    const unsigned c = ingest_fcol(row, col, filters, xt);
    const ushort4 r = raw4[i];
    const unsigned short v = c == 0 ? r.x : c == 1 ? r.y : c == 2 ? r.z : r.w;
    const float m = c == 0 ? wb.x : c == 1 ? wb.y : c == 2 ? wb.z : wb.w;
    dense[i] = (float)v * m;
  }
}

// adjust_maximum's scan of the sparse buffer at channel fcol_bayer(row, col,
// filters): the dense sample where that channel is the site's own channel,
// 0 where it is not (the X-Trans case; for Bayer they always agree).
__global__ void k_cfa_max_dense(const float* __restrict__ dense, int w, int h, uint32_t filters, XtPat36 xt,
                                float* out) {
  const size_t n = (size_t)w * h;
  float m = 0.f;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const unsigned row = (unsigned)(i / w), col = (unsigned)(i % w);
    unsigned own = ingest_fcol(row, col, filters, xt);
    if (own == 3) own = 1;
    const float v = own == fcol3(row, col, filters) ? dense[i] : 0.f;
    if (v > m) m = v;
  }
  m = warp_max(m);
  if ((threadIdx.x & 31) == 0) atomic_max_float(out, m);
}

XtPat36 make_pat(const char* xtrans) {
  XtPat36 x{};
  if (xtrans) memcpy(x.p, xtrans, 36);
  return x;
}

}  // namespace

// Elements of raw_image the frame covers (X-Trans rows are raw_width apart,
// Bayer rows raw_pitch bytes apart).
size_t raw_image_elems(const lre_raw_frame& f) {
  return f.raw_height * (f.filters == LRE_FILTERS_XTRANS ? f.raw_width : f.raw_pitch / 2);
}

bool fuji_honeycomb(const lre_raw_frame& f) { return f.fuji_width > 0 && f.filters >= 1000; }

// fuji_width' and the rotated size (core/libraw_wrapper.cpp:1710-1718);
// false when the reference leaves the image as it is.
bool fuji_rotate_size(int fuji_width_io, int shrink, size_t h, int* fw, size_t* wide, size_t* high) {
  *fw = (fuji_width_io - 1 + shrink) >> shrink;
  if (*fw <= 0) return false;
  const double step = std::sqrt(0.5);
  const int wide_i = static_cast<int>(*fw / step);
  const int high_i = static_cast<int>((static_cast<int>(h) - *fw) / step);
  if (wide_i <= 1 || high_i <= 1) return false;
  *wide = (size_t)wide_i;
  *high = (size_t)high_i;
  return true;
}

lre_status launch_fuji_rotate(Context* c, const float* in, size_t w, size_t h, int fuji_width_io, int shrink,
                              float* out) {
  int fw;
  size_t wide, high;
  if (!fuji_rotate_size(fuji_width_io, shrink, h, &fw, &wide, &high))
    return fail(c, LRE_ERR_INVALID_ARGUMENT, "fuji_rotate: the reference leaves this image unrotated");
  k_fuji_rotate<<<grid_for(wide * high, 256, c->sm_count * 8), 256, 0, c->stream>>>(in, w, h, fw, out, wide, high);
  count_launch(c);
  return check_launch(c, "fuji_rotate");
}

lre_status launch_raw2image(Context* c, const uint16_t* raw, const lre_raw_frame& f, uint16_t* image4) {
  const uint32_t filters = f.filters;
  const char* xtrans = f.xtrans;
  const int shrink = f.shrink ? 1 : 0;
  const size_t iw = (f.width + shrink) >> shrink, ih = (f.height + shrink) >> shrink;
  if (fuji_honeycomb(f)) {
    k_raw2image_fuji<<<grid_for(iw * ih, 256, c->sm_count * 8), 256, 0, c->stream>>>(
        raw, (int)f.raw_width, (int)f.raw_height, f.raw_pitch / 2, (int)f.top_margin, (int)f.left_margin,
        (int)f.width, (int)f.height, shrink, filters, f.fuji_width, f.fuji_layout ? 1 : 0,
        reinterpret_cast<ushort4*>(image4), (int)iw, (int)ih);
    count_launch(c);
    return check_launch(c, "raw2image (Fuji honeycomb)");
  }
  k_raw2image<<<grid_for(iw * ih, 256, c->sm_count * 8), 256, 0, c->stream>>>(
      raw, (int)f.raw_width, (int)f.raw_height, f.raw_pitch / 2, (int)f.top_margin, (int)f.left_margin,
      (int)f.width, (int)f.height, shrink, filters, make_pat(xtrans), reinterpret_cast<ushort4*>(image4), (int)iw,
      (int)ih);
  count_launch(c);
  return check_launch(c, "raw2image");
}

lre_status launch_green_matching(Context* c, uint16_t* raw4, const uint16_t* copy, size_t w, size_t h,
                                 uint32_t filters, unsigned maximum) {
  if (filters == LRE_FILTERS_XTRANS) return LRE_OK;
  LRE_CUDA_TRY(c, cudaMemcpyAsync(const_cast<uint16_t*>(copy), raw4, w * h * 8, cudaMemcpyDeviceToDevice, c->stream));
  k_green_matching<<<grid_for(w * h / 4 + 1, 256, c->sm_count * 8), 256, 0, c->stream>>>(
      reinterpret_cast<const ushort4*>(copy), reinterpret_cast<ushort4*>(raw4), (int)w, (int)h, (int)maximum);
  count_launch(c);
  return check_launch(c, "green_matching");
}

lre_status launch_wb_dense(Context* c, const uint16_t* raw4, float* dense, size_t w, size_t h, const float wb[4],
                           uint32_t filters, const char* xtrans) {
  k_wb_dense<<<grid_for(w * h, 256, c->sm_count * 8), 256, 0, c->stream>>>(
      reinterpret_cast<const ushort4*>(raw4), dense, (int)w, (int)h, make_float4(wb[0], wb[1], wb[2], wb[3]), filters,
      make_pat(xtrans));
  count_launch(c);
  return check_launch(c, "white_balance (dense)");
}

lre_status launch_cfa_max_dense(Context* c, const float* dense, size_t w, size_t h, uint32_t filters,
                                const char* xtrans, float* d_out) {
  LRE_CUDA_TRY(c, cudaMemsetAsync(d_out, 0, sizeof(float), c->stream));
  k_cfa_max_dense<<<grid_for(w * h, 256, c->sm_count * 4), 256, 0, c->stream>>>(dense, (int)w, (int)h, filters,
                                                                                make_pat(xtrans), d_out);
  count_launch(c);
  return check_launch(c, "adjust_maximum scan");
}

}  // namespace lre

// ------------------------------------------------------------------ C ABI
using lre::Context;

namespace {

Context* CX(lre_ctx* p) { return reinterpret_cast<Context*>(p); }

lre_status check_frame(Context* c, const lre_raw_frame* f) {
  if (!f) return lre::fail(c, LRE_ERR_INVALID_ARGUMENT, "raw frame: null");
  if (f->width == 0 || f->height == 0 || f->raw_width == 0 || f->raw_height == 0)
    return lre::fail(c, LRE_ERR_INVALID_ARGUMENT, "raw frame: empty image");
  if (f->top_margin >= f->raw_height || f->left_margin >= f->raw_width)
    return lre::fail(c, LRE_ERR_INVALID_ARGUMENT, "raw frame: margins outside raw_image");
  if (f->filters != LRE_FILTERS_XTRANS && (f->raw_pitch < 2 * f->raw_width || (f->raw_pitch & 1)))
    return lre::fail(c, LRE_ERR_INVALID_ARGUMENT, "raw frame: raw_pitch must be an even byte count >= 2 * raw_width");
  if (f->filters != LRE_FILTERS_XTRANS && f->filters < 1000)
    return lre::fail(c, LRE_ERR_INVALID_ARGUMENT, "raw frame: filters is neither a Bayer word nor X-Trans");
  if (f->cblack[4] * f->cblack[5] > 36)
    return lre::fail(c, LRE_ERR_INVALID_ARGUMENT, "raw frame: positional black pattern larger than 6x6");
  if (f->width > (1u << 20) || f->height > (1u << 20)) return lre::fail(c, LRE_ERR_INVALID_ARGUMENT, "raw frame: too large");
  if (f->fuji_width < 0 || f->fuji_width > 65535)
    return lre::fail(c, LRE_ERR_INVALID_ARGUMENT, "raw frame: fuji_width outside LibRaw's 16-bit range");
  return LRE_OK;
}

// adjust_maximum's adoption rule (core/libraw_wrapper.cpp:1010-1087).
float adopt_maximum(float threshold, float real_max, float maximum) {
  if (threshold < 0.00001f) return maximum;
  const float thr = threshold > 0.99999f ? 0.75f : threshold;
  if (real_max > 0 && real_max < maximum && real_max > maximum * thr) return real_max;
  return maximum;
}

// Ingest + develop on device buffers.  Synchronises once when the maximum is
// scanned (the demosaic is parameterised by it).
lre_status develop_raw_device(Context* c, const uint16_t* d_raw, const lre_raw_frame& f, void* d_out,
                              const lre_develop_params& p_in, float* maximum_used) {
  const int shrink = f.shrink ? 1 : 0;
  const size_t iw = (f.width + shrink) >> shrink, ih = (f.height + shrink) >> shrink;
  lre_develop_params p = p_in;
  p.filters = f.filters;
  memcpy(p.xtrans, f.xtrans, 36);
  LRE_TRY(lre::develop_validate(c, &p, iw, ih));
  const size_t n = iw * ih;
  const size_t a4 = (n * 8 + 255) & ~size_t(255), mos = (n * 4 + 255) & ~size_t(255);
  // ingest buffers sit above the develop chain's workspace: reserve both,
  // then take the ingest part from the top of a separate arena region
  const size_t chain = lre::develop_ws_bytes(p, iw, ih);
  c->ws.reset();
  LRE_CUDA_TRY(c, c->ws.reserve(chain + 2 * a4 + mos + 4096, c->stream));
  (void)c->ws.take(chain);  // the chain's region (develop_device rewinds to 0 and re-takes it)
  uint16_t* img4 = reinterpret_cast<uint16_t*>(c->ws.take(a4));
  uint16_t* copy = reinterpret_cast<uint16_t*>(c->ws.take(a4));
  float* dense = reinterpret_cast<float*>(c->ws.take(mos));
  if (!img4 || !copy || !dense) return lre::fail(c, LRE_ERR_OUT_OF_MEMORY, "develop_raw: workspace too small");
  LRE_TRY(lre::launch_raw2image(c, d_raw, f, img4));
  LRE_TRY(lre::launch_black_level(c, img4, iw, ih, f.cblack, 6 + (size_t)f.cblack[4] * f.cblack[5], f.black, f.maximum));
  if (f.green_matching) LRE_TRY(lre::launch_green_matching(c, img4, copy, iw, ih, f.filters, f.maximum));
  // scale_colors (core/libraw_wrapper.cpp:1545-1553) sits between green
  // matching and the white balance; it also lowers color.maximum by black,
  // which adjust_maximum then compares against
  float wb[4] = {f.wb[0], f.wb[1], f.wb[2], f.wb[3]};
  float maximum = (float)f.maximum;
  if (f.derive_wb) {
    lre_wb_result r;
    LRE_TRY(lre::derive_wb_device(c, img4, iw, ih, f.filters, f.xtrans, f.maximum, f.black, f.wb_in, &r));
    for (int k = 0; k < 4; k++) wb[k] = r.scale_mul[k];
    maximum = (float)r.maximum;
  }
  LRE_TRY(lre::launch_wb_dense(c, img4, dense, iw, ih, wb, f.filters, f.xtrans));
  if (f.adjust_maximum_thr >= 0.00001f) {
    float real_max = f.data_maximum;
    if (real_max == 0.f) {
      float* d_m = c->d_scalars + 8;
      LRE_TRY(lre::launch_cfa_max_dense(c, dense, iw, ih, f.filters, f.xtrans, d_m));
      LRE_CUDA_TRY(c, cudaMemcpyAsync(&real_max, d_m, sizeof(float), cudaMemcpyDeviceToHost, c->stream));
      LRE_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    }
    maximum = adopt_maximum(f.adjust_maximum_thr, real_max, maximum);
  }
  if (maximum_used) *maximum_used = maximum;
  p.maximum_value = maximum;
  // develop_device resets the arena and re-takes from offset 0, i.e. within
  // the chain region reserved above, so the ingest buffers stay intact
  return lre::develop_device(c, dense, d_out, iw, ih, p);
}

}  // namespace

extern "C" {

lre_status lre_raw2image(lre_ctx* ctx, const uint16_t* raw_image, const lre_raw_frame* f, uint16_t* image4) {
  Context* c = CX(ctx);
  if (!c) return LRE_ERR_INVALID_ARGUMENT;
  if (!raw_image || !image4) return lre::fail(c, LRE_ERR_INVALID_ARGUMENT, "raw2image: null buffer");
  LRE_TRY(check_frame(c, f));
  std::lock_guard<std::mutex> lk(c->mu);
  cudaSetDevice(c->device);
  LRE_TRY(lre::check_injection(c));
  const int shrink = f->shrink ? 1 : 0;
  const size_t n_in = lre::raw_image_elems(*f);
  const size_t n_out = ((f->width + shrink) >> shrink) * ((f->height + shrink) >> shrink) * 4;
  LRE_TRY(lre::ensure_buffer(c, &c->d_in, &c->d_in_cap, n_in * 2));
  LRE_TRY(lre::ensure_buffer(c, &c->d_out, &c->d_out_cap, n_out * 2));
  LRE_TRY(lre::copy_h2d(c, c->d_in, raw_image, n_in * 2, c->stream));
  LRE_TRY(lre::launch_raw2image(c, reinterpret_cast<const uint16_t*>(c->d_in), *f, reinterpret_cast<uint16_t*>(c->d_out)));
  LRE_TRY(lre::copy_d2h(c, image4, c->d_out, n_out * 2, c->stream));
  LRE_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  return LRE_OK;
}

lre_status lre_green_matching(lre_ctx* ctx, uint16_t* raw4, size_t width, size_t height, uint32_t filters,
                              unsigned maximum) {
  Context* c = CX(ctx);
  if (!c) return LRE_ERR_INVALID_ARGUMENT;
  if (!raw4 || width == 0 || height == 0) return lre::fail(c, LRE_ERR_INVALID_ARGUMENT, "green_matching: bad image");
  std::lock_guard<std::mutex> lk(c->mu);
  cudaSetDevice(c->device);
  LRE_TRY(lre::check_injection(c));
  const size_t bytes = width * height * 8;
  LRE_TRY(lre::ensure_buffer(c, &c->d_in, &c->d_in_cap, bytes));
  LRE_TRY(lre::ensure_buffer(c, &c->d_out, &c->d_out_cap, bytes));
  LRE_TRY(lre::copy_h2d(c, c->d_in, raw4, bytes, c->stream));
  LRE_TRY(lre::launch_green_matching(c, reinterpret_cast<uint16_t*>(c->d_in), reinterpret_cast<uint16_t*>(c->d_out),
                                     width, height, filters, maximum));
  LRE_TRY(lre::copy_d2h(c, raw4, c->d_in, bytes, c->stream));
  LRE_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  return LRE_OK;
}

lre_status lre_fuji_rotate_size(int fuji_width, int shrink, size_t width, size_t height, size_t* out_w,
                                size_t* out_h) {
  (void)width;
  if (!out_w || !out_h) return LRE_ERR_INVALID_ARGUMENT;
  int fw;
  if (!lre::fuji_rotate_size(fuji_width, shrink ? 1 : 0, height, &fw, out_w, out_h)) *out_w = *out_h = 0;
  return LRE_OK;
}

lre_status lre_dev_fuji_rotate(lre_ctx* ctx, const float* in, size_t width, size_t height, int fuji_width, int shrink,
                               float* out) {
  Context* c = CX(ctx);
  if (!c) return LRE_ERR_INVALID_ARGUMENT;
  if (!in || !out || width < 2 || height < 2) return lre::fail(c, LRE_ERR_INVALID_ARGUMENT, "fuji_rotate: bad image");
  cudaSetDevice(c->device);
  LRE_TRY(lre::check_injection(c));
  return lre::launch_fuji_rotate(c, in, width, height, fuji_width, shrink ? 1 : 0, out);
}

lre_status lre_fuji_rotate(lre_ctx* ctx, const float* in, size_t width, size_t height, int fuji_width, int shrink,
                           float* out) {
  Context* c = CX(ctx);
  if (!c) return LRE_ERR_INVALID_ARGUMENT;
  if (!in || !out || width < 2 || height < 2) return lre::fail(c, LRE_ERR_INVALID_ARGUMENT, "fuji_rotate: bad image");
  int fw;
  size_t wide, high;
  if (!lre::fuji_rotate_size(fuji_width, shrink ? 1 : 0, height, &fw, &wide, &high))
    return lre::fail(c, LRE_ERR_INVALID_ARGUMENT, "fuji_rotate: the reference leaves this image unrotated");
  std::lock_guard<std::mutex> lk(c->mu);
  cudaSetDevice(c->device);
  LRE_TRY(lre::check_injection(c));
  const size_t in_bytes = width * height * 12, out_bytes = wide * high * 12;
  LRE_TRY(lre::ensure_buffer(c, &c->d_in, &c->d_in_cap, in_bytes));
  LRE_TRY(lre::ensure_buffer(c, &c->d_out, &c->d_out_cap, out_bytes));
  LRE_TRY(lre::copy_h2d(c, c->d_in, in, in_bytes, c->stream));
  LRE_TRY(lre::launch_fuji_rotate(c, reinterpret_cast<const float*>(c->d_in), width, height, fuji_width,
                                  shrink ? 1 : 0, reinterpret_cast<float*>(c->d_out)));
  LRE_TRY(lre::copy_d2h(c, out, c->d_out, out_bytes, c->stream));
  LRE_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  return LRE_OK;
}

lre_status lre_dev_develop_raw(lre_ctx* ctx, const uint16_t* raw_image, const lre_raw_frame* f, void* out,
                               const lre_develop_params* params, float* maximum_used) {
  Context* c = CX(ctx);
  if (!c) return LRE_ERR_INVALID_ARGUMENT;
  if (!raw_image || !out || !params) return lre::fail(c, LRE_ERR_INVALID_ARGUMENT, "develop_raw: null argument");
  LRE_TRY(check_frame(c, f));
  cudaSetDevice(c->device);
  LRE_TRY(lre::check_injection(c));
  return develop_raw_device(c, raw_image, *f, out, *params, maximum_used);
}

lre_status lre_develop_raw(lre_ctx* ctx, const uint16_t* raw_image, const lre_raw_frame* f, void* out,
                           const lre_develop_params* params, float* maximum_used) {
  Context* c = CX(ctx);
  if (!c) return LRE_ERR_INVALID_ARGUMENT;
  if (!raw_image || !out || !params) return lre::fail(c, LRE_ERR_INVALID_ARGUMENT, "develop_raw: null argument");
  LRE_TRY(check_frame(c, f));
  std::lock_guard<std::mutex> lk(c->mu);
  cudaSetDevice(c->device);
  LRE_TRY(lre::check_injection(c));
  const int shrink = f->shrink ? 1 : 0;
  const size_t iw = (f->width + shrink) >> shrink, ih = (f->height + shrink) >> shrink;
  const size_t n_in = lre::raw_image_elems(*f);
  const size_t out_bytes = iw * ih * 3 * (params->output_bits == 16 ? 2 : 4);
  LRE_TRY(lre::ensure_buffer(c, &c->d_in, &c->d_in_cap, n_in * 2));
  LRE_TRY(lre::ensure_buffer(c, &c->d_out, &c->d_out_cap, out_bytes));
  LRE_TRY(lre::copy_h2d(c, c->d_in, raw_image, n_in * 2, c->stream));
  LRE_TRY(develop_raw_device(c, reinterpret_cast<const uint16_t*>(c->d_in), *f, c->d_out, *params, maximum_used));
  LRE_TRY(lre::copy_d2h(c, out, c->d_out, out_bytes, c->stream));
  LRE_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  return LRE_OK;
}

}  // extern "C"
