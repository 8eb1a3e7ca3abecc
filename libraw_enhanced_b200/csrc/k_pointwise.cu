// k_pointwise.cu -- streaming stages: ACES tone map, white balance, black
// level, CFA packing, quantisation and the global reductions (max G, max CFA
// sample).  All are HBM-bound: grid-stride loops, 16-byte vector accesses
// where the pointers allow, grids sized to a multiple of the SM count.
#include "common.cuh"
#include "lre_internal.h"

namespace lre {

__global__ void k_tone_mapping_v4(const float4* __restrict__ in, float4* __restrict__ out, size_t n4,
                                  float s) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n4; i += (size_t)gridDim.x * blockDim.x) {
    float4 v = in[i];
    v.x = aces(v.x) * s;
    v.y = aces(v.y) * s;
    v.z = aces(v.z) * s;
    v.w = aces(v.w) * s;
    out[i] = v;
  }
}

__global__ void k_tone_mapping_s(const float* in, float* out, size_t begin, size_t n, float s) {
  for (size_t i = begin + blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    out[i] = aces(in[i]) * s;
}

lre_status launch_tone_mapping(Context* c, const float* in, float* out, size_t n_px, float after_scale) {
  size_t n = n_px * 3;
  bool aligned = ((reinterpret_cast<uintptr_t>(in) | reinterpret_cast<uintptr_t>(out)) & 15) == 0;
  size_t n4 = aligned ? n / 4 : 0;
  unsigned grid = grid_for(n4 ? n4 : n, 256, c->sm_count * 8);
  if (n4) {
    k_tone_mapping_v4<<<grid, 256, 0, c->stream>>>(reinterpret_cast<const float4*>(in),
                                                   reinterpret_cast<float4*>(out), n4, after_scale);
    count_launch(c);
  }
  if (n4 * 4 < n) {
    k_tone_mapping_s<<<aligned ? 1 : grid, 256, 0, c->stream>>>(in, out, n4 * 4, n, after_scale);
    count_launch(c);
  }
  return check_launch(c, "tone_mapping");
}

// White balance, core/cpu_accelerator.cpp:2808-2869: only each site's own
// channel of the float RGB buffer is written.
struct XTransPat {
  char p[36];
};

__global__ void k_white_balance(const ushort4* __restrict__ raw4, float* __restrict__ rgb, int w, int h,
                                float4 wb, uint32_t filters, XTransPat xt) {
  size_t n = (size_t)w * h;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    unsigned row = (unsigned)(i / w), col = (unsigned)(i % w);
    unsigned c = filters == LRE_FILTERS_XTRANS ? (unsigned)xt.p[(row % 6) * 6 + col % 6]
                                               : fcol_native(row, col, filters);
    ushort4 r = raw4[i];
    unsigned short v = c == 0 ? r.x : c == 1 ? r.y : c == 2 ? r.z : r.w;
    float m = c == 0 ? wb.x : c == 1 ? wb.y : c == 2 ? wb.z : wb.w;
    float out = (float)v * m;
    if (c == 3) c = 1;
    rgb[i * 3 + c] = out;
  }
}

lre_status launch_white_balance(Context* c, const uint16_t* raw4, float* rgb, size_t w, size_t h,
                                const float wb[4], uint32_t filters, const char* xtrans) {
  XTransPat xt{};
  if (xtrans) memcpy(xt.p, xtrans, 36);
  k_white_balance<<<grid_for(w * h, 256, c->sm_count * 8), 256, 0, c->stream>>>(
      reinterpret_cast<const ushort4*>(raw4), rgb, (int)w, (int)h, make_float4(wb[0], wb[1], wb[2], wb[3]),
      filters, xt);
  count_launch(c);
  return check_launch(c, "white_balance");
}

// Black level, core/libraw_wrapper.cpp:401-491 (bit-exact integer path).
__global__ void k_black_level(ushort4* raw4, int w, int h, const unsigned* __restrict__ cb, int mode,
                              unsigned black, int maximum) {
  size_t n = (size_t)w * h;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
    ushort4 v = raw4[q];
    int sub[4];
    if (mode == 2) {
      int row = (int)(q / w), col = (int)(q % w);
      int pos = (int)cb[6 + (row % cb[4]) * cb[5] + (col % cb[5])];
      for (int c = 0; c < 4; c++) sub[c] = pos + (int)cb[c];
    } else if (mode == 1) {
      for (int c = 0; c < 4; c++) sub[c] = (int)cb[c];
    } else {
      for (int c = 0; c < 4; c++) sub[c] = (int)black;
    }
    int x[4] = {v.x, v.y, v.z, v.w};
    for (int c = 0; c < 4; c++) {
      int t = x[c] - sub[c];
      if (t < 0) t = 0;
      if (t > maximum) t = maximum;
      x[c] = t;
    }
    raw4[q] = make_ushort4((unsigned short)x[0], (unsigned short)x[1], (unsigned short)x[2], (unsigned short)x[3]);
  }
}

lre_status launch_black_level(Context* c, uint16_t* raw4, size_t w, size_t h, const unsigned* cblack,
                              size_t cblack_len, unsigned black, unsigned maximum) {
  unsigned cb[6] = {0, 0, 0, 0, 0, 0};
  for (size_t i = 0; i < 6 && i < cblack_len; i++) cb[i] = cblack[i];
  int mode = (cb[4] && cb[5]) ? 2 : ((cb[0] || cb[1] || cb[2] || cb[3]) ? 1 : 0);
  unsigned* d_cb = nullptr;
  size_t need = 6;
  if (mode == 2) {
    need = 6 + (size_t)cb[4] * cb[5];
    if (cblack_len < need) return fail(c, LRE_ERR_INVALID_ARGUMENT, "cblack pattern shorter than cblack[4]*cblack[5]");
  }
  d_cb = reinterpret_cast<unsigned*>(c->ws.take(need * sizeof(unsigned)));
  if (!d_cb) return fail(c, LRE_ERR_OUT_OF_MEMORY, "workspace too small for cblack table");
  LRE_CUDA_TRY(c, cudaMemcpyAsync(d_cb, cblack, need * sizeof(unsigned), cudaMemcpyHostToDevice, c->stream));
  k_black_level<<<grid_for(w * h, 256, c->sm_count * 8), 256, 0, c->stream>>>(
      reinterpret_cast<ushort4*>(raw4), (int)w, (int)h, d_cb, mode, black, (int)maximum);
  count_launch(c);
  return check_launch(c, "black_level");
}

// Max over CFA samples (adjust_maximum, core/libraw_wrapper.cpp:1038-1051).
// raw_c_stride 3: sparse (H,W,3) layout reading channel fcol_bayer; 1: dense.
__global__ void k_cfa_max(const float* __restrict__ raw, int cstride, int w, int h, uint32_t filters,
                          float* out) {
  size_t n = (size_t)w * h;
  float m = 0.f;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    unsigned row = (unsigned)(i / w), col = (unsigned)(i % w);
    float v = cstride == 1 ? raw[i] : raw[i * 3 + fcol3(row, col, filters)];
    m = fmaxf(m, v);
  }
  m = warp_max(m);
  if ((threadIdx.x & 31) == 0) atomic_max_float(out, m);
}

lre_status launch_cfa_max(Context* c, const float* raw, int raw_c_stride, size_t w, size_t h,
                          uint32_t filters, float* d_out) {
  LRE_CUDA_TRY(c, cudaMemsetAsync(d_out, 0, sizeof(float), c->stream));
  k_cfa_max<<<grid_for(w * h, 256, c->sm_count * 4), 256, 0, c->stream>>>(raw, raw_c_stride, (int)w, (int)h,
                                                                          filters, d_out);
  count_launch(c);
  return check_launch(c, "cfa_max");
}

// max over one channel of an RGB image; clamp0 folds max(0, v) in (the
// reductions of defringe and axial CA start from 0 / 1e-6 on the host).
__global__ void k_channel_max(const float* __restrict__ rgb, size_t n, int ch, float* out) {
  float m = -INFINITY;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    m = fmaxf(m, rgb[i * 3 + ch]);
  m = warp_max(m);
  if ((threadIdx.x & 31) == 0) atomic_max_float(out, m);
}

__global__ void k_init_scalar(float* p, float v) { *p = v; }

lre_status launch_channel_max(Context* c, const float* rgb, size_t n_px, int channel, float* d_out, bool clamp0) {
  k_init_scalar<<<1, 1, 0, c->stream>>>(d_out, clamp0 ? 0.0f : -INFINITY);
  k_channel_max<<<grid_for(n_px, 256, c->sm_count * 4), 256, 0, c->stream>>>(rgb, n_px, channel, d_out);
  count_launch(c, 2);
  return check_launch(c, "channel_max");
}

// Output quantisation, core/python_bindings.cpp:241-256.
__global__ void k_quantize_u16(const float* __restrict__ in, uint16_t* __restrict__ out, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    float v = clampf(in[i], 0.f, 1.f);
    out[i] = (uint16_t)(v * 65535.0f + 0.5f);
  }
}
__global__ void k_quantize_u8(const float* __restrict__ in, uint8_t* __restrict__ out, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    float v = clampf(in[i], 0.f, 1.f);
    out[i] = (uint8_t)(v * 255.0f + 0.5f);
  }
}

lre_status launch_quantize_u16(Context* c, const float* in, uint16_t* out, size_t n) {
  k_quantize_u16<<<grid_for(n, 256, c->sm_count * 8), 256, 0, c->stream>>>(in, out, n);
  count_launch(c);
  return check_launch(c, "quantize_u16");
}
lre_status launch_quantize_u8(Context* c, const float* in, uint8_t* out, size_t n) {
  k_quantize_u8<<<grid_for(n, 256, c->sm_count * 8), 256, 0, c->stream>>>(in, out, n);
  count_launch(c);
  return check_launch(c, "quantize_u8");
}

// Sparse (H,W,3) raw buffer -> dense CFA mosaic (each site's own channel).
__global__ void k_pack_cfa(const float* __restrict__ raw, float* __restrict__ dense, int w, int h,
                           uint32_t filters, XTransPat xt) {
  size_t n = (size_t)w * h;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    unsigned row = (unsigned)(i / w), col = (unsigned)(i % w);
    unsigned c = filters == LRE_FILTERS_XTRANS ? (unsigned)xt.p[(row % 6) * 6 + col % 6] : fcol3(row, col, filters);
    dense[i] = raw[i * 3 + c];
  }
}

lre_status launch_pack_cfa(Context* c, const float* raw_rgb, float* dense, size_t w, size_t h, uint32_t filters,
                           const char* xtrans) {
  XTransPat xt{};
  if (xtrans) memcpy(xt.p, xtrans, 36);
  k_pack_cfa<<<grid_for(w * h, 256, c->sm_count * 8), 256, 0, c->stream>>>(raw_rgb, dense, (int)w, (int)h,
                                                                          filters, xt);
  count_launch(c);
  return check_launch(c, "pack_cfa");
}

}  // namespace lre
