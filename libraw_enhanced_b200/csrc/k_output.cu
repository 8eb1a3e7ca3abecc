// k_output.cu -- the output end of process_raw_to_rgb: camera -> output
// colour space (3x4 matrix), the output space's gamma encoding, and the
// 8/16-bit quantisation of ProcessedImageData.to_numpy, as separate stages
// and as one fused epilogue (12 B/px read, 3 or 6 B/px written).
//
// Semantics: core/cpu_accelerator.cpp:2874-2897 (convert_color_space),
// :2903-2978 (gamma_correct and its encoders), core/python_bindings.cpp:
// 235-257 (to_numpy).  std::pow(float, float) is evaluated in double and
// rounded once (pow_cr), so results can differ from glibc's powf by an ulp.
#include "common.cuh"
#include "lre_internal.h"
#include "stencil.cuh"

namespace lre {

namespace {

struct Mat34 {
  float m[12];
};

// ColorSpace values of core/metal/constants.h:28-38.
enum : int { CS_SRGB = 1, CS_ADOBE = 2, CS_WIDE = 3, CS_PROPHOTO = 4, CS_P3D65 = 7, CS_REC2020 = 8 };

__device__ __forceinline__ float pure_power(float v, float p) {
  if (v <= 0.0f) return 0.0f;
  return pow_cr(v, 1.0f / p);
}

__device__ __forceinline__ float gamma_encode(float v, float gamma_power, float gamma_slope, int cs) {
  switch (cs) {
    case CS_SRGB:
    case CS_P3D65:
      return (v <= 0.0031308f) ? 12.92f * v : 1.055f * pow_cr(v, 1.0f / 2.4f) - 0.055f;
    case CS_ADOBE:
    case CS_WIDE:
      return pure_power(v, 2.222f);
    case CS_PROPHOTO:
      return pure_power(v, 1.8f);
    case CS_REC2020: {
      const float a = 1.09929682680944f, b = 0.018053968510807f;
      return (v < b) ? 4.5f * v : a * pow_cr(v, 0.45f) - (a - 1.0f);
    }
    default:
      if (v <= 0.0f) return 0.0f;
      if (gamma_slope <= 0.f) return pow_cr(v, 1.0f / gamma_power);
      return (v < 1.0f / gamma_slope) ? v * gamma_slope : pow_cr(v, 1.0f / gamma_power);
  }
}

__device__ __forceinline__ void transform3(const Mat34& t, const float* in, float* out) {
  out[0] = t.m[0] * in[0] + t.m[1] * in[1] + t.m[2] * in[2] + t.m[3];
  out[1] = t.m[4] * in[0] + t.m[5] * in[1] + t.m[6] * in[2] + t.m[7];
  out[2] = t.m[8] * in[0] + t.m[9] * in[1] + t.m[10] * in[2] + t.m[11];
}

__global__ void k_color_space(const float* __restrict__ in, float* __restrict__ out, size_t n, Mat34 t) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    float v[3] = {in[i * 3], in[i * 3 + 1], in[i * 3 + 2]}, o[3];
    transform3(t, v, o);
    out[i * 3] = o[0];
    out[i * 3 + 1] = o[1];
    out[i * 3 + 2] = o[2];
  }
}

__global__ void k_gamma(const float* __restrict__ in, float* __restrict__ out, size_t n, float gp, float gs, int cs) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    out[i] = gamma_encode(in[i], gp, gs, cs);
}

// Fused: transform, gamma, then to_numpy's quantisation (bits 8 or 16) or
// float output (bits 32).
template <int BITS>
__global__ void k_epilogue(const float* __restrict__ in, void* __restrict__ out, size_t n, Mat34 t, float gp, float gs,
                           int cs) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    float v[3] = {in[i * 3], in[i * 3 + 1], in[i * 3 + 2]}, o[3];
    transform3(t, v, o);
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const float g = gamma_encode(o[c], gp, gs, cs);
      if (BITS == 8) {
        static_cast<uint8_t*>(out)[i * 3 + c] = (uint8_t)(sclamp(g, 0.f, 1.f) * 255.0f + 0.5f);
      } else if (BITS == 16) {
        static_cast<uint16_t*>(out)[i * 3 + c] = (uint16_t)(sclamp(g, 0.f, 1.f) * 65535.0f + 0.5f);
      } else {
        static_cast<float*>(out)[i * 3 + c] = g;
      }
    }
  }
}

Mat34 mat(const float* t) {
  Mat34 m;
  for (int i = 0; i < 12; i++) m.m[i] = t[i];
  return m;
}

}  // namespace

lre_status launch_color_space(Context* c, const float* in, float* out, size_t n_px, const float transform[12]) {
  k_color_space<<<grid_for(n_px, 256, c->sm_count * 8), 256, 0, c->stream>>>(in, out, n_px, mat(transform));
  count_launch(c);
  return check_launch(c, "convert_color_space");
}

lre_status launch_gamma(Context* c, const float* in, float* out, size_t n_px, float gamma_power, float gamma_slope,
                        int color_space) {
  k_gamma<<<grid_for(n_px * 3, 256, c->sm_count * 8), 256, 0, c->stream>>>(in, out, n_px * 3, gamma_power,
                                                                            gamma_slope, color_space);
  count_launch(c);
  return check_launch(c, "gamma_correct");
}

lre_status launch_output_epilogue(Context* c, const float* in, void* out, size_t n_px, const float transform[12],
                                  float gamma_power, float gamma_slope, int color_space, int bits) {
  const unsigned g = grid_for(n_px, 256, c->sm_count * 8);
  if (bits == 8)
    k_epilogue<8><<<g, 256, 0, c->stream>>>(in, out, n_px, mat(transform), gamma_power, gamma_slope, color_space);
  else if (bits == 16)
    k_epilogue<16><<<g, 256, 0, c->stream>>>(in, out, n_px, mat(transform), gamma_power, gamma_slope, color_space);
  else
    k_epilogue<32><<<g, 256, 0, c->stream>>>(in, out, n_px, mat(transform), gamma_power, gamma_slope, color_space);
  count_launch(c);
  return check_launch(c, "output epilogue");
}

}  // namespace lre

using lre::Context;

extern "C" {

lre_status lre_output_epilogue(lre_ctx* ctx, const float* in, void* out, size_t width, size_t height,
                               const float transform[12], float gamma_power, float gamma_slope,
                               int output_color_space, int bits) {
  Context* c = reinterpret_cast<Context*>(ctx);
  if (!c) return LRE_ERR_INVALID_ARGUMENT;
  if (!in || !out || !transform || width == 0 || height == 0 || (bits != 8 && bits != 16 && bits != 32))
    return lre::fail(c, LRE_ERR_INVALID_ARGUMENT, "output_epilogue: bad arguments (bits must be 8, 16 or 32)");
  std::lock_guard<std::mutex> lk(c->mu);
  cudaSetDevice(c->device);
  LRE_TRY(lre::check_injection(c));
  const size_t n = width * height, in_bytes = n * 12, out_bytes = n * 3 * (size_t)(bits / 8);
  LRE_TRY(lre::ensure_buffer(c, &c->d_in, &c->d_in_cap, in_bytes));
  LRE_TRY(lre::ensure_buffer(c, &c->d_out, &c->d_out_cap, out_bytes));
  LRE_TRY(lre::copy_h2d(c, c->d_in, in, in_bytes, c->stream));
  LRE_TRY(lre::launch_output_epilogue(c, reinterpret_cast<const float*>(c->d_in), c->d_out, n, transform, gamma_power,
                                      gamma_slope, output_color_space, bits));
  LRE_TRY(lre::copy_d2h(c, out, c->d_out, out_bytes, c->stream));
  LRE_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  return LRE_OK;
}

lre_status lre_dev_output_epilogue(lre_ctx* ctx, const float* in, void* out, size_t width, size_t height,
                                   const float transform[12], float gamma_power, float gamma_slope,
                                   int output_color_space, int bits) {
  Context* c = reinterpret_cast<Context*>(ctx);
  if (!c) return LRE_ERR_INVALID_ARGUMENT;
  if (!in || !out || !transform || width == 0 || height == 0 || (bits != 8 && bits != 16 && bits != 32))
    return lre::fail(c, LRE_ERR_INVALID_ARGUMENT, "output_epilogue: bad arguments (bits must be 8, 16 or 32)");
  cudaSetDevice(c->device);
  LRE_TRY(lre::check_injection(c));
  return lre::launch_output_epilogue(c, in, out, width * height, transform, gamma_power, gamma_slope,
                                     output_color_space, bits);
}

}  // extern "C"
