// stencil.cuh -- exact-semantics helpers shared by the stencil kernels:
// std::min/std::max/std::clamp with the C++ library's argument-order rules
// (they matter for NaN and signed zeros), and a shared-memory separable
// Gaussian blur that reproduces the reference's clamp-to-edge, tap-order
// float accumulation bit for bit.
#pragma once

#include "common.cuh"

namespace lre {

// std::max(a, b) returns (a < b) ? b : a; std::min(a, b) returns (b < a) ? b : a.
__device__ __forceinline__ float smax(float a, float b) { return (a < b) ? b : a; }
__device__ __forceinline__ float smin(float a, float b) { return (b < a) ? b : a; }
// std::clamp(v, lo, hi)
__device__ __forceinline__ float sclamp(float v, float lo, float hi) { return (v < lo) ? lo : ((hi < v) ? hi : v); }
// smoothstep of core/cpu_accelerator.cpp:3321-3324 with std::clamp.
__device__ __forceinline__ float ssmooth(float e0, float e1, float x) {
  float t = sclamp((x - e0) / (e1 - e0), 0.0f, 1.0f);
  return t * t * (3.0f - 2.0f * t);
}

constexpr int GAUSS_MAX_KS = 32;
struct GaussTaps {
  int ks;
  float w[2 * GAUSS_MAX_KS + 1];
};

// Host: the reference's defringe kernel (core/cpu_accelerator.cpp:4033-4046),
// computed with the host libm so the taps are the reference's taps.
GaussTaps make_defringe_taps(float radius);

}  // namespace lre
