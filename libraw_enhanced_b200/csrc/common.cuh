// common.cuh -- device helpers shared by the develop kernels.
//
// Arithmetic note: the library is compiled with --fmad=false so every
// expression rounds exactly like the reference's CPU code (built without FP
// contraction).  Helpers below keep the reference's operation order.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace lre {

// LibRaw filters word -> native colour 0..3 (core/metal/shader_common.h:63-65).
__host__ __device__ __forceinline__ unsigned fcol_native(unsigned row, unsigned col, uint32_t filters) {
  return filters >> ((((row << 1) & 14) | (col & 1)) << 1) & 3;
}
// G2 folded into G (core/metal/shader_common.h:67-69).
__host__ __device__ __forceinline__ unsigned fcol3(unsigned row, unsigned col, uint32_t filters) {
  unsigned c = fcol_native(row, col, filters);
  return c == 3 ? 1u : c;
}

// smoothstep exactly as core/cpu_accelerator.cpp:3321-3324.
__device__ __forceinline__ float sstep(float e0, float e1, float x) {
  float t = (x - e0) / (e1 - e0);
  t = fminf(fmaxf(t, 0.0f), 1.0f);
  return t * t * (3.0f - 2.0f * t);
}

__device__ __forceinline__ float clampf(float v, float lo, float hi) { return fminf(fmaxf(v, lo), hi); }

// ACES filmic curve, core/cpu_accelerator.cpp:3048-3056.
__device__ __forceinline__ float aces(float x) {
  const float a = 2.51f, b = 0.03f, c = 2.43f, d = 0.59f, e = 0.14f;
  return (x * (a * x + b)) / (x * (c * x + d) + e);
}

// Median of three with the reference's swap network (shader_common.h:52-58).
__device__ __forceinline__ float median3(float a, float b, float c) {
  if (a > b) { float t = a; a = b; b = t; }
  if (b > c) { float t = b; b = c; c = t; }
  if (a > b) { float t = a; a = b; b = t; }
  return b;
}

// Float max via integer atomics (valid for any initial value, NaN-free data).
__device__ __forceinline__ void atomic_max_float(float* addr, float v) {
  if (v >= 0.0f)
    atomicMax(reinterpret_cast<int*>(addr), __float_as_int(v));
  else
    atomicMin(reinterpret_cast<unsigned*>(addr), __float_as_uint(v));
}

// Warp / block reductions.
__device__ __forceinline__ float warp_max(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
// Max of a non-negative value over the CTA, folded into *addr with one
// atomic per CTA (every thread of the CTA must call it).
__device__ __forceinline__ void block_max_atomic(float v, float* addr) {
  __shared__ float s_wmax[32];
  v = warp_max(v);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) s_wmax[w] = v;
  __syncthreads();
  if (w == 0) {
    float x = lane < (int)((blockDim.x + 31) >> 5) ? s_wmax[lane] : 0.f;
    x = warp_max(x);
    if (lane == 0) atomic_max_float(addr, x);
  }
}
__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ unsigned long long warp_sum_u64(unsigned long long v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Correctly rounded float log / exp through double precision.  The reference
// calls glibc's logf/expf (errors below 1 ulp); evaluating in double and
// rounding once lands on the correctly rounded float, which is what glibc
// returns for all but a vanishing fraction of inputs, so per-pixel decisions
// downstream match the CPU far more often than with single-precision logf.
__device__ __forceinline__ float log_cr(float x) { return (float)log((double)x); }
__device__ __forceinline__ float exp_cr(float x) { return (float)exp((double)x); }
__device__ __forceinline__ float pow_cr(float x, float y) { return (float)pow((double)x, (double)y); }

}  // namespace lre
