/*
 * simd_shim.h -- test infrastructure for the oracle build only.
 *
 * The reference CPU accelerator (core/cpu_accelerator.cpp:3107-3319,
 * enhance_micro_contrast) uses Apple's <simd/simd.h> `vector_float3` type.
 * Linux has no such header, so this force-included shim supplies a type with
 * the same element-wise float semantics (4 lanes, the 4th unused, exactly as
 * Apple's 16-byte float3).  Every operator is a plain per-lane IEEE float
 * operation, so results are identical to the per-channel scalar arithmetic.
 */
#pragma once
struct vector_float3 {
  float v[4];
  float& operator[](int i) { return v[i]; }
  const float& operator[](int i) const { return v[i]; }
};
static inline vector_float3 simd_make_float3(float x) { return vector_float3{{x, x, x, 0.f}}; }
static inline vector_float3 simd_make_float3(float x, float y, float z) { return vector_float3{{x, y, z, 0.f}}; }
#define LRE_VF3_BINOP(OP)                                                                  \
  static inline vector_float3 operator OP(const vector_float3& a, const vector_float3& b) { \
    return vector_float3{{a.v[0] OP b.v[0], a.v[1] OP b.v[1], a.v[2] OP b.v[2], 0.f}};     \
  }                                                                                        \
  static inline vector_float3 operator OP(const vector_float3& a, float b) {               \
    return vector_float3{{a.v[0] OP b, a.v[1] OP b, a.v[2] OP b, 0.f}};                    \
  }                                                                                        \
  static inline vector_float3 operator OP(float a, const vector_float3& b) {               \
    return vector_float3{{a OP b.v[0], a OP b.v[1], a OP b.v[2], 0.f}};                    \
  }
LRE_VF3_BINOP(+)
LRE_VF3_BINOP(-)
LRE_VF3_BINOP(*)
LRE_VF3_BINOP(/)
#undef LRE_VF3_BINOP
static inline vector_float3& operator+=(vector_float3& a, const vector_float3& b) {
  a.v[0] += b.v[0];
  a.v[1] += b.v[1];
  a.v[2] += b.v[2];
  return a;
}
