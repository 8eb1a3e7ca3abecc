/*
 * ref_capi.cpp -- TEST INFRASTRUCTURE (oracle), never part of the product.
 *
 * A flat C ABI over the reference's own CPU accelerator
 * (core/cpu_accelerator.{h,cpp} of uniuyuni/libraw_enhanced), compiled from the
 * reference sources where they lie by oracle/Makefile.  Only tests/, the smoke
 * check and bench.py's CPU-baseline leg load the resulting
 * oracle/_ref/liblre_ref.so; it is the checker the CUDA path is compared
 * against, not something the product calls.
 *
 * Buffers are the reference's layouts: interleaved float (H,W,3) images
 * (ImageBufferFloat, core/accelerator.h:70-80) and uint16[4] per pixel raw
 * images (ImageBuffer, core/accelerator.h:59-68).  Each entry point returns 1
 * on success and 0 on failure, exactly like the bool the reference returns.
 *
 * The reference logs heavily to std::cout; the wrapper mutes std::cout for the
 * duration of a call (unless LRE_REF_VERBOSE is set) so test output stays
 * readable.  Muting changes no arithmetic.
 */
#include "cpu_accelerator.h"

#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <iostream>

#ifdef _OPENMP
#include <omp.h>
#endif

using libraw_enhanced::CPUAccelerator;
using libraw_enhanced::ImageBuffer;
using libraw_enhanced::ImageBufferFloat;

namespace {

struct MuteCout {
  std::streambuf* saved = nullptr;
  MuteCout() {
    if (!std::getenv("LRE_REF_VERBOSE")) saved = std::cout.rdbuf(nullptr);
  }
  ~MuteCout() {
    if (saved) {
      std::cout.rdbuf(saved);
      std::cout.clear();
    }
  }
};

CPUAccelerator& accel() {
  static CPUAccelerator* a = [] {
    MuteCout m;
    auto* p = new CPUAccelerator();
    p->initialize();
    return p;
  }();
  return *a;
}

ImageBufferFloat fbuf(const float* p, size_t w, size_t h) {
  ImageBufferFloat b;
  b.image = reinterpret_cast<float(*)[3]>(const_cast<float*>(p));
  b.width = w;
  b.height = h;
  b.channels = 3;
  return b;
}

}  // namespace

extern "C" {

int ref_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

void ref_set_num_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

/* core/cpu_accelerator.cpp:1635-1653 (AMaZE + border_interpolate(4)) */
int ref_demosaic_bayer_amaze(const float* raw, float* rgb, size_t w, size_t h, uint32_t filters,
                             const float cam_mul[4], float maximum_value) {
  MuteCout m;
  ImageBufferFloat in = fbuf(raw, w, h), out = fbuf(rgb, w, h);
  const float cm[4] = {cam_mul[0], cam_mul[1], cam_mul[2], cam_mul[3]};
  return accel().demosaic_bayer_amaze(in, out, filters, cm, maximum_value) ? 1 : 0;
}

/* core/cpu_accelerator.cpp:74-156 (bilinear Bayer demosaic + border(1)) */
int ref_demosaic_bayer_linear(const float* raw, float* rgb, size_t w, size_t h, uint32_t filters,
                              float maximum_value) {
  MuteCout m;
  ImageBufferFloat in = fbuf(raw, w, h), out = fbuf(rgb, w, h);
  return accel().demosaic_bayer_linear(in, out, filters, maximum_value) ? 1 : 0;
}

/* core/cpu_accelerator.cpp:617-633 (AAHD demosaic: AAHD_Processor at
 * :177-601, border_interpolate(2)).  Its hide_hots and refine_hv_dirs are
 * OpenMP row loops that rewrite in place, and its channel min/max scan is an
 * unsynchronised OpenMP loop, so tests call this with one thread. */
int ref_demosaic_bayer_aahd(const float* raw, float* rgb, size_t w, size_t h, uint32_t filters,
                            float maximum_value) {
  MuteCout m;
  ImageBufferFloat in = fbuf(raw, w, h), out = fbuf(rgb, w, h);
  return accel().demosaic_bayer_aahd(in, out, filters, maximum_value) ? 1 : 0;
}

/* core/cpu_accelerator.cpp:1043-1137 (DCB demosaic: sparse + 8-neighbour
 * bilinear seed, DCB_Processor::run_dcb at :998-1035, /maximum,
 * border_interpolate(3)).  Several of DCB's in-place passes are OpenMP
 * row-parallel loops whose rows read rows the same loop rewrites (nyquist,
 * pp, the last color_full loop); their defined result is the sequential one,
 * so tests call this with ref_set_num_threads(1). */
int ref_demosaic_bayer_dcb(const float* raw, float* rgb, size_t w, size_t h, uint32_t filters,
                           float maximum_value, int iterations, int dcb_enhance) {
  MuteCout m;
  ImageBufferFloat in = fbuf(raw, w, h), out = fbuf(rgb, w, h);
  return accel().demosaic_bayer_dcb(in, out, filters, maximum_value, iterations, dcb_enhance != 0) ? 1 : 0;
}

/* core/cpu_accelerator.cpp:2767-2784 (X-Trans 1-pass / 3-pass) */
int ref_demosaic_xtrans(const float* raw, float* rgb, size_t w, size_t h, const char xtrans[36],
                        const float color_matrix[12], float maximum_value, int passes) {
  MuteCout m;
  ImageBufferFloat in = fbuf(raw, w, h), out = fbuf(rgb, w, h);
  char xt[6][6];
  float cmat[3][4];
  std::memcpy(xt, xtrans, 36);
  std::memcpy(cmat, color_matrix, sizeof(cmat));
  bool ok = passes == 1 ? accel().demosaic_xtrans_1pass(in, out, xt, cmat, maximum_value)
                        : accel().demosaic_xtrans_3pass(in, out, xt, cmat, maximum_value);
  return ok ? 1 : 0;
}

/* core/cpu_accelerator.cpp:2789-2869 (white balance, Bayer and X-Trans) */
int ref_apply_white_balance(const uint16_t* raw4, float* rgb, size_t w, size_t h, const float wb[4],
                            uint32_t filters, const char xtrans[36]) {
  MuteCout m;
  ImageBuffer in;
  in.image = reinterpret_cast<uint16_t(*)[4]>(const_cast<uint16_t*>(raw4));
  in.width = w;
  in.height = h;
  in.channels = 4;
  ImageBufferFloat out = fbuf(rgb, w, h);
  char xt[6][6];
  std::memcpy(xt, xtrans, 36);
  return accel().apply_white_balance(in, out, wb, filters, xt) ? 1 : 0;
}

/* core/cpu_accelerator.cpp:3034-3068 (ACES tone map) */
int ref_tone_mapping(const float* in, float* out, size_t w, size_t h, float after_scale) {
  MuteCout m;
  ImageBufferFloat a = fbuf(in, w, h), b = fbuf(out, w, h);
  return accel().tone_mapping(a, b, after_scale) ? 1 : 0;
}

/* core/cpu_accelerator.cpp:2874-2897 (convert_color_space, 3x4 matrix) */
int ref_convert_color_space(const float* in, float* out, size_t w, size_t h, const float transform[12]) {
  MuteCout m;
  ImageBufferFloat a = fbuf(in, w, h), b = fbuf(out, w, h);
  float t[3][4];
  for (int i = 0; i < 12; i++) t[i / 4][i % 4] = transform[i];
  return accel().convert_color_space(a, b, t) ? 1 : 0;
}

/* core/cpu_accelerator.cpp:2903-2978 (gamma_correct) */
int ref_gamma_correct(const float* in, float* out, size_t w, size_t h, float gamma_power, float gamma_slope,
                      int output_color_space) {
  MuteCout m;
  ImageBufferFloat a = fbuf(in, w, h), b = fbuf(out, w, h);
  return accel().gamma_correct(a, b, gamma_power, gamma_slope, output_color_space) ? 1 : 0;
}

/* core/cpu_accelerator.cpp:3130-3319 (micro-contrast) */
int ref_enhance_micro_contrast(const float* in, float* out, size_t w, size_t h, float threshold,
                               float strength, float target_contrast, const float* mask) {
  MuteCout m;
  ImageBufferFloat a = fbuf(in, w, h), b = fbuf(out, w, h);
  return accel().enhance_micro_contrast(a, b, threshold, strength, target_contrast, mask) ? 1 : 0;
}

/* core/cpu_accelerator.cpp:3939-5064 (defringe) */
int ref_defringe(const float* in, float* out, size_t w, size_t h, float radius, float edge_threshold,
                 float chroma_threshold, float strength, int green, float green_scale) {
  MuteCout m;
  ImageBufferFloat a = fbuf(in, w, h), b = fbuf(out, w, h);
  return accel().defringe(a, b, radius, edge_threshold, chroma_threshold, strength, green != 0,
                          green_scale)
             ? 1
             : 0;
}

/* core/cpu_accelerator.cpp:3496-3673 (lateral CA, pyramidal LK) */
int ref_ca_register_lateral(const float* in, float* out, size_t w, size_t h, int cell, int iters,
                            float max_shift, float min_conf, int levels) {
  MuteCout m;
  ImageBufferFloat a = fbuf(in, w, h), b = fbuf(out, w, h);
  return accel().ca_register_lateral(a, b, cell, iters, max_shift, min_conf, levels) ? 1 : 0;
}

/* core/cpu_accelerator.cpp:3799-3928 (axial CA guided filter) */
int ref_ca_axial_cleanup(const float* in, float* out, size_t w, size_t h, int radius, float eps,
                         float strength) {
  MuteCout m;
  ImageBufferFloat a = fbuf(in, w, h), b = fbuf(out, w, h);
  return accel().ca_axial_cleanup(a, b, radius, eps, strength) ? 1 : 0;
}

/* core/cpu_accelerator.cpp:46-68 (pre_interpolate) */
int ref_pre_interpolate(float* rgb, size_t w, size_t h, uint32_t filters, const char xtrans[36],
                        int half_size) {
  MuteCout m;
  ImageBufferFloat a = fbuf(rgb, w, h);
  char xt[6][6];
  std::memcpy(xt, xtrans, 36);
  return accel().pre_interpolate(a, filters, xt, half_size != 0) ? 1 : 0;
}

}  // extern "C"
