// cuda_accelerator.h -- C++ drop-in for libraw_enhanced's GPUAccelerator.
//
// Same method set and argument meaning as GPUAccelerator
// (core/gpu_accelerator.h:18-118 in uniuyuni/libraw_enhanced), implemented on
// the C ABI of liblre_cuda.so (include/lre_cuda.h).  Buffers are the
// reference's ImageBuffer / ImageBufferFloat (core/accelerator.h:59-80).
// Inside libraw_enhanced, define LRE_USE_REFERENCE_TYPES and include this
// after "accelerator.h" to use the reference's own structs; otherwise
// layout-identical structs are declared here.
//
// Methods return false on failure and keep the message in last_error(),
// matching the reference's bool contract.
#pragma once

#include <cstdint>
#include <string>

#include "../../include/lre_cuda.h"

#ifdef LRE_USE_REFERENCE_TYPES
namespace lre_types = libraw_enhanced;
#else
namespace lre_types {
struct ImageBuffer {
  uint16_t (*image)[4] = nullptr;
  size_t width = 0;
  size_t height = 0;
  size_t channels = 0;
  bool is_valid() const { return image != nullptr && width > 0 && height > 0 && channels > 0; }
};
struct ImageBufferFloat {
  float (*image)[3] = nullptr;
  size_t width = 0;
  size_t height = 0;
  size_t channels = 3;
  bool is_valid() const { return image != nullptr && width > 0 && height > 0 && channels > 0; }
};
}  // namespace lre_types
#endif

namespace lre {

class CudaAccelerator {
 public:
  using ImageBuffer = lre_types::ImageBuffer;
  using ImageBufferFloat = lre_types::ImageBufferFloat;

  CudaAccelerator() = default;
  ~CudaAccelerator() {
    if (ctx_) lre_destroy(ctx_);
  }
  CudaAccelerator(const CudaAccelerator&) = delete;
  CudaAccelerator& operator=(const CudaAccelerator&) = delete;

  // GPUAccelerator::initialize / is_available / get_device_info
  bool initialize(int device = 0) {
    if (ctx_) return true;
    lre_status st = lre_create(device, &ctx_);
    if (st != LRE_OK) {
      ctx_ = nullptr;
      err_ = "lre_create failed (no usable sm_100 device)";
      return false;
    }
    return true;
  }
  bool is_available() const { return ctx_ != nullptr; }
  std::string get_device_info() const {
    char buf[256] = {0};
    if (!ctx_ || lre_device_info(ctx_, buf, sizeof(buf)) != LRE_OK) return "CUDA (unavailable)";
    return buf;
  }
  const std::string& last_error() const { return err_; }
  lre_ctx* context() const { return ctx_; }

  bool demosaic_bayer_linear(const ImageBufferFloat& raw, ImageBufferFloat& rgb, uint32_t filters,
                             float maximum_value) {
    if (!same(raw, rgb)) return bad("demosaic_bayer_linear: buffer size mismatch");
    return ok(lre_demosaic_bayer_linear(ctx_, f(raw), f(rgb), raw.width, raw.height, filters, maximum_value));
  }
  // Accelerator::demosaic_bayer_dcb / demosaic_bayer_aahd (core/accelerator.h:269-277); the
  // reference's GPU path has neither and falls back to the CPU (core/accelerator.cpp:159-199).
  bool demosaic_bayer_dcb(const ImageBufferFloat& raw, ImageBufferFloat& rgb, uint32_t filters,
                          float maximum_value, int iterations = 1, bool dcb_enhance = true) {
    if (!same(raw, rgb)) return bad("demosaic_bayer_dcb: buffer size mismatch");
    return ok(lre_demosaic_bayer_dcb(ctx_, f(raw), f(rgb), raw.width, raw.height, filters, maximum_value,
                                     iterations, dcb_enhance ? 1 : 0));
  }
  bool demosaic_bayer_aahd(const ImageBufferFloat& raw, ImageBufferFloat& rgb, uint32_t filters,
                           float maximum_value) {
    if (!same(raw, rgb)) return bad("demosaic_bayer_aahd: buffer size mismatch");
    return ok(lre_demosaic_bayer_aahd(ctx_, f(raw), f(rgb), raw.width, raw.height, filters, maximum_value));
  }
  bool demosaic_bayer_amaze(const ImageBufferFloat& raw, ImageBufferFloat& rgb, uint32_t filters,
                            const float (&cam_mul)[4], float maximum_value) {
    if (!same(raw, rgb)) return bad("demosaic_bayer_amaze: mismatched buffers");
    return ok(lre_demosaic_bayer_amaze(ctx_, f(raw), f(rgb), raw.width, raw.height, filters, cam_mul, maximum_value));
  }
  bool demosaic_xtrans_1pass(const ImageBufferFloat& raw, ImageBufferFloat& rgb, const char (&xtrans)[6][6],
                             const float (&color_matrix)[3][4], float maximum_value) {
    if (!same(raw, rgb)) return bad("demosaic_xtrans_1pass: mismatched buffers");
    return ok(lre_demosaic_xtrans_1pass(ctx_, f(raw), f(rgb), raw.width, raw.height, &xtrans[0][0],
                                        &color_matrix[0][0], maximum_value));
  }
  bool demosaic_xtrans_3pass(const ImageBufferFloat& raw, ImageBufferFloat& rgb, const char (&xtrans)[6][6],
                             const float (&color_matrix)[3][4], float maximum_value) {
    if (!same(raw, rgb)) return bad("demosaic_xtrans_3pass: mismatched buffers");
    return ok(lre_demosaic_xtrans_3pass(ctx_, f(raw), f(rgb), raw.width, raw.height, &xtrans[0][0],
                                        &color_matrix[0][0], maximum_value));
  }
  bool apply_white_balance(const ImageBuffer& raw, ImageBufferFloat& rgb, const float wb[4], uint32_t filters,
                           const char xtrans[6][6]) {
    if (!raw.is_valid() || !rgb.is_valid() || raw.width != rgb.width || raw.height != rgb.height)
      return bad("apply_white_balance: invalid buffers");
    return ok(lre_apply_white_balance(ctx_, &raw.image[0][0], &rgb.image[0][0], raw.width, raw.height, wb, filters,
                                      xtrans ? &xtrans[0][0] : nullptr));
  }
  bool convert_color_space(const ImageBufferFloat& in, ImageBufferFloat& out, const float transform[3][4]) {
    if (!same(in, out)) return bad("convert_color_space: buffer size mismatch");
    return ok(lre_convert_color_space(ctx_, f(in), f(out), in.width, in.height, &transform[0][0]));
  }
  // defaults as GPUAccelerator::gamma_correct (core/gpu_accelerator.h:70-74)
  bool gamma_correct(const ImageBufferFloat& in, ImageBufferFloat& out, float gamma_power = 0.f,
                     float gamma_slope = 0.f, int output_color_space = 1) {
    if (!same(in, out)) return bad("gamma_correct: buffer size mismatch");
    return ok(lre_gamma_correct(ctx_, f(in), f(out), in.width, in.height, gamma_power, gamma_slope, output_color_space));
  }
  bool tone_mapping(const ImageBufferFloat& in, ImageBufferFloat& out, float after_scale) {
    if (!same(in, out)) return bad("tone_mapping: mismatched buffers");
    return ok(lre_tone_mapping(ctx_, f(in), f(out), in.width, in.height, after_scale));
  }
  bool enhance_micro_contrast(const ImageBufferFloat& in, ImageBufferFloat& out, float threshold, float strength,
                              float target_contrast, const float* mask = nullptr) {
    if (!same(in, out)) return bad("enhance_micro_contrast: mismatched buffers");
    return ok(lre_enhance_micro_contrast(ctx_, f(in), f(out), in.width, in.height, threshold, strength,
                                         target_contrast, mask));
  }
  bool apply_detail_preserving_tonemap(const ImageBufferFloat& in, ImageBufferFloat& out) {
    if (!same(in, out)) return bad("apply_detail_preserving_tonemap: mismatched buffers");
    return ok(lre_detail_tonemap(ctx_, f(in), f(out), in.width, in.height));
  }
  bool ca_register_lateral(const ImageBufferFloat& in, ImageBufferFloat& out, int cell_size, int max_iterations,
                           float max_shift, float min_confidence, int pyramid_levels) {
    if (!same(in, out)) return bad("ca_register_lateral: mismatched buffers");
    return ok(lre_ca_register_lateral(ctx_, f(in), f(out), in.width, in.height, cell_size, max_iterations, max_shift,
                                      min_confidence, pyramid_levels));
  }
  bool ca_axial_cleanup(const ImageBufferFloat& in, ImageBufferFloat& out, int radius, float epsilon, float strength) {
    if (!same(in, out)) return bad("ca_axial_cleanup: mismatched buffers");
    return ok(lre_ca_axial_cleanup(ctx_, f(in), f(out), in.width, in.height, radius, epsilon, strength));
  }
  bool defringe(const ImageBufferFloat& in, ImageBufferFloat& out, float radius, float edge_threshold,
                float chroma_threshold, float strength, bool defringe_green, float green_strength_scale) {
    if (!same(in, out)) return bad("defringe: mismatched buffers");
    return ok(lre_defringe(ctx_, f(in), f(out), in.width, in.height, radius, edge_threshold, chroma_threshold, strength,
                           defringe_green ? 1 : 0, green_strength_scale));
  }

 private:
  lre_ctx* ctx_ = nullptr;
  std::string err_;

  static float* f(const ImageBufferFloat& b) { return &b.image[0][0]; }
  bool same(const ImageBufferFloat& a, const ImageBufferFloat& b) {
    if (!ctx_ && !initialize()) return false;
    return a.is_valid() && b.is_valid() && a.width == b.width && a.height == b.height && a.channels == 3 &&
           b.channels == 3;
  }
  bool bad(const char* msg) {
    if (err_.empty() || ctx_) err_ = msg;
    return false;
  }
  bool ok(lre_status st) {
    if (st == LRE_OK) return true;
    err_ = ctx_ ? lre_last_error(ctx_) : "no context";
    return false;
  }
};

}  // namespace lre
