// capi.cu -- extern "C" entry points: argument checks, staging of host
// buffers, workspace planning, and the plain per-image develop pipeline.
#include <cstring>
#include <mutex>
#include <string>

#include "lre_internal.h"

using lre::Context;

namespace {

Context* C(lre_ctx* p) { return reinterpret_cast<Context*>(p); }

lre_status check_img(Context* c, const void* a, const void* b, size_t w, size_t h, const char* what) {
  if (!a || !b) return lre::fail(c, LRE_ERR_INVALID_ARGUMENT, std::string(what) + ": null buffer");
  if (w == 0 || h == 0) return lre::fail(c, LRE_ERR_INVALID_ARGUMENT, std::string(what) + ": empty image");
  if (w > (1u << 20) || h > (1u << 20) || w * h > (size_t(1) << 31))
    return lre::fail(c, LRE_ERR_INVALID_ARGUMENT, std::string(what) + ": image too large");
  return LRE_OK;
}

// Prepare the context for a call: device, fault injection, workspace.
lre_status begin(Context* c, size_t ws_bytes) {
  cudaSetDevice(c->device);
  LRE_TRY(lre::check_injection(c));
  c->ws.reset();
  if (ws_bytes) LRE_CUDA_TRY(c, c->ws.reserve(ws_bytes, c->stream));
  return LRE_OK;
}

// Host-buffer helper: RGB(in) -> device, run `fn(d_in, d_out)`, device -> RGB(out).
template <typename Fn>
lre_status host_rgb_stage(Context* c, const float* in, float* out, size_t w, size_t h, size_t ws, Fn fn) {
  std::lock_guard<std::mutex> lk(c->mu);
  LRE_TRY(begin(c, ws));
  const size_t bytes = w * h * 3 * sizeof(float);
  LRE_TRY(lre::ensure_buffer(c, &c->d_in, &c->d_in_cap, bytes));
  float* d = reinterpret_cast<float*>(c->d_in);
  LRE_TRY(lre::copy_h2d(c, d, in, bytes, c->stream));
  LRE_TRY(fn(d));
  LRE_TRY(lre::copy_d2h(c, out, d, bytes, c->stream));
  LRE_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  return LRE_OK;
}

}  // namespace

extern "C" {

// ------------------------------------------------------------ tone mapping
lre_status lre_dev_tone_mapping(lre_ctx* ctx, const float* in, float* out, size_t w, size_t h, float s) {
  Context* c = C(ctx);
  if (!c) return LRE_ERR_INVALID_ARGUMENT;
  LRE_TRY(check_img(c, in, out, w, h, "tone_mapping"));
  LRE_TRY(begin(c, 0));
  return lre::launch_tone_mapping(c, in, out, w * h, s);
}

lre_status lre_tone_mapping(lre_ctx* ctx, const float* in, float* out, size_t w, size_t h, float s) {
  Context* c = C(ctx);
  if (!c) return LRE_ERR_INVALID_ARGUMENT;
  LRE_TRY(check_img(c, in, out, w, h, "tone_mapping"));
  return host_rgb_stage(c, in, out, w, h, 0, [&](float* d) { return lre::launch_tone_mapping(c, d, d, w * h, s); });
}

// ------------------------------------------------------------ axial CA
static lre_status axial_dev(Context* c, const float* in, float* out, size_t w, size_t h, int r, float eps, float s) {
  float* dmax = c->d_scalars;
  LRE_TRY(lre::launch_channel_max(c, in, w * h, 1, dmax, /*clamp0=*/true));
  return lre::launch_axial_ca(c, in, out, w, h, r, eps, s, dmax);
}

lre_status lre_dev_ca_axial_cleanup(lre_ctx* ctx, const float* in, float* out, size_t w, size_t h, int r,
                                    float eps, float s) {
  Context* c = C(ctx);
  if (!c) return LRE_ERR_INVALID_ARGUMENT;
  LRE_TRY(check_img(c, in, out, w, h, "ca_axial_cleanup"));
  LRE_TRY(begin(c, lre::ws_bytes_axial(w, h, r)));
  return axial_dev(c, in, out, w, h, r, eps, s);
}

lre_status lre_ca_axial_cleanup(lre_ctx* ctx, const float* in, float* out, size_t w, size_t h, int r, float eps,
                                float s) {
  Context* c = C(ctx);
  if (!c) return LRE_ERR_INVALID_ARGUMENT;
  LRE_TRY(check_img(c, in, out, w, h, "ca_axial_cleanup"));
  return host_rgb_stage(c, in, out, w, h, lre::ws_bytes_axial(w, h, r),
                        [&](float* d) { return axial_dev(c, d, d, w, h, r, eps, s); });
}

// ------------------------------------------------------------ defringe
lre_status lre_dev_defringe(lre_ctx* ctx, const float* in, float* out, size_t w, size_t h, float radius, float edge,
                            float chroma, float strength, int green, float green_scale) {
  Context* c = C(ctx);
  if (!c) return LRE_ERR_INVALID_ARGUMENT;
  LRE_TRY(check_img(c, in, out, w, h, "defringe"));
  LRE_TRY(begin(c, lre::ws_bytes_defringe(w, h, radius)));
  return lre::launch_defringe(c, in, out, w, h, radius, edge, chroma, strength, green != 0, green_scale, nullptr);
}

lre_status lre_defringe(lre_ctx* ctx, const float* in, float* out, size_t w, size_t h, float radius, float edge,
                        float chroma, float strength, int green, float green_scale) {
  Context* c = C(ctx);
  if (!c) return LRE_ERR_INVALID_ARGUMENT;
  LRE_TRY(check_img(c, in, out, w, h, "defringe"));
  return host_rgb_stage(c, in, out, w, h, lre::ws_bytes_defringe(w, h, radius), [&](float* d) {
    return lre::launch_defringe(c, d, d, w, h, radius, edge, chroma, strength, green != 0, green_scale, nullptr);
  });
}

// ------------------------------------------------------------ detail tonemap
lre_status lre_dev_detail_tonemap(lre_ctx* ctx, const float* in, float* out, size_t w, size_t h) {
  Context* c = C(ctx);
  if (!c) return LRE_ERR_INVALID_ARGUMENT;
  LRE_TRY(check_img(c, in, out, w, h, "detail_tonemap"));
  LRE_TRY(begin(c, lre::ws_bytes_detail_tonemap(w, h)));
  return lre::launch_detail_tonemap(c, in, out, w, h);
}

lre_status lre_detail_tonemap(lre_ctx* ctx, const float* in, float* out, size_t w, size_t h) {
  Context* c = C(ctx);
  if (!c) return LRE_ERR_INVALID_ARGUMENT;
  LRE_TRY(check_img(c, in, out, w, h, "detail_tonemap"));
  return host_rgb_stage(c, in, out, w, h, lre::ws_bytes_detail_tonemap(w, h),
                        [&](float* d) { return lre::launch_detail_tonemap(c, d, d, w, h); });
}

// ------------------------------------------------------------ micro-contrast
lre_status lre_dev_enhance_micro_contrast(lre_ctx* ctx, const float* in, float* out, size_t w, size_t h, float thr,
                                          float strength, float target, const float* mask) {
  Context* c = C(ctx);
  if (!c) return LRE_ERR_INVALID_ARGUMENT;
  LRE_TRY(check_img(c, in, out, w, h, "enhance_micro_contrast"));
  LRE_TRY(begin(c, lre::ws_bytes_micro_contrast(w, h)));
  return lre::launch_micro_contrast(c, in, out, w, h, thr, strength, target, mask);
}

lre_status lre_enhance_micro_contrast(lre_ctx* ctx, const float* in, float* out, size_t w, size_t h, float thr,
                                      float strength, float target, const float* mask) {
  Context* c = C(ctx);
  if (!c) return LRE_ERR_INVALID_ARGUMENT;
  LRE_TRY(check_img(c, in, out, w, h, "enhance_micro_contrast"));
  std::lock_guard<std::mutex> lk(c->mu);
  LRE_TRY(begin(c, lre::ws_bytes_micro_contrast(w, h) + (mask ? w * h * sizeof(float) + 256 : 0)));
  const size_t bytes = w * h * 3 * sizeof(float);
  LRE_TRY(lre::ensure_buffer(c, &c->d_in, &c->d_in_cap, bytes));
  float* d = reinterpret_cast<float*>(c->d_in);
  LRE_TRY(lre::copy_h2d(c, d, in, bytes, c->stream));
  float* dmask = nullptr;
  if (mask) {
    dmask = reinterpret_cast<float*>(c->ws.take(w * h * sizeof(float)));
    LRE_TRY(lre::copy_h2d(c, dmask, mask, w * h * sizeof(float), c->stream));
  }
  LRE_TRY(lre::launch_micro_contrast(c, d, d, w, h, thr, strength, target, dmask));
  LRE_TRY(lre::copy_d2h(c, out, d, bytes, c->stream));
  LRE_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  return LRE_OK;
}

// ------------------------------------------------------------ lateral CA
lre_status lre_dev_ca_register_lateral(lre_ctx* ctx, const float* in, float* out, size_t w, size_t h, int cell,
                                       int iters, float max_shift, float min_conf, int levels) {
  Context* c = C(ctx);
  if (!c) return LRE_ERR_INVALID_ARGUMENT;
  LRE_TRY(check_img(c, in, out, w, h, "ca_register_lateral"));
  LRE_TRY(begin(c, lre::ws_bytes_lateral(w, h, cell, levels, in == out)));
  return lre::launch_lateral_ca(c, in, out, w, h, cell, iters, max_shift, min_conf, levels);
}

lre_status lre_ca_register_lateral(lre_ctx* ctx, const float* in, float* out, size_t w, size_t h, int cell, int iters,
                                   float max_shift, float min_conf, int levels) {
  Context* c = C(ctx);
  if (!c) return LRE_ERR_INVALID_ARGUMENT;
  LRE_TRY(check_img(c, in, out, w, h, "ca_register_lateral"));
  return host_rgb_stage(c, in, out, w, h, lre::ws_bytes_lateral(w, h, cell, levels, true), [&](float* d) {
    return lre::launch_lateral_ca(c, d, d, w, h, cell, iters, max_shift, min_conf, levels);
  });
}

// ------------------------------------------------------------ demosaic
lre_status lre_dev_demosaic_bayer_amaze(lre_ctx* ctx, const float* raw, float* rgb, size_t w, size_t h,
                                        uint32_t filters, const float cam_mul[4], float maximum_value) {
  Context* c = C(ctx);
  if (!c) return LRE_ERR_INVALID_ARGUMENT;
  LRE_TRY(check_img(c, raw, rgb, w, h, "demosaic_bayer_amaze"));
  if (!cam_mul) return lre::fail(c, LRE_ERR_INVALID_ARGUMENT, "demosaic_bayer_amaze: null cam_mul");
  if (filters == LRE_FILTERS_XTRANS || filters < 1000)
    return lre::fail(c, LRE_ERR_INVALID_ARGUMENT, "demosaic_bayer_amaze: not a Bayer filters word");
  LRE_TRY(begin(c, lre::ws_bytes_amaze(w, h)));
  return lre::launch_amaze(c, raw, 1, rgb, w, h, filters, cam_mul, maximum_value);
}

lre_status lre_dev_demosaic_bayer_linear(lre_ctx* ctx, const float* raw, float* rgb, size_t w, size_t h,
                                         uint32_t filters, float maximum_value) {
  Context* c = C(ctx);
  if (!c) return LRE_ERR_INVALID_ARGUMENT;
  LRE_TRY(check_img(c, raw, rgb, w, h, "demosaic_bayer_linear"));
  if (filters == LRE_FILTERS_XTRANS || filters < 1000)
    return lre::fail(c, LRE_ERR_INVALID_ARGUMENT, "demosaic_bayer_linear: not a Bayer filters word");
  cudaSetDevice(c->device);
  LRE_TRY(lre::check_injection(c));
  return lre::launch_bayer_linear(c, raw, 1, rgb, w, h, filters, maximum_value);
}

lre_status lre_demosaic_bayer_linear(lre_ctx* ctx, const float* raw_rgb, float* rgb, size_t w, size_t h,
                                     uint32_t filters, float maximum_value) {
  Context* c = C(ctx);
  if (!c) return LRE_ERR_INVALID_ARGUMENT;
  LRE_TRY(check_img(c, raw_rgb, rgb, w, h, "demosaic_bayer_linear"));
  if (filters == LRE_FILTERS_XTRANS || filters < 1000)
    return lre::fail(c, LRE_ERR_INVALID_ARGUMENT, "demosaic_bayer_linear: not a Bayer filters word");
  std::lock_guard<std::mutex> lk(c->mu);
  LRE_TRY(begin(c, 0));
  const size_t bytes = w * h * 3 * sizeof(float);
  LRE_TRY(lre::ensure_buffer(c, &c->d_in, &c->d_in_cap, bytes));
  LRE_TRY(lre::ensure_buffer(c, &c->d_out, &c->d_out_cap, bytes));
  float* din = reinterpret_cast<float*>(c->d_in);
  float* dout = reinterpret_cast<float*>(c->d_out);
  LRE_TRY(lre::copy_h2d(c, din, raw_rgb, bytes, c->stream));
  LRE_TRY(lre::launch_bayer_linear(c, din, 3, dout, w, h, filters, maximum_value));
  LRE_TRY(lre::copy_d2h(c, rgb, dout, bytes, c->stream));
  LRE_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  return LRE_OK;
}

lre_status lre_dev_demosaic_bayer_dcb(lre_ctx* ctx, const float* raw, float* rgb, size_t w, size_t h,
                                      uint32_t filters, float maximum_value, int iterations, int dcb_enhance) {
  Context* c = C(ctx);
  if (!c) return LRE_ERR_INVALID_ARGUMENT;
  LRE_TRY(check_img(c, raw, rgb, w, h, "demosaic_bayer_dcb"));
  LRE_TRY(begin(c, lre::ws_bytes_dcb(w, h)));
  return lre::launch_dcb(c, raw, 1, rgb, w, h, filters, maximum_value, iterations, dcb_enhance != 0, nullptr);
}

lre_status lre_demosaic_bayer_dcb(lre_ctx* ctx, const float* raw_rgb, float* rgb, size_t w, size_t h,
                                  uint32_t filters, float maximum_value, int iterations, int dcb_enhance) {
  Context* c = C(ctx);
  if (!c) return LRE_ERR_INVALID_ARGUMENT;
  LRE_TRY(check_img(c, raw_rgb, rgb, w, h, "demosaic_bayer_dcb"));
  std::lock_guard<std::mutex> lk(c->mu);
  LRE_TRY(begin(c, lre::ws_bytes_dcb(w, h)));
  const size_t bytes = w * h * 3 * sizeof(float);
  LRE_TRY(lre::ensure_buffer(c, &c->d_in, &c->d_in_cap, bytes));
  LRE_TRY(lre::ensure_buffer(c, &c->d_out, &c->d_out_cap, bytes));
  float* din = reinterpret_cast<float*>(c->d_in);
  float* dout = reinterpret_cast<float*>(c->d_out);
  LRE_TRY(lre::copy_h2d(c, din, raw_rgb, bytes, c->stream));
  LRE_TRY(lre::launch_dcb(c, din, 3, dout, w, h, filters, maximum_value, iterations, dcb_enhance != 0, nullptr));
  LRE_TRY(lre::copy_d2h(c, rgb, dout, bytes, c->stream));
  LRE_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  return LRE_OK;
}

lre_status lre_dev_recover_highlights(lre_ctx* ctx, const float* in, float* out, size_t w, size_t h, float thr,
                                      float* mask_out, const float* wb_rgb, float* max_val_out) {
  Context* c = C(ctx);
  if (!c) return LRE_ERR_INVALID_ARGUMENT;
  LRE_TRY(check_img(c, in, out, w, h, "recover_highlights"));
  LRE_TRY(begin(c, lre::ws_bytes_highlights(w, h)));
  return lre::launch_recover_highlights(c, in, out, w, h, thr, mask_out, wb_rgb, max_val_out, nullptr);
}

lre_status lre_recover_highlights(lre_ctx* ctx, const float* in, float* out, size_t w, size_t h, float thr,
                                  float* mask_out, const float* wb_rgb, float* max_val_out) {
  Context* c = C(ctx);
  if (!c) return LRE_ERR_INVALID_ARGUMENT;
  LRE_TRY(check_img(c, in, out, w, h, "recover_highlights"));
  std::lock_guard<std::mutex> lk(c->mu);
  LRE_TRY(begin(c, lre::ws_bytes_highlights(w, h)));
  const size_t bytes = w * h * 3 * sizeof(float);
  const size_t mbytes = w * h * sizeof(float);
  LRE_TRY(lre::ensure_buffer(c, &c->d_in, &c->d_in_cap, bytes));
  LRE_TRY(lre::ensure_buffer(c, &c->d_out, &c->d_out_cap, bytes));
  if (mask_out) LRE_TRY(lre::ensure_buffer(c, &c->d_aux, &c->d_aux_cap, mbytes));
  float* din = reinterpret_cast<float*>(c->d_in);
  float* dout = reinterpret_cast<float*>(c->d_out);
  float* dmask = mask_out ? reinterpret_cast<float*>(c->d_aux) : nullptr;
  float* dmax = c->d_scalars + 40;
  LRE_TRY(lre::copy_h2d(c, din, in, bytes, c->stream));
  LRE_TRY(lre::launch_recover_highlights(c, din, dout, w, h, thr, dmask, wb_rgb, dmax, nullptr));
  LRE_TRY(lre::copy_d2h(c, out, dout, bytes, c->stream));
  if (mask_out) LRE_TRY(lre::copy_d2h(c, mask_out, dmask, mbytes, c->stream));
  if (max_val_out) LRE_CUDA_TRY(c, cudaMemcpyAsync(max_val_out, dmax, sizeof(float), cudaMemcpyDeviceToHost, c->stream));
  LRE_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  return LRE_OK;
}

lre_status lre_dev_demosaic_bayer_aahd(lre_ctx* ctx, const float* raw, float* rgb, size_t w, size_t h,
                                       uint32_t filters, float maximum_value) {
  Context* c = C(ctx);
  if (!c) return LRE_ERR_INVALID_ARGUMENT;
  LRE_TRY(check_img(c, raw, rgb, w, h, "demosaic_bayer_aahd"));
  LRE_TRY(begin(c, lre::ws_bytes_aahd(w, h)));
  return lre::launch_aahd(c, raw, 1, rgb, w, h, filters, maximum_value, nullptr);
}

lre_status lre_demosaic_bayer_aahd(lre_ctx* ctx, const float* raw_rgb, float* rgb, size_t w, size_t h,
                                   uint32_t filters, float maximum_value) {
  Context* c = C(ctx);
  if (!c) return LRE_ERR_INVALID_ARGUMENT;
  LRE_TRY(check_img(c, raw_rgb, rgb, w, h, "demosaic_bayer_aahd"));
  std::lock_guard<std::mutex> lk(c->mu);
  LRE_TRY(begin(c, lre::ws_bytes_aahd(w, h)));
  const size_t bytes = w * h * 3 * sizeof(float);
  LRE_TRY(lre::ensure_buffer(c, &c->d_in, &c->d_in_cap, bytes));
  LRE_TRY(lre::ensure_buffer(c, &c->d_out, &c->d_out_cap, bytes));
  float* din = reinterpret_cast<float*>(c->d_in);
  float* dout = reinterpret_cast<float*>(c->d_out);
  LRE_TRY(lre::copy_h2d(c, din, raw_rgb, bytes, c->stream));
  LRE_TRY(lre::launch_aahd(c, din, 3, dout, w, h, filters, maximum_value, nullptr));
  LRE_TRY(lre::copy_d2h(c, rgb, dout, bytes, c->stream));
  LRE_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  return LRE_OK;
}

lre_status lre_demosaic_bayer_amaze(lre_ctx* ctx, const float* raw_rgb, float* rgb, size_t w, size_t h,
                                    uint32_t filters, const float cam_mul[4], float maximum_value) {
  Context* c = C(ctx);
  if (!c) return LRE_ERR_INVALID_ARGUMENT;
  LRE_TRY(check_img(c, raw_rgb, rgb, w, h, "demosaic_bayer_amaze"));
  if (!cam_mul) return lre::fail(c, LRE_ERR_INVALID_ARGUMENT, "demosaic_bayer_amaze: null cam_mul");
  if (filters == LRE_FILTERS_XTRANS || filters < 1000)
    return lre::fail(c, LRE_ERR_INVALID_ARGUMENT, "demosaic_bayer_amaze: not a Bayer filters word");
  std::lock_guard<std::mutex> lk(c->mu);
  LRE_TRY(begin(c, lre::ws_bytes_amaze(w, h)));
  const size_t bytes = w * h * 3 * sizeof(float);
  LRE_TRY(lre::ensure_buffer(c, &c->d_in, &c->d_in_cap, bytes));
  LRE_TRY(lre::ensure_buffer(c, &c->d_out, &c->d_out_cap, bytes));
  float* din = reinterpret_cast<float*>(c->d_in);
  float* dout = reinterpret_cast<float*>(c->d_out);
  LRE_TRY(lre::copy_h2d(c, din, raw_rgb, bytes, c->stream));
  LRE_TRY(lre::launch_amaze(c, din, 3, dout, w, h, filters, cam_mul, maximum_value));
  LRE_TRY(lre::copy_d2h(c, rgb, dout, bytes, c->stream));
  LRE_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  return LRE_OK;
}

static lre_status xtrans_host(lre_ctx* ctx, const float* raw_rgb, float* rgb, size_t w, size_t h, const char* xtrans,
                              float maximum_value, int passes) {
  Context* c = C(ctx);
  if (!c) return LRE_ERR_INVALID_ARGUMENT;
  LRE_TRY(check_img(c, raw_rgb, rgb, w, h, "demosaic_xtrans"));
  if (!xtrans) return lre::fail(c, LRE_ERR_INVALID_ARGUMENT, "demosaic_xtrans: null xtrans pattern");
  std::lock_guard<std::mutex> lk(c->mu);
  LRE_TRY(begin(c, lre::ws_bytes_xtrans(w, h, passes, xtrans)));
  const size_t bytes = w * h * 3 * sizeof(float);
  LRE_TRY(lre::ensure_buffer(c, &c->d_in, &c->d_in_cap, bytes));
  LRE_TRY(lre::ensure_buffer(c, &c->d_out, &c->d_out_cap, bytes));
  float* din = reinterpret_cast<float*>(c->d_in);
  float* dout = reinterpret_cast<float*>(c->d_out);
  LRE_TRY(lre::copy_h2d(c, din, raw_rgb, bytes, c->stream));
  LRE_TRY(lre::launch_xtrans(c, din, 3, dout, w, h, xtrans, maximum_value, passes));
  LRE_TRY(lre::copy_d2h(c, rgb, dout, bytes, c->stream));
  LRE_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  return LRE_OK;
}

lre_status lre_demosaic_xtrans_1pass(lre_ctx* ctx, const float* raw_rgb, float* rgb, size_t w, size_t h,
                                     const char xtrans[36], const float color_matrix[12], float maximum_value) {
  (void)color_matrix;
  return xtrans_host(ctx, raw_rgb, rgb, w, h, xtrans, maximum_value, 1);
}

lre_status lre_demosaic_xtrans_3pass(lre_ctx* ctx, const float* raw_rgb, float* rgb, size_t w, size_t h,
                                     const char xtrans[36], const float color_matrix[12], float maximum_value) {
  (void)color_matrix;
  return xtrans_host(ctx, raw_rgb, rgb, w, h, xtrans, maximum_value, 3);
}

lre_status lre_dev_demosaic_xtrans(lre_ctx* ctx, const float* raw, float* rgb, size_t w, size_t h, const char xtrans[36],
                                   float maximum_value, int passes) {
  Context* c = C(ctx);
  if (!c) return LRE_ERR_INVALID_ARGUMENT;
  LRE_TRY(check_img(c, raw, rgb, w, h, "demosaic_xtrans"));
  if (!xtrans) return lre::fail(c, LRE_ERR_INVALID_ARGUMENT, "demosaic_xtrans: null xtrans pattern");
  LRE_TRY(begin(c, lre::ws_bytes_xtrans(w, h, passes, xtrans)));
  return lre::launch_xtrans(c, raw, 1, rgb, w, h, xtrans, maximum_value, passes);
}

// ------------------------------------------------------------ white balance
lre_status lre_apply_white_balance(lre_ctx* ctx, const uint16_t* raw4, float* rgb, size_t w, size_t h,
                                   const float wb[4], uint32_t filters, const char xtrans[36]) {
  Context* c = C(ctx);
  if (!c) return LRE_ERR_INVALID_ARGUMENT;
  LRE_TRY(check_img(c, raw4, rgb, w, h, "apply_white_balance"));
  if (!wb) return lre::fail(c, LRE_ERR_INVALID_ARGUMENT, "apply_white_balance: null wb");
  if (filters == LRE_FILTERS_XTRANS && !xtrans)
    return lre::fail(c, LRE_ERR_INVALID_ARGUMENT, "apply_white_balance: null xtrans pattern");
  std::lock_guard<std::mutex> lk(c->mu);
  LRE_TRY(begin(c, 0));
  const size_t in_bytes = w * h * 4 * sizeof(uint16_t), out_bytes = w * h * 3 * sizeof(float);
  LRE_TRY(lre::ensure_buffer(c, &c->d_in, &c->d_in_cap, in_bytes));
  LRE_TRY(lre::ensure_buffer(c, &c->d_out, &c->d_out_cap, out_bytes));
  LRE_TRY(lre::copy_h2d(c, c->d_in, raw4, in_bytes, c->stream));
  // untouched channels keep the caller's values, as in the reference
  LRE_TRY(lre::copy_h2d(c, c->d_out, rgb, out_bytes, c->stream));
  LRE_TRY(lre::launch_white_balance(c, reinterpret_cast<const uint16_t*>(c->d_in), reinterpret_cast<float*>(c->d_out),
                                    w, h, wb, filters, xtrans));
  LRE_TRY(lre::copy_d2h(c, rgb, c->d_out, out_bytes, c->stream));
  LRE_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  return LRE_OK;
}

// ------------------------------------------------------------ integer pieces
lre_status lre_black_level(lre_ctx* ctx, uint16_t* raw4, size_t w, size_t h, const unsigned* cblack,
                           size_t cblack_len, unsigned black, unsigned maximum) {
  Context* c = C(ctx);
  if (!c) return LRE_ERR_INVALID_ARGUMENT;
  LRE_TRY(check_img(c, raw4, raw4, w, h, "black_level"));
  if (!cblack || cblack_len < 6) return lre::fail(c, LRE_ERR_INVALID_ARGUMENT, "black_level: cblack needs >= 6 entries");
  std::lock_guard<std::mutex> lk(c->mu);
  LRE_TRY(begin(c, (cblack_len + 64) * sizeof(unsigned) + 256));
  const size_t bytes = w * h * 4 * sizeof(uint16_t);
  LRE_TRY(lre::ensure_buffer(c, &c->d_in, &c->d_in_cap, bytes));
  LRE_TRY(lre::copy_h2d(c, c->d_in, raw4, bytes, c->stream));
  LRE_TRY(lre::launch_black_level(c, reinterpret_cast<uint16_t*>(c->d_in), w, h, cblack, cblack_len, black, maximum));
  LRE_TRY(lre::copy_d2h(c, raw4, c->d_in, bytes, c->stream));
  LRE_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  return LRE_OK;
}

lre_status lre_adjust_maximum(lre_ctx* ctx, const float* raw_rgb, size_t w, size_t h, uint32_t filters, float threshold,
                              float* data_maximum, float* maximum) {
  Context* c = C(ctx);
  if (!c) return LRE_ERR_INVALID_ARGUMENT;
  if (!data_maximum || !maximum) return lre::fail(c, LRE_ERR_INVALID_ARGUMENT, "adjust_maximum: null result pointer");
  // core/libraw_wrapper.cpp:1010-1087
  if (threshold < 0.00001f) return LRE_OK;
  float thr = threshold > 0.99999f ? 0.75f : threshold;
  float real_max = *data_maximum;
  if (real_max == 0.f && raw_rgb) {
    LRE_TRY(check_img(c, raw_rgb, raw_rgb, w, h, "adjust_maximum"));
    std::lock_guard<std::mutex> lk(c->mu);
    LRE_TRY(begin(c, 0));
    const size_t bytes = w * h * 3 * sizeof(float);
    LRE_TRY(lre::ensure_buffer(c, &c->d_in, &c->d_in_cap, bytes));
    LRE_TRY(lre::copy_h2d(c, c->d_in, raw_rgb, bytes, c->stream));
    LRE_TRY(lre::launch_cfa_max(c, reinterpret_cast<const float*>(c->d_in), 3, w, h, filters, c->d_scalars));
    LRE_CUDA_TRY(c, cudaMemcpyAsync(&real_max, c->d_scalars, sizeof(float), cudaMemcpyDeviceToHost, c->stream));
    LRE_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    *data_maximum = real_max;
  }
  float cur = *maximum;
  if (real_max > 0 && real_max < cur && real_max > cur * thr) *maximum = real_max;
  return LRE_OK;
}

lre_status lre_dev_quantize_u16(lre_ctx* ctx, const float* in, uint16_t* out, size_t n) {
  Context* c = C(ctx);
  if (!c || !in || !out) return LRE_ERR_INVALID_ARGUMENT;
  LRE_TRY(begin(c, 0));
  return lre::launch_quantize_u16(c, in, out, n);
}

static lre_status quantize_host(lre_ctx* ctx, const float* in, void* out, size_t n, int bits) {
  Context* c = C(ctx);
  if (!c) return LRE_ERR_INVALID_ARGUMENT;
  if (!in || !out) return lre::fail(c, LRE_ERR_INVALID_ARGUMENT, "quantize: null buffer");
  if (n == 0) return LRE_OK;
  std::lock_guard<std::mutex> lk(c->mu);
  LRE_TRY(begin(c, 0));
  const size_t ob = n * (bits == 16 ? 2 : 1);
  LRE_TRY(lre::ensure_buffer(c, &c->d_in, &c->d_in_cap, n * sizeof(float)));
  LRE_TRY(lre::ensure_buffer(c, &c->d_out, &c->d_out_cap, ob));
  LRE_TRY(lre::copy_h2d(c, c->d_in, in, n * sizeof(float), c->stream));
  if (bits == 16)
    LRE_TRY(lre::launch_quantize_u16(c, reinterpret_cast<float*>(c->d_in), reinterpret_cast<uint16_t*>(c->d_out), n));
  else
    LRE_TRY(lre::launch_quantize_u8(c, reinterpret_cast<float*>(c->d_in), reinterpret_cast<uint8_t*>(c->d_out), n));
  LRE_TRY(lre::copy_d2h(c, out, c->d_out, ob, c->stream));
  LRE_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  return LRE_OK;
}

lre_status lre_quantize_u16(lre_ctx* ctx, const float* in, uint16_t* out, size_t n) {
  return quantize_host(ctx, in, out, n, 16);
}
lre_status lre_quantize_u8(lre_ctx* ctx, const float* in, uint8_t* out, size_t n) {
  return quantize_host(ctx, in, out, n, 8);
}


lre_status lre_convert_color_space(lre_ctx* ctx, const float* in, float* out, size_t w, size_t h,
                                   const float transform[12]) {
  Context* c = C(ctx);
  if (!c) return LRE_ERR_INVALID_ARGUMENT;
  if (!in || !out || !transform || w == 0 || h == 0)
    return lre::fail(c, LRE_ERR_INVALID_ARGUMENT, "convert_color_space: bad arguments");
  return host_rgb_stage(c, in, out, w, h, 0, [&](float* d) { return lre::launch_color_space(c, d, d, w * h, transform); });
}

lre_status lre_gamma_correct(lre_ctx* ctx, const float* in, float* out, size_t w, size_t h, float gamma_power,
                             float gamma_slope, int output_color_space) {
  Context* c = C(ctx);
  if (!c) return LRE_ERR_INVALID_ARGUMENT;
  if (!in || !out || w == 0 || h == 0) return lre::fail(c, LRE_ERR_INVALID_ARGUMENT, "gamma_correct: bad arguments");
  return host_rgb_stage(c, in, out, w, h, 0, [&](float* d) {
    return lre::launch_gamma(c, d, d, w * h, gamma_power, gamma_slope, output_color_space);
  });
}

lre_status lre_dev_convert_color_space(lre_ctx* ctx, const float* in, float* out, size_t w, size_t h,
                                       const float transform[12]) {
  Context* c = C(ctx);
  if (!c) return LRE_ERR_INVALID_ARGUMENT;
  if (!in || !out || !transform) return lre::fail(c, LRE_ERR_INVALID_ARGUMENT, "convert_color_space: null argument");
  cudaSetDevice(c->device);
  return lre::launch_color_space(c, in, out, w * h, transform);
}

lre_status lre_dev_gamma_correct(lre_ctx* ctx, const float* in, float* out, size_t w, size_t h, float gamma_power,
                                 float gamma_slope, int output_color_space) {
  Context* c = C(ctx);
  if (!c) return LRE_ERR_INVALID_ARGUMENT;
  if (!in || !out) return lre::fail(c, LRE_ERR_INVALID_ARGUMENT, "gamma_correct: null argument");
  cudaSetDevice(c->device);
  return lre::launch_gamma(c, in, out, w * h, gamma_power, gamma_slope, output_color_space);
}

}  // extern "C"
