// lre_internal.h -- host-side runtime shared by the CUDA translation units.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <functional>
#include <cstddef>
#include <cstdint>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/lre_cuda.h"

namespace lre {

class HostStager;  // pinned bounce ring for pageable host buffers (host_stage.cu)

// One 256-byte-aligned bump arena on the device.  `reset()` releases every
// allocation at once; the arena only grows (reallocation synchronises the
// stream first, so pointers handed out earlier in the same call stay valid
// only until the next reset).
class Workspace {
 public:
  ~Workspace();
  cudaError_t reserve(size_t bytes, cudaStream_t s);
  // Returns nullptr when the arena is too small; callers size it first with
  // reserve() from the plan of the stage they run.
  void* take(size_t bytes);
  void reset() { used_ = 0; }
  // Frees the arena (the caller has synchronised every stream using it).
  void release();
  void rewind(size_t mark) { used_ = mark; }
  size_t capacity() const { return cap_; }
  size_t used() const { return used_; }

 private:
  char* base_ = nullptr;
  size_t cap_ = 0;
  size_t used_ = 0;
};

// Planner for workspace use: stage code first sums its buffers with add(),
// the context reserves the total, then the same sizes are taken in order.
struct WsPlan {
  size_t total = 0;
  size_t add(size_t bytes) {
    size_t off = total;
    total += (bytes + 255) & ~size_t(255);
    return off;
  }
};

// Kernel-shape choices that do not change results (picked by the batch
// autotuner, or set with lre_set_tuning).
struct Tuning {
  int axial_strip = 128;    // guided-filter strip width (columns per CTA): 128 or 64
  int axial_rows = 128;     // guided-filter output rows per CTA: 128 or 64
  int blur_tile = 64;       // defringe register-tiled blur output tile edge: 64 or 32
};

struct Context {
  int device = 0;
  Tuning tune;
  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;
  Workspace ws;
  std::string last_error;
  std::atomic<uint64_t> launches{0};
  int inject_countdown = 0;
  // staging for host-buffer entry points
  void* d_in = nullptr;
  size_t d_in_cap = 0;
  void* d_out = nullptr;
  size_t d_out_cap = 0;
  void* d_aux = nullptr;
  size_t d_aux_cap = 0;
  float* d_scalars = nullptr;  // 64 floats of per-call scalars (reductions)
  // Host-buffer develop: a copy stream and events so the mosaic upload
  // overlaps the demosaic (created on first use, destroyed with the context).
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t band_ev[8] = {};
  cudaEvent_t tail_ev[8] = {};  // rows of the final RGB ready for download
  std::mutex mu;               // one host-buffer call at a time per context
  int sm_count = 148;
  // Bound of each device-side wait of the in-order sweeps, in SM clock
  // cycles (0: the default, ~2 s), and a one-shot host-side fault injection:
  // the next sweep's band `sweep_hold_band` never reports its progress.
  long long sweep_wait_cycles = 0;
  int sweep_hold_band = -1;
  HostStager* stager = nullptr;  // created on the first large pageable copy
};

// Host <-> device copies of the host-buffer entry points (host_stage.cu):
// pageable buffers above a few MB go through the context's pinned chunk ring
// with a parallel host memcpy; page-locked buffers and small copies are
// direct.  copy_h2d returns once the source may be reused; copy_d2h returns
// when the data is in `dst` (it synchronises `s`).
lre_status copy_h2d(Context* c, void* dst, const void* src, size_t bytes, cudaStream_t s);
lre_status copy_d2h(Context* c, void* dst, const void* src, size_t bytes, cudaStream_t s);
void destroy_stager(Context* c);

// Status helpers.
lre_status fail(Context* c, lre_status st, const std::string& msg);
lre_status cuda_fail(Context* c, cudaError_t e, const char* what);
lre_status check_launch(Context* c, const char* what);
lre_status check_injection(Context* c);

#define LRE_CUDA_TRY(ctx, call)                                        \
  do {                                                                 \
    cudaError_t _e = (call);                                           \
    if (_e != cudaSuccess) return ::lre::cuda_fail((ctx), _e, #call);  \
  } while (0)

#define LRE_TRY(expr)                    \
  do {                                   \
    lre_status _s = (expr);              \
    if (_s != LRE_OK) return _s;         \
  } while (0)

// Grow-only device buffers used by the host-buffer entry points.
lre_status ensure_buffer(Context* c, void** p, size_t* cap, size_t bytes);

inline unsigned grid_for(size_t n, unsigned block, unsigned max_blocks = 148u * 16u) {
  size_t g = (n + block - 1) / block;
  if (g < 1) g = 1;
  if (g > max_blocks) g = max_blocks;
  return (unsigned)g;
}

inline void count_launch(Context* c, uint64_t n = 1) { c->launches.fetch_add(n); }

// --- stage launchers (device pointers, enqueue on c->stream) -------------
lre_status launch_tone_mapping(Context* c, const float* in, float* out, size_t n_px, float after_scale);
lre_status launch_white_balance(Context* c, const uint16_t* raw4, float* rgb, size_t w, size_t h,
                                const float wb[4], uint32_t filters, const char* xtrans);
lre_status launch_black_level(Context* c, uint16_t* raw4, size_t w, size_t h, const unsigned* cblack,
                              size_t cblack_len, unsigned black, unsigned maximum);
lre_status launch_cfa_max(Context* c, const float* raw, int raw_c_stride, size_t w, size_t h,
                          uint32_t filters, float* d_out);
lre_status launch_quantize_u16(Context* c, const float* in, uint16_t* out, size_t n);
lre_status launch_quantize_u8(Context* c, const float* in, uint8_t* out, size_t n);
lre_status launch_pack_cfa(Context* c, const float* raw_rgb, float* dense, size_t w, size_t h,
                           uint32_t filters, const char* xtrans);
lre_status launch_channel_max(Context* c, const float* rgb, size_t n_px, int channel, float* d_out,
                              bool clamp0);
// tone_scale >= 0: the ACES tone map (after_scale tone_scale) that follows
// the filter is applied to its output in the same pass (bit for bit the
// separate stage); < 0: plain filter output.
lre_status launch_axial_ca(Context* c, const float* in, float* out, size_t w, size_t h, int radius,
                           float eps, float strength, const float* d_max_g, float tone_scale = -1.f);
// The guided filter in row bands (out of place): after pass B of each band,
// rows_done(row_lo, row_hi) enqueues what may follow on those rows.
lre_status launch_axial_ca_banded(Context* c, const float* in, float* out, size_t w, size_t h, int radius, float eps,
                                  float strength, const float* d_max_g, int bands,
                                  const std::function<lre_status(size_t, size_t)>& rows_done,
                                  float tone_scale = -1.f);
// in_max_g (nullable): max(0, max G) of `in`, already reduced on the device
// by the stage that wrote it (the defringe then skips its own reduction).
// out_max_g (nullable): receives max(0, max G) of `out`, reduced in the
// main pass for the stage that follows.
lre_status launch_defringe(Context* c, const float* in, float* out, size_t w, size_t h, float radius,
                           float edge_thr, float chroma_thr, float strength, bool green,
                           float green_scale, const float* in_max_g = nullptr, float* out_max_g = nullptr);
lre_status launch_detail_tonemap(Context* c, const float* in, float* out, size_t w, size_t h);
lre_status launch_micro_contrast(Context* c, const float* in, float* out, size_t w, size_t h,
                                 float threshold, float strength, float target, const float* mask);
lre_status launch_lateral_ca(Context* c, const float* in, float* out, size_t w, size_t h, int cell,
                             int iters, float max_shift, float min_conf, int levels);
// max_g (nullable): receives max(0, max G) of the finished RGB (AMaZE's
// interior outputs and the interpolated border), reduced in the kernels.
lre_status launch_amaze(Context* c, const float* raw, int raw_c_stride, float* rgb, size_t w, size_t h,
                        uint32_t filters, const float cam_mul[4], float maximum_value, float* max_g = nullptr);
// AMaZE on a mosaic still in host memory: the upload runs in row chunks on
// copy_stream and each band of tile rows starts as soon as the rows it reads
// have arrived (results identical to launch_amaze).  d_mosaic receives the
// whole mosaic.
lre_status launch_amaze_from_host(Context* c, const float* h_mosaic, float* d_mosaic, float* rgb, size_t w,
                                  size_t h, uint32_t filters, const float cam_mul[4], float maximum_value,
                                  cudaStream_t copy_stream, cudaEvent_t* events, int n_events,
                                  float* max_g = nullptr);
lre_status launch_xtrans(Context* c, const float* raw, int raw_c_stride, float* rgb, size_t w,
                         size_t h, const char* xtrans, float maximum_value, int passes);

// Workspace bytes each stage needs for a w x h image (0 when none).
size_t ws_bytes_axial(size_t w, size_t h, int radius);
size_t ws_bytes_defringe(size_t w, size_t h, float radius);
size_t ws_bytes_detail_tonemap(size_t w, size_t h);
size_t ws_bytes_micro_contrast(size_t w, size_t h);
size_t ws_bytes_lateral(size_t w, size_t h, int cell, int levels, bool in_place);
size_t ws_bytes_amaze(size_t w, size_t h);
// xtrans (nullable): the 6x6 pattern; with it the size is that of the kernel
// the pattern selects, without it the larger of the two.
size_t ws_bytes_xtrans(size_t w, size_t h, int passes, const char* xtrans = nullptr);

}  // namespace lre

namespace lre {
// The per-image develop chain (pipeline.cu), shared by the plain entry
// points, the batch runner and the request server.
lre_status develop_validate(Context* c, const lre_develop_params* p, size_t w, size_t h);
size_t develop_ws_bytes(const lre_develop_params& p, size_t w, size_t h);
lre_status develop_device(Context* c, const float* mosaic, void* out, size_t w, size_t h,
                          const lre_develop_params& p);
}  // namespace lre

namespace lre {
// On-device raw ingest (k_ingest.cu).
size_t raw_image_elems(const lre_raw_frame& f);
lre_status launch_raw2image(Context* c, const uint16_t* raw, const lre_raw_frame& f, uint16_t* image4);
lre_status launch_green_matching(Context* c, uint16_t* raw4, const uint16_t* copy, size_t w, size_t h,
                                 uint32_t filters, unsigned maximum);
lre_status launch_wb_dense(Context* c, const uint16_t* raw4, float* dense, size_t w, size_t h, const float wb[4],
                           uint32_t filters, const char* xtrans);
lre_status launch_cfa_max_dense(Context* c, const float* dense, size_t w, size_t h, uint32_t filters,
                                const char* xtrans, float* d_out);
// scale_colors' multipliers (k_wb.cu): the auto-WB channel sums of the
// device uint16[4] image when needed (synchronises), then the host logic.
bool wb_needs_sums(const lre_wb_inputs& in);
lre_status wb_multipliers(const lre_wb_inputs& in, uint32_t filters, unsigned maximum, unsigned black,
                          const uint64_t* sums, const uint64_t* counts, lre_wb_result* out);
lre_status derive_wb_device(Context* c, const uint16_t* d_raw4, size_t w, size_t h, uint32_t filters,
                            const char* xtrans, unsigned maximum, unsigned black, const lre_wb_inputs& in,
                            lre_wb_result* out);
}  // namespace lre

namespace lre {
// Output end of the pipeline (k_output.cu).
lre_status launch_color_space(Context* c, const float* in, float* out, size_t n_px, const float transform[12]);
lre_status launch_gamma(Context* c, const float* in, float* out, size_t n_px, float gamma_power, float gamma_slope,
                        int color_space);
lre_status launch_output_epilogue(Context* c, const float* in, void* out, size_t n_px, const float transform[12],
                                  float gamma_power, float gamma_slope, int color_space, int bits);
}  // namespace lre

namespace lre {
// LibRaw border interpolation of the `band`-px frame (k_amaze.cu) and the
// bilinear Bayer demosaic (k_linear.cu).
// max_g (nullable): the max of the border pixels' final G is folded into it.
lre_status launch_border_interp(Context* c, float* rgb, size_t w, size_t h, uint32_t filters, int band,
                                float* max_g = nullptr);
lre_status launch_bayer_linear(Context* c, const float* raw, int raw_c_stride, float* rgb, size_t w, size_t h,
                               uint32_t filters, float maximum_value);
// DCB and AAHD Bayer demosaics (k_dcb.cu, k_aahd.cu).  Their in-order
// sweeps raise a device error flag if a band's bounded wait expires.  With
// d_err == nullptr the launcher synchronises the stream and reports the flag
// as LRE_ERR_TIMEOUT; otherwise it ORs into *d_err (device) and returns
// without synchronising.
size_t ws_bytes_dcb(size_t w, size_t h);
lre_status launch_dcb(Context* c, const float* raw, int raw_c_stride, float* rgb, size_t w, size_t h,
                      uint32_t filters, float maximum_value, int iterations, bool enhance, int* d_err);
size_t ws_bytes_aahd(size_t w, size_t h);
// Highlight recovery (k_highlights.cu).  in may equal out; mask_out (W*H
// floats, device) and d_max_val_out (device) may be null; wb_rgb is host.
// d_err follows the DCB/AAHD convention above.
size_t ws_bytes_highlights(size_t w, size_t h);
lre_status launch_recover_highlights(Context* c, const float* in, float* out, size_t w, size_t h,
                                     float saturation_threshold, float* mask_out, const float* wb_rgb,
                                     float* d_max_val_out, int* d_err);
// Uploads AAHD's gamma table to the context's device (once per device).
lre_status aahd_upload_gamma(Context* c);
// True for filters words with a 2x2 Bayer layout (green checkerboard, R and
// B on the other two sites), which DCB and AAHD need.
bool bayer_2x2_layout(uint32_t filters);
lre_status launch_aahd(Context* c, const float* raw, int raw_c_stride, float* rgb, size_t w, size_t h,
                       uint32_t filters, float maximum_value, int* d_err);
}  // namespace lre
