// pipeline.cu -- the plain per-image develop: one upload of the CFA mosaic,
// every stage on device-resident buffers, one download.
//
// Stage order follows process_raw_to_rgb (core/libraw_wrapper.cpp:1477-1853):
// demosaic -> tone map -> lateral CA -> axial CA -> defringe, or, with
// stage_order = 1, demosaic -> defringe -> axial CA -> tone map (the order of
// the 51 MP develop workload).  Only the axial guided filter reads a
// neighbourhood of the previous stage's output after writing, so it is the
// one stage run out of place (ping-pong between two RGB buffers); every
// other stage runs in place.
#include <algorithm>
#include <cstring>
#include <functional>

#include "lre_internal.h"

using lre::Context;

namespace {

Context* C(lre_ctx* p) { return reinterpret_cast<Context*>(p); }

size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

// Demosaic routing (Accelerator::demosaic_compute, core/accelerator.cpp:90-129).
enum class Demosaic { Amaze, Linear, Dcb, Aahd, Xtrans1, Xtrans3 };

Demosaic route(const lre_develop_params& p) {
  if (p.filters == LRE_FILTERS_XTRANS)
    return (p.demosaic_algorithm == 0 || p.xtrans_passes == 1) ? Demosaic::Xtrans1 : Demosaic::Xtrans3;
  switch (p.demosaic_algorithm) {
    case 0: return Demosaic::Linear;
    case 4: return Demosaic::Dcb;
    case 12: return Demosaic::Aahd;
    default: return Demosaic::Amaze;
  }
}

size_t stage_ws(const lre_develop_params& p, size_t w, size_t h) {
  size_t m = 0;
  switch (route(p)) {
    case Demosaic::Xtrans1: m = std::max(m, lre::ws_bytes_xtrans(w, h, 1)); break;
    case Demosaic::Xtrans3: m = std::max(m, lre::ws_bytes_xtrans(w, h, 3, p.xtrans)); break;
    case Demosaic::Dcb: m = std::max(m, lre::ws_bytes_dcb(w, h)); break;
    case Demosaic::Aahd: m = std::max(m, lre::ws_bytes_aahd(w, h)); break;
    case Demosaic::Linear: break;
    case Demosaic::Amaze: m = std::max(m, lre::ws_bytes_amaze(w, h)); break;
  }
  if (p.highlight_recovery) m = std::max(m, lre::ws_bytes_highlights(w, h));
  if (p.lateral_ca_correction)
    m = std::max(m, lre::ws_bytes_lateral(w, h, p.lateral_ca_cell_size, p.lateral_ca_pyramid_levels, true));
  if (p.defringe) m = std::max(m, lre::ws_bytes_defringe(w, h, p.defringe_radius));
  if (p.axial_ca_correction) m = std::max(m, lre::ws_bytes_axial(w, h, p.axial_ca_radius));
  if (p.tone_mapping == 2) m = std::max(m, lre::ws_bytes_detail_tonemap(w, h));
  return m + 4096;
}

lre_status validate(Context* c, const lre_develop_params* p, size_t w, size_t h) {
  if (!p) return lre::fail(c, LRE_ERR_INVALID_ARGUMENT, "develop: null params");
  if (w < 32 || h < 32) return lre::fail(c, LRE_ERR_INVALID_ARGUMENT, "develop: image smaller than 32x32");
  if (w > (1u << 20) || h > (1u << 20) || w * h > (size_t(1) << 31))
    return lre::fail(c, LRE_ERR_INVALID_ARGUMENT, "develop: image too large");
  if (p->filters != LRE_FILTERS_XTRANS && p->filters < 1000)
    return lre::fail(c, LRE_ERR_INVALID_ARGUMENT, "develop: filters is neither a Bayer word nor X-Trans");
  if (p->filters != LRE_FILTERS_XTRANS && (p->demosaic_algorithm == 4 || p->demosaic_algorithm == 12) &&
      !lre::bayer_2x2_layout(p->filters))
    return lre::fail(c, LRE_ERR_INVALID_ARGUMENT, "develop: DCB and AAHD need a 2x2 Bayer layout");
  if (p->output_bits != 32 && p->output_bits != 16)
    return lre::fail(c, LRE_ERR_INVALID_ARGUMENT, "develop: output_bits must be 32 or 16");
  if (p->axial_ca_correction && p->axial_ca_radius > 16)
    return lre::fail(c, LRE_ERR_INVALID_ARGUMENT, "develop: axial_ca_radius > 16 is not supported");
  return LRE_OK;
}

// Runs the stage chain on device buffers; returns the buffer holding the
// final RGB in *result.
lre_status ensure_copy_stream(Context* c) {
  if (!c->copy_stream) LRE_CUDA_TRY(c, cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking));
  for (cudaEvent_t& e : c->band_ev)
    if (!e) LRE_CUDA_TRY(c, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  for (cudaEvent_t& e : c->tail_ev)
    if (!e) LRE_CUDA_TRY(c, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  return LRE_OK;
}

// Called for each row band [r0, r1) of the final RGB (buffer `rgb`) as soon
// as its last stage is enqueued, when the chain can finish in row bands.
using RowsReady = std::function<lre_status(const float* rgb, size_t r0, size_t r1)>;

// The chain can hand out its result in row bands when it ends with the axial
// guided filter followed only by pointwise work (the 51 MP workload's order:
// ... -> defringe -> axial -> ACES tone map).
bool banded_tail(const lre_develop_params& p) {
  return p.stage_order == 1 && p.axial_ca_correction && p.tone_mapping != 2;
}

// h_mosaic (nullable): the mosaic is still in host memory and d_mosaic is
// its destination; the AMaZE route overlaps the upload with the demosaic,
// every other route uploads it first.
// tail (nullable): when banded_tail(p), the axial filter and the tone map run
// in row bands and each finished band is passed to *tail.
lre_status run_chain(Context* c, const float* d_mosaic, float* rgb_a, float* rgb_b, size_t w, size_t h,
                     const lre_develop_params& p, float** result, const float* h_mosaic = nullptr,
                     const RowsReady* tail = nullptr) {
  float* cur = rgb_a;
  float* other = rgb_b;
  const size_t mark = c->ws.used();
  // The in-order sweeps of DCB/AAHD and highlight recovery report a time-out
  // through a device flag (d_scalars[63]); the host-buffer entry point reads
  // it after its final synchronisation.
  int* d_err = reinterpret_cast<int*>(c->d_scalars + 63);
  if (h_mosaic && route(p) != Demosaic::Amaze)
    LRE_TRY(lre::copy_h2d(c, const_cast<float*>(d_mosaic), h_mosaic, w * h * sizeof(float), c->stream));
  // cur_max_g: a device scalar holding max(0, max G) of `cur`, when the stage
  // that wrote `cur` reduced it on the way (nullptr otherwise).  Defringe and
  // the axial filter each need that maximum of their input; with the
  // 51 MP order (demosaic -> defringe -> axial) the producer supplies it and
  // saves a full read of the image per consumer.
  float* cur_max_g = nullptr;
  const bool max_after_demosaic =
      p.stage_order == 1 && !p.highlight_recovery && (p.defringe || p.axial_ca_correction);
  switch (route(p)) {
    case Demosaic::Xtrans1:
    case Demosaic::Xtrans3:
      LRE_TRY(lre::launch_xtrans(c, d_mosaic, 1, cur, w, h, p.xtrans, p.maximum_value,
                                 route(p) == Demosaic::Xtrans1 ? 1 : 3));
      break;
    case Demosaic::Linear:
      LRE_TRY(lre::launch_bayer_linear(c, d_mosaic, 1, cur, w, h, p.filters, p.maximum_value));
      break;
    case Demosaic::Dcb:
      LRE_CUDA_TRY(c, cudaMemsetAsync(d_err, 0, sizeof(int), c->stream));
      LRE_TRY(lre::launch_dcb(c, d_mosaic, 1, cur, w, h, p.filters, p.maximum_value, 1, true, d_err));
      break;
    case Demosaic::Aahd:
      LRE_CUDA_TRY(c, cudaMemsetAsync(d_err, 0, sizeof(int), c->stream));
      LRE_TRY(lre::launch_aahd(c, d_mosaic, 1, cur, w, h, p.filters, p.maximum_value, d_err));
      break;
    case Demosaic::Amaze:
      if (h_mosaic) {
        LRE_TRY(ensure_copy_stream(c));
        // the copy stream must not start before earlier work on the mosaic buffer
        LRE_CUDA_TRY(c, cudaEventRecord(c->band_ev[7], c->stream));
        LRE_CUDA_TRY(c, cudaStreamWaitEvent(c->copy_stream, c->band_ev[7], 0));
        LRE_TRY(lre::launch_amaze_from_host(c, h_mosaic, const_cast<float*>(d_mosaic), cur, w, h, p.filters, p.cam_mul,
                                            p.maximum_value, c->copy_stream, c->band_ev, 6,
                                            max_after_demosaic ? c->d_scalars + 2 : nullptr));
      } else {
        LRE_TRY(lre::launch_amaze(c, d_mosaic, 1, cur, w, h, p.filters, p.cam_mul, p.maximum_value,
                                  max_after_demosaic ? c->d_scalars + 2 : nullptr));
      }
      if (max_after_demosaic) cur_max_g = c->d_scalars + 2;
      break;
  }
  c->ws.rewind(mark);
  if (p.highlight_recovery) {
    cur_max_g = nullptr;
    if (route(p) != Demosaic::Dcb && route(p) != Demosaic::Aahd)
      LRE_CUDA_TRY(c, cudaMemsetAsync(d_err, 0, sizeof(int), c->stream));
    LRE_TRY(lre::launch_recover_highlights(c, cur, cur, w, h, p.highlight_threshold, nullptr, nullptr, nullptr, d_err));
  }
  c->ws.rewind(mark);
  auto tone = [&]() -> lre_status {
    if (p.tone_mapping) cur_max_g = nullptr;
    if (p.tone_mapping == 1) LRE_TRY(lre::launch_tone_mapping(c, cur, cur, w * h, p.tone_after_scale));
    if (p.tone_mapping == 2) {
      LRE_TRY(lre::launch_detail_tonemap(c, cur, cur, w, h));
      c->ws.rewind(mark);
    }
    return LRE_OK;
  };
  auto lateral = [&]() -> lre_status {
    if (!p.lateral_ca_correction) return LRE_OK;
    cur_max_g = nullptr;
    LRE_TRY(lre::launch_lateral_ca(c, cur, cur, w, h, p.lateral_ca_cell_size, p.lateral_ca_max_iterations,
                                   p.lateral_ca_max_shift, p.lateral_ca_min_confidence, p.lateral_ca_pyramid_levels));
    c->ws.rewind(mark);
    return LRE_OK;
  };
  const bool in_bands = tail && banded_tail(p);
  // In the 51 MP order an ACES tone map right after the axial filter runs
  // inside the filter's last pass (same bits, one pass over the image less).
  const bool tone_in_axial = p.stage_order == 1 && p.axial_ca_correction && p.tone_mapping == 1;
  const float tone_scale = tone_in_axial ? p.tone_after_scale : -1.f;
  auto axial = [&]() -> lre_status {
    if (!p.axial_ca_correction) return LRE_OK;
    float* dmax = cur_max_g;
    if (!dmax) {
      dmax = c->d_scalars + 1;
      LRE_TRY(lre::launch_channel_max(c, cur, w * h, 1, dmax, true));
    }
    if (in_bands) {
      float* dst = other;
      LRE_TRY(lre::launch_axial_ca_banded(
          c, cur, dst, w, h, p.axial_ca_radius, p.axial_ca_epsilon, p.axial_ca_strength, dmax, 8,
          [&](size_t r0, size_t r1) -> lre_status { return (*tail)(dst, r0, r1); }, tone_scale));
    } else {
      LRE_TRY(lre::launch_axial_ca(c, cur, other, w, h, p.axial_ca_radius, p.axial_ca_epsilon, p.axial_ca_strength,
                                   dmax, tone_scale));
    }
    std::swap(cur, other);
    cur_max_g = nullptr;
    c->ws.rewind(mark);
    return LRE_OK;
  };
  auto defringe = [&]() -> lre_status {
    if (!p.defringe) return LRE_OK;
    // the axial filter follows directly in the 51 MP order
    float* out_max = (p.stage_order == 1 && p.axial_ca_correction) ? c->d_scalars + 3 : nullptr;
    LRE_TRY(lre::launch_defringe(c, cur, cur, w, h, p.defringe_radius, p.defringe_edge_threshold,
                                 p.defringe_chroma_threshold, p.defringe_strength, p.defringe_green != 0,
                                 p.defringe_green_strength, cur_max_g, out_max));
    cur_max_g = out_max;
    c->ws.rewind(mark);
    return LRE_OK;
  };
  if (p.stage_order == 1) {
    LRE_TRY(defringe());
    LRE_TRY(axial());
    if (!tone_in_axial) LRE_TRY(tone());
  } else {
    LRE_TRY(tone());
    LRE_TRY(lateral());
    LRE_TRY(axial());
    LRE_TRY(defringe());
  }
  *result = cur;
  return LRE_OK;
}

}  // namespace

namespace lre {

lre_status develop_validate(Context* c, const lre_develop_params* p, size_t w, size_t h) { return validate(c, p, w, h); }

size_t develop_ws_bytes(const lre_develop_params& p, size_t w, size_t h) {
  const size_t rgb_bytes = align256(w * h * 12);
  return (p.output_bits == 32 ? 1 : 2) * rgb_bytes + stage_ws(p, w, h) + 4096;
}

// The whole chain on device buffers, enqueued on c->stream (validated
// parameters).  Float output doubles as the first RGB buffer.
lre_status develop_device(Context* c, const float* mosaic, void* out, size_t w, size_t h,
                          const lre_develop_params& p) {
  const size_t rgb_bytes = align256(w * h * 12);
  const bool float_out = p.output_bits == 32;
  c->ws.reset();
  LRE_CUDA_TRY(c, c->ws.reserve(develop_ws_bytes(p, w, h), c->stream));
  float* rgb_a = float_out ? reinterpret_cast<float*>(out) : reinterpret_cast<float*>(c->ws.take(rgb_bytes));
  float* rgb_b = reinterpret_cast<float*>(c->ws.take(rgb_bytes));
  if (!rgb_a || !rgb_b) return fail(c, LRE_ERR_OUT_OF_MEMORY, "develop: workspace too small");
  float* res = nullptr;
  LRE_TRY(run_chain(c, mosaic, rgb_a, rgb_b, w, h, p, &res));
  if (float_out) {
    if (res != out) LRE_CUDA_TRY(c, cudaMemcpyAsync(out, res, w * h * 12, cudaMemcpyDeviceToDevice, c->stream));
  } else {
    LRE_TRY(launch_quantize_u16(c, res, reinterpret_cast<uint16_t*>(out), w * h * 3));
  }
  return LRE_OK;
}

}  // namespace lre

extern "C" {

void lre_develop_params_default(lre_develop_params* p) {
  if (!p) return;
  memset(p, 0, sizeof(*p));
  // ProcessingParams defaults (core/accelerator.h:83-177)
  p->filters = 0x94949494u;  // RGGB
  p->cam_mul[0] = p->cam_mul[1] = p->cam_mul[2] = p->cam_mul[3] = 1.f;
  p->maximum_value = 1.f;
  p->xtrans_passes = 3;
  p->lateral_ca_correction = 0;
  p->lateral_ca_cell_size = 96;
  p->lateral_ca_max_iterations = 3;
  p->lateral_ca_max_shift = 6.0f;
  p->lateral_ca_min_confidence = 0.02f;
  p->lateral_ca_pyramid_levels = 3;
  p->axial_ca_correction = 0;
  p->axial_ca_radius = 6;
  p->axial_ca_epsilon = 1e-4f;
  p->axial_ca_strength = 0.3f;
  p->defringe = 0;
  p->defringe_radius = 10.0f;
  p->defringe_edge_threshold = 0.1f;
  p->defringe_chroma_threshold = 0.15f;
  p->defringe_strength = 10.0f;
  p->defringe_green = 0;
  p->defringe_green_strength = 0.3f;
  p->tone_mapping = 0;
  p->tone_after_scale = 1.0f;
  p->output_bits = 32;
  p->stage_order = 0;
  p->demosaic_algorithm = 1;
  p->highlight_recovery = 0;
  p->highlight_threshold = 1.0f;
}

lre_status lre_dev_develop(lre_ctx* ctx, const float* mosaic, void* out, size_t w, size_t h,
                           const lre_develop_params* params) {
  Context* c = C(ctx);
  if (!c) return LRE_ERR_INVALID_ARGUMENT;
  if (!mosaic || !out) return lre::fail(c, LRE_ERR_INVALID_ARGUMENT, "develop: null buffer");
  LRE_TRY(validate(c, params, w, h));
  cudaSetDevice(c->device);
  LRE_TRY(lre::check_injection(c));
  return lre::develop_device(c, mosaic, out, w, h, *params);
}

lre_status lre_develop(lre_ctx* ctx, const float* mosaic, void* out, size_t w, size_t h,
                       const lre_develop_params* params) {
  Context* c = C(ctx);
  if (!c) return LRE_ERR_INVALID_ARGUMENT;
  if (!mosaic || !out) return lre::fail(c, LRE_ERR_INVALID_ARGUMENT, "develop: null buffer");
  LRE_TRY(validate(c, params, w, h));
  std::lock_guard<std::mutex> lk(c->mu);
  cudaSetDevice(c->device);
  LRE_TRY(lre::check_injection(c));
  const lre_develop_params& p = *params;
  const size_t in_bytes = w * h * 4;
  const size_t out_bytes = w * h * 3 * (p.output_bits == 16 ? 2 : 4);
  LRE_TRY(lre::ensure_buffer(c, &c->d_in, &c->d_in_cap, in_bytes));
  LRE_TRY(lre::ensure_buffer(c, &c->d_out, &c->d_out_cap, out_bytes));
  const size_t rgb_bytes = align256(w * h * 12);
  c->ws.reset();
  LRE_CUDA_TRY(c, c->ws.reserve(2 * rgb_bytes + stage_ws(p, w, h), c->stream));
  float* rgb_a = reinterpret_cast<float*>(c->ws.take(rgb_bytes));
  float* rgb_b = reinterpret_cast<float*>(c->ws.take(rgb_bytes));
  float* res = nullptr;
  const size_t px_bytes = 3 * (p.output_bits == 16 ? 2 : 4);
  if (banded_tail(p)) {
    // The download overlaps the rest of the chain: each row band of the
    // result (quantised when 16-bit) is downloaded on the copy stream once
    // the main stream has finished it.  All kernels are enqueued before the
    // first copy, so a pageable destination (whose copies return only when
    // done) does not hold back the kernel queue.
    LRE_TRY(ensure_copy_stream(c));
    struct Band {
      const void* src;
      size_t r0, r1;
    };
    Band bands[8];
    int nb = 0;
    const RowsReady tail = [&](const float* rgb, size_t r0, size_t r1) -> lre_status {
      if (nb >= 8) return lre::fail(c, LRE_ERR_INVALID_ARGUMENT, "develop: internal: more than 8 row bands");
      const void* src = rgb + r0 * w * 3;
      if (p.output_bits == 16) {
        uint16_t* q = reinterpret_cast<uint16_t*>(c->d_out) + r0 * w * 3;
        LRE_TRY(lre::launch_quantize_u16(c, rgb + r0 * w * 3, q, (r1 - r0) * w * 3));
        src = q;
      }
      LRE_CUDA_TRY(c, cudaEventRecord(c->tail_ev[nb], c->stream));
      bands[nb++] = {src, r0, r1};
      return LRE_OK;
    };
    LRE_TRY(run_chain(c, reinterpret_cast<const float*>(c->d_in), rgb_a, rgb_b, w, h, p, &res, mosaic, &tail));
    for (int b = 0; b < nb; b++) {
      LRE_CUDA_TRY(c, cudaStreamWaitEvent(c->copy_stream, c->tail_ev[b], 0));
      LRE_TRY(lre::copy_d2h(c, static_cast<char*>(out) + bands[b].r0 * w * px_bytes, bands[b].src,
                            (bands[b].r1 - bands[b].r0) * w * px_bytes, c->copy_stream));
    }
    LRE_CUDA_TRY(c, cudaStreamSynchronize(c->copy_stream));
  } else {
    LRE_TRY(run_chain(c, reinterpret_cast<const float*>(c->d_in), rgb_a, rgb_b, w, h, p, &res, mosaic));
    if (p.output_bits == 16) {
      LRE_TRY(lre::launch_quantize_u16(c, res, reinterpret_cast<uint16_t*>(c->d_out), w * h * 3));
      LRE_TRY(lre::copy_d2h(c, out, c->d_out, out_bytes, c->stream));
    } else {
      LRE_TRY(lre::copy_d2h(c, out, res, out_bytes, c->stream));
    }
  }
  LRE_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  const Demosaic d = route(p);
  if (d == Demosaic::Dcb || d == Demosaic::Aahd || p.highlight_recovery) {
    int err = 0;
    LRE_CUDA_TRY(c, cudaMemcpy(&err, c->d_scalars + 63, sizeof(int), cudaMemcpyDeviceToHost));
    if (err) return lre::fail(c, LRE_ERR_TIMEOUT, "develop: a demosaic sweep band timed out");
  }
  return LRE_OK;
}

}  // extern "C"
