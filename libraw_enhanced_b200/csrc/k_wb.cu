// k_wb.cu -- LibRaw's white-balance multiplier derivation (scale_colors).
//
// Semantics: core/libraw_wrapper.cpp:602-845 (LibRawWrapper::Impl::
// scale_colors), the part that decides the multipliers the pipeline hands to
// apply_white_balance (core/libraw_wrapper.cpp:1545-1553):
//   * params.user_mul replaces color.pre_mul (:612-618);
//   * grey-world auto-WB (:623-664): per-native-colour means of the
//     black-subtracted uint16[4] image, G2 folded into G, pre_mul =
//     (G/R, 1, G/B, 1).  The reference sums 16-bit samples in double, which
//     is exact below 2^53, so the device forms exact 64-bit integer sums in
//     any order and the host converts them once;
//   * camera WB from color.white (:740-772), the Nikon sRAW daylight case
//     (:774-784), the pre_mul[1] / pre_mul[3] defaults (:786-792);
//   * maximum -= black on the unsigned LibRaw field (:800);
//   * normalisation by the smallest multiplier unless auto-WB ran
//     (:802-826).
// The host arithmetic keeps the reference's types (float fields, double
// intermediates, unsigned maximum), so the multipliers are bit-exact.
#include <cstring>
#include <limits>

#include "common.cuh"
#include "lre_internal.h"

namespace lre {

namespace {

struct Pat36 {
  char p[36];
};

// One CTA reduces its share into shared 64-bit counters, then adds them to
// the global sums with one atomic per counter.
__global__ void k_channel_sums(const ushort4* __restrict__ raw4, int w, int h, uint32_t filters, Pat36 xt,
                               unsigned long long* __restrict__ out /* [8]: sums[4], counts[4] */) {
  __shared__ unsigned long long s[8];
  if (threadIdx.x < 8) s[threadIdx.x] = 0ull;
  __syncthreads();
  unsigned long long sum[4] = {0ull, 0ull, 0ull, 0ull};
  unsigned cnt[4] = {0u, 0u, 0u, 0u};
  const size_t n = (size_t)w * h;
  const bool is_xt = filters == LRE_FILTERS_XTRANS;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const unsigned row = (unsigned)(i / w), col = (unsigned)(i % w);
    const unsigned c = is_xt ? (unsigned)xt.p[((row + 6) % 6) * 6 + (col + 6) % 6] : fcol_native(row, col, filters);
    const ushort4 v = raw4[i];
    const unsigned val = c == 0 ? v.x : c == 1 ? v.y : c == 2 ? v.z : v.w;
#pragma unroll
    for (int k = 0; k < 4; k++)
      if ((unsigned)k == c) {
        sum[k] += val;
        cnt[k] += 1u;
      }
  }
#pragma unroll
  for (int k = 0; k < 4; k++) {
    unsigned long long a = sum[k], b = cnt[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      a += __shfl_down_sync(0xffffffffu, a, o);
      b += __shfl_down_sync(0xffffffffu, b, o);
    }
    if ((threadIdx.x & 31) == 0) {
      atomicAdd(&s[k], a);
      atomicAdd(&s[4 + k], b);
    }
  }
  __syncthreads();
  if (threadIdx.x < 8 && s[threadIdx.x]) atomicAdd(&out[threadIdx.x], s[threadIdx.x]);
}

// fcol_bayer_native (core/metal/shader_common.h:63-65) on the host.
unsigned host_fcol_native(unsigned row, unsigned col, uint32_t filters) {
  return filters >> ((((row << 1) & 14) | (col & 1)) << 1) & 3;
}

lre_status dev_sums(Context* c, const uint16_t* d_raw4, size_t w, size_t h, uint32_t filters, const char* xtrans,
                    uint64_t sums[4], uint64_t counts[4]) {
  unsigned long long* d = reinterpret_cast<unsigned long long*>(c->d_scalars + 16);  // 8 x u64, 8-byte aligned
  LRE_CUDA_TRY(c, cudaMemsetAsync(d, 0, 8 * sizeof(unsigned long long), c->stream));
  Pat36 xt{};
  if (xtrans) memcpy(xt.p, xtrans, 36);
  k_channel_sums<<<grid_for(w * h, 256, c->sm_count * 4), 256, 0, c->stream>>>(
      reinterpret_cast<const ushort4*>(d_raw4), (int)w, (int)h, filters, xt, d);
  count_launch(c);
  LRE_TRY(check_launch(c, "channel_sums"));
  unsigned long long host[8];
  LRE_CUDA_TRY(c, cudaMemcpyAsync(host, d, sizeof(host), cudaMemcpyDeviceToHost, c->stream));
  LRE_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  for (int k = 0; k < 4; k++) {
    sums[k] = host[k];
    counts[k] = host[4 + k];
  }
  return LRE_OK;
}

}  // namespace

bool wb_needs_sums(const lre_wb_inputs& in) {
  // should_use_auto_wb (:623-632); cam_mul[0] < -0.5 compares in double
  return in.use_auto_wb ||
         (in.use_camera_wb &&
          ((double)in.cam_mul[0] < -0.5 || (in.cam_mul[0] <= 0.00001f && !in.camerawb_fallback_to_daylight)));
}

lre_status wb_multipliers(const lre_wb_inputs& in, uint32_t filters, unsigned maximum, unsigned black,
                          const uint64_t* sums, const uint64_t* counts, lre_wb_result* out) {
  lre_wb_result r;
  memset(&r, 0, sizeof(r));
  float pre_mul[4];
  memcpy(pre_mul, in.pre_mul, sizeof(pre_mul));
  if (in.user_mul[0]) memcpy(pre_mul, in.user_mul, sizeof(pre_mul));

  const bool auto_wb = wb_needs_sums(in);
  if (auto_wb) {
    if (!sums || !counts) return LRE_ERR_INVALID_ARGUMENT;
    // p = 1: pow(x, 1.0) and pow(mean, 1.0) are exact identities
    double norm[4], count[4];
    for (int c = 0; c < 4; c++) {
      norm[c] = (double)sums[c];
      count[c] = (double)counts[c];
    }
    norm[1] += norm[3];
    count[1] += count[3];
    for (int c = 0; c < 3; c++) norm[c] = norm[c] / count[c];
    pre_mul[0] = (float)(norm[1] / norm[0]);
    pre_mul[1] = 1.0f;
    pre_mul[2] = (float)(norm[1] / norm[2]);
    pre_mul[3] = 1.0f;
  }

  if (in.use_camera_wb && in.cam_mul[0] > 0.00001f) {
    unsigned sum[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (unsigned row = 0; row < 8; row++)
      for (unsigned col = 0; col < 8; col++) {
        const unsigned c = host_fcol_native(row, col, filters);
        // ushort - unsigned wraps as unsigned, then converts to int
        const int val = (int)((unsigned)in.white[row][col] - in.cblack[c]);
        if (val > 0) sum[c] += (unsigned)val;
        sum[c + 4]++;
      }
    if (in.as_shot_wb_applied) {
      pre_mul[0] = pre_mul[1] = pre_mul[2] = pre_mul[3] = 1.0f;
    } else if (sum[0] && sum[1] && sum[2] && sum[3]) {
      for (int c = 0; c < 4; c++) pre_mul[c] = (float)sum[c + 4] / (float)sum[c];
    } else if (in.cam_mul[0] > 0.00001f && in.cam_mul[2] > 0.00001f) {
      memcpy(pre_mul, in.cam_mul, sizeof(pre_mul));
    } else {
      r.bad_camera_wb = 1;
    }
  }

  if (in.as_shot_wb_applied && !in.use_camera_wb && !in.use_auto_wb && in.cam_mul[0] > 0.00001f &&
      in.cam_mul[1] > 0.00001f && in.cam_mul[2] > 0.00001f)
    for (int c = 0; c < 3; c++) pre_mul[c] /= in.cam_mul[c];

  if (pre_mul[1] == 0) pre_mul[1] = 1;
  if (pre_mul[3] == 0) pre_mul[3] = in.colors < 4 ? pre_mul[1] : 1;

  maximum -= black;

  if (!auto_wb) {
    double dmin = std::numeric_limits<double>::max();
    for (int c = 0; c < 4; c++)
      if (dmin > pre_mul[c]) dmin = pre_mul[c];
    if (dmin > 0.00001 && maximum > 0) {
      for (int c = 0; c < 4; c++) r.scale_mul[c] = (float)(pre_mul[c] / dmin);
    } else {
      for (int c = 0; c < 4; c++) r.scale_mul[c] = 1.0f;
    }
  } else {
    for (int c = 0; c < 4; c++) r.scale_mul[c] = pre_mul[c];
  }
  // the pipeline's effective_wb when params.no_auto_scale (:1545-1553)
  if (in.no_auto_scale)
    for (int c = 0; c < 4; c++) r.scale_mul[c] = 1.0f;
  memcpy(r.pre_mul, pre_mul, sizeof(pre_mul));
  r.maximum = maximum;
  r.auto_wb = auto_wb ? 1 : 0;
  *out = r;
  return LRE_OK;
}

lre_status derive_wb_device(Context* c, const uint16_t* d_raw4, size_t w, size_t h, uint32_t filters,
                            const char* xtrans, unsigned maximum, unsigned black, const lre_wb_inputs& in,
                            lre_wb_result* out) {
  uint64_t sums[4] = {0, 0, 0, 0}, counts[4] = {0, 0, 0, 0};
  const bool need = !in.no_auto_scale && wb_needs_sums(in);
  if (need) LRE_TRY(dev_sums(c, d_raw4, w, h, filters, xtrans, sums, counts));
  const lre_status st = wb_multipliers(in, filters, maximum, black, need ? sums : nullptr, need ? counts : nullptr, out);
  if (st != LRE_OK) return fail(c, st, "scale_colors: channel sums missing");
  return LRE_OK;
}

}  // namespace lre

using lre::Context;

extern "C" {

int lre_wb_needs_channel_sums(const lre_wb_inputs* in) { return in && lre::wb_needs_sums(*in) ? 1 : 0; }

lre_status lre_wb_multipliers(const lre_wb_inputs* in, uint32_t filters, unsigned maximum, unsigned black,
                              const uint64_t channel_sums[4], const uint64_t channel_counts[4], lre_wb_result* out) {
  if (!in || !out) return LRE_ERR_INVALID_ARGUMENT;
  return lre::wb_multipliers(*in, filters, maximum, black, channel_sums, channel_counts, out);
}

lre_status lre_dev_channel_sums(lre_ctx* ctx, const uint16_t* raw4, size_t width, size_t height, uint32_t filters,
                                const char xtrans[36], uint64_t sums[4], uint64_t counts[4]) {
  Context* c = reinterpret_cast<Context*>(ctx);
  if (!c) return LRE_ERR_INVALID_ARGUMENT;
  if (!raw4 || !sums || !counts || width == 0 || height == 0)
    return lre::fail(c, LRE_ERR_INVALID_ARGUMENT, "channel_sums: bad argument");
  if (filters == LRE_FILTERS_XTRANS && !xtrans)
    return lre::fail(c, LRE_ERR_INVALID_ARGUMENT, "channel_sums: X-Trans needs its pattern");
  cudaSetDevice(c->device);
  LRE_TRY(lre::check_injection(c));
  return lre::dev_sums(c, raw4, width, height, filters, xtrans, sums, counts);
}

lre_status lre_channel_sums(lre_ctx* ctx, const uint16_t* raw4, size_t width, size_t height, uint32_t filters,
                            const char xtrans[36], uint64_t sums[4], uint64_t counts[4]) {
  Context* c = reinterpret_cast<Context*>(ctx);
  if (!c) return LRE_ERR_INVALID_ARGUMENT;
  if (!raw4 || !sums || !counts || width == 0 || height == 0)
    return lre::fail(c, LRE_ERR_INVALID_ARGUMENT, "channel_sums: bad argument");
  if (filters == LRE_FILTERS_XTRANS && !xtrans)
    return lre::fail(c, LRE_ERR_INVALID_ARGUMENT, "channel_sums: X-Trans needs its pattern");
  std::lock_guard<std::mutex> lk(c->mu);
  cudaSetDevice(c->device);
  LRE_TRY(lre::check_injection(c));
  const size_t bytes = width * height * 8;
  LRE_TRY(lre::ensure_buffer(c, &c->d_in, &c->d_in_cap, bytes));
  LRE_TRY(lre::copy_h2d(c, c->d_in, raw4, bytes, c->stream));
  return lre::dev_sums(c, reinterpret_cast<const uint16_t*>(c->d_in), width, height, filters, xtrans, sums, counts);
}

}  // extern "C"
