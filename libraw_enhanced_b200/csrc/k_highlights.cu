// k_highlights.cu -- highlight recovery (the develop pipeline's
// recover_highlights, core/libraw_wrapper.cpp:1095-1383, run for
// highlight_mode > 2 at :1677-1683, and the standalone
// LibRawWrapper::recover_highlights_numpy, :3066-3096).
//
// The reference runs five loops over an interleaved float[3] image:
//   1. per pixel: the optional soft highlight mask, the highlight test
//      (R and B >= threshold) and, for unclipped highlights, the float sums
//      of R/G and B/G in pixel order;
//   2. per highlight pixel: max over channels, G from R and B through the
//      mean ratios, R and B pulled toward G, the white test;
//   3. per white pixel off the 1-px frame: the 8-neighbour mean, all
//      computed before any is written;
//   4. per highlight pixel off the 2-px frame, in pixel order, in place: the
//      LoCA green lift, which reads 3x3 and 5x5 neighbourhoods that earlier
//      pixels of the same loop may have rewritten.
//
// Here:
//   * loop 1 is one thread per pixel; its two float sums are sequential in
//     the reference, so the terms are compacted in pixel order (block counts,
//     one scan, an order-preserving scatter) and one warp adds them in that
//     order, bit for bit;
//   * loops 2 and 3 are one thread per pixel on R/G/B planes;
//   * loop 4 is an in-order sweep (sweep.cuh): a pixel reads rewritten
//     pixels up to two rows up and two columns right, so rows walk three
//     columns apart (skew 3) through a 256-column shared-memory ring.
// Arithmetic is the reference's operation for operation (--fmad=false; the
// 5x5 ratio sums in double).
#include <cfloat>

#include "common.cuh"
#include "lre_internal.h"
#include "stencil.cuh"
#include "sweep.cuh"

namespace lre {

namespace {

constexpr int kHlBlock = 256;

struct HlParams {
  float thr;
  float chroma_lo, chroma_inv;
  float inv_wb[3];
  float mask_inv;
};

// Loop 1 per pixel (:1150-1191): mask, highlight flag, candidate flag.
__global__ void k_hl_pass1(const float* __restrict__ in, size_t n, HlParams P, float* __restrict__ mask,
                           uint8_t* __restrict__ flags, int* __restrict__ block_counts) {
  const size_t i = (size_t)blockIdx.x * kHlBlock + threadIdx.x;
  int cand = 0;
  if (i < n) {
    const float p0 = in[i * 3], p1 = in[i * 3 + 1], p2 = in[i * 3 + 2];
    if (mask) {
      float t = (p1 - 0.95f) * P.mask_inv;
      if (t < 0.f) t = 0.f; else if (t > 1.f) t = 1.f;
      const float w_g = t * t * (3.f - 2.f * t);
      const float r_n = p0 * P.inv_wb[0], g_n = p1 * P.inv_wb[1], b_n = p2 * P.inv_wb[2];
      const float mx = smax(r_n, smax(g_n, b_n));
      const float mn = smin(r_n, smin(g_n, b_n));
      const float chroma = (mx > 1e-6f) ? (mx - mn) / mx : 0.f;
      float ct = (chroma - P.chroma_lo) * P.chroma_inv;
      if (ct < 0.f) ct = 0.f; else if (ct > 1.f) ct = 1.f;
      const float neutrality = 1.f - ct * ct * (3.f - 2.f * ct);
      mask[i] = w_g * neutrality;
    }
    uint8_t f = 0;
    if (p0 >= P.thr && p2 >= P.thr) {
      f = 1;
      if (p0 < 0.95f && p1 >= P.thr && p1 < 0.95f && p2 < 0.95f) {
        f = 3;
        cand = 1;
      }
    }
    flags[i] = f;
  }
  const int c = __syncthreads_count(cand);
  if (threadIdx.x == 0) block_counts[blockIdx.x] = c;
}

// Exclusive scan of the per-block candidate counts (one CTA; the total goes
// to block_off[nb]).
__global__ void k_hl_scan(const int* __restrict__ counts, int nb, int* __restrict__ off) {
  __shared__ int warp_sums[32];
  __shared__ int carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int base = 0; base < nb; base += 1024) {
    const int i = base + threadIdx.x;
    const int v = i < nb ? counts[i] : 0;
    int x = v;
    for (int d = 1; d < 32; d <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, x, d);
      if ((threadIdx.x & 31) >= d) x += y;
    }
    if ((threadIdx.x & 31) == 31) warp_sums[threadIdx.x >> 5] = x;
    __syncthreads();
    if (threadIdx.x < 32) {
      int w = warp_sums[threadIdx.x];
      for (int d = 1; d < 32; d <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, w, d);
        if (threadIdx.x >= d) w += y;
      }
      warp_sums[threadIdx.x] = w;
    }
    __syncthreads();
    const int wp = (threadIdx.x >> 5) ? warp_sums[(threadIdx.x >> 5) - 1] : 0;
    if (i < nb) off[i] = carry + wp + x - v;
    __syncthreads();
    if (threadIdx.x == 1023) carry += wp + x;
    __syncthreads();
  }
  if (threadIdx.x == 0) off[nb] = carry;
}

// The candidates' R/G and B/G terms, scattered in pixel order.
__global__ void k_hl_compact(const float* __restrict__ in, size_t n, const uint8_t* __restrict__ flags,
                             const int* __restrict__ block_off, float* __restrict__ t_rg,
                             float* __restrict__ t_bg) {
  __shared__ int warp_base[kHlBlock / 32];
  const size_t i = (size_t)blockIdx.x * kHlBlock + threadIdx.x;
  const bool cand = i < n && flags[i] == 3;
  const unsigned b = __ballot_sync(0xffffffffu, cand);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) warp_base[warp] = __popc(b);
  __syncthreads();
  if (threadIdx.x == 0) {
    int s = 0;
    for (int k = 0; k < kHlBlock / 32; k++) {
      const int c = warp_base[k];
      warp_base[k] = s;
      s += c;
    }
  }
  __syncthreads();
  if (cand) {
    const int pos = block_off[blockIdx.x] + warp_base[warp] + __popc(b & ((1u << lane) - 1));
    const float p0 = in[i * 3], p1 = in[i * 3 + 1], p2 = in[i * 3 + 2];
    t_rg[pos] = p0 / p1;
    t_bg[pos] = p2 / p1;
  }
}

// grf / gbf / count as the reference accumulates them (:1182-1196): float
// sums in pixel order.  Lanes stage 32 terms at a time in shared memory;
// lane 0 adds them in order.  scal[0] = grf, scal[1] = gbf.
__global__ void k_hl_ratio_sums(const float* __restrict__ t_rg, const float* __restrict__ t_bg,
                                const int* __restrict__ total, float* __restrict__ scal) {
  __shared__ float a[32], b[32];
  const int k = *total;
  float grf = 0.f, gbf = 0.f, count = 0.f;
  for (int base = 0; base < k; base += 32) {
    const int m = min(32, k - base);
    if ((int)threadIdx.x < m) {
      a[threadIdx.x] = t_rg[base + threadIdx.x];
      b[threadIdx.x] = t_bg[base + threadIdx.x];
    }
    __syncwarp();
    if (threadIdx.x == 0)
      for (int j = 0; j < m; j++) {
        grf += a[j];
        gbf += b[j];
        count += 1.f;
      }
    __syncwarp();
  }
  if (threadIdx.x == 0) {
    if (count > 0.f) {
      grf /= count;
      gbf /= count;
    } else {
      grf = 1.f;
      gbf = 1.f;
    }
    scal[0] = grf;
    scal[1] = gbf;
  }
}

// Loop 2 (:1207-1251) on every highlight pixel, writing planes (non-highlight
// pixels copy through); flag bit 2 marks white pixels.  scal[2] = max_val.
__global__ void k_hl_pass2(const float* __restrict__ in, size_t n, HlParams P, uint8_t* __restrict__ flags,
                           float* __restrict__ R, float* __restrict__ G, float* __restrict__ B,
                           float* __restrict__ hl, float* __restrict__ scal) {
  const float grf = scal[0], gbf = scal[1];
  float local_max = 0.f;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    float p0 = in[i * 3], p1 = in[i * 3 + 1], p2 = in[i * 3 + 2];
    uint8_t f = flags[i];
    if (f & 1) {
      local_max = smax(local_max, smax(p0, smax(p1, p2)));
      p1 = (p0 / grf + p2 / gbf) * 0.5f;
      const float sp = (p0 < p2) ? p0 : p2;
      const float sl = (smin(sp, 1.f) - P.thr) / (P.thr);
      p0 = p0 * (1.f - sl) + (p1 * grf) * sl;
      p2 = p2 * (1.f - sl) + (p1 * gbf) * sl;
      p1 = (p0 / grf + p2 / gbf) * 0.5f;
      if (p1 >= 0.95f) flags[i] = f | 4;
    }
    R[i] = p0;
    G[i] = p1;
    B[i] = p2;
    hl[i] = (f & 1) ? 1.f : 0.f;
  }
  block_max_atomic(local_max, scal + 2);
}

// Loop 3 (:1259-1296): white pixels off the 1-px frame take the mean of their
// 8 neighbours, all read before any is written (out of place).
__global__ void k_hl_white(const float* __restrict__ R, const float* __restrict__ G, const float* __restrict__ B,
                           const uint8_t* __restrict__ flags, float* __restrict__ R2, float* __restrict__ G2,
                           float* __restrict__ B2, int W, int H) {
  const size_t n = (size_t)W * H;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const int y = (int)(i / W), x = (int)(i % W);
    const float* src[3] = {R, G, B};
    float* dst[3] = {R2, G2, B2};
    const bool white = (flags[i] & 4) && x > 0 && x < W - 1 && y > 0 && y < H - 1;
    for (int c = 0; c < 3; c++) {
      const float* s = src[c];
      dst[c][i] = white ? (s[i - W - 1] + s[i - W] + s[i - W + 1] + s[i - 1] + s[i + 1] + s[i + W - 1] + s[i + W] +
                           s[i + W + 1]) *
                              (1.f / 8.f)
                        : s[i];
    }
  }
}

// Loop 4 (:1301-1377), in pixel order: state R, G, B; input the highlight
// flag.  aux[0] = threshold, aux[1] = max_val.
struct OpLoca {
  static constexpr int NS = 3, NP = 4, HALO = 2, SKEW = 3, PAIR = 1, NCH = 1, LAG = 0, RING = 256;
  template <class T>
  __device__ static void cell(const T& t, int y, int x, const Geo& g) {
    if (t(3, y, x) == 0.f) return;
    const float thr = g.aux[0], max_val = g.aux[1];
    float p0 = t(0, y, x), p1 = t(1, y, x), p2 = t(2, y, x);
    const float l = smax(p0, smax(p1, p2));
    if (l < thr * 0.90f) return;
    float local_max = 0.0f, local_min = FLT_MAX;
#pragma unroll
    for (int dy = -1; dy <= 1; ++dy)
#pragma unroll
      for (int dx = -1; dx <= 1; ++dx) {
        const float nl = smax(t(0, y + dy, x + dx), smax(t(1, y + dy, x + dx), t(2, y + dy, x + dx)));
        local_max = smax(local_max, nl);
        local_min = smin(local_min, nl);
      }
    if ((local_max - local_min) < 0.015f) return;
    const float rb = 0.5f * (p0 + p2);
    if (rb <= p1 * 1.04f) return;
    // Unrolled, so each weight 1.0 / (1 + |dx| + |dy|) is the same correctly
    // rounded double, folded at compile time.
    double ratio_sum = 0.0, ratio_w = 0.0;
#pragma unroll
    for (int dy = -2; dy <= 2; ++dy)
#pragma unroll
      for (int dx = -2; dx <= 2; ++dx) {
        const float n0 = t(0, y + dy, x + dx), n1 = t(1, y + dy, x + dx), n2 = t(2, y + dy, x + dx);
        const float nrb = 0.5f * (n0 + n2);
        const float nl = smax(n0, smax(n1, n2));
        if (nl < thr * 0.75f || nrb <= 1e-6f) continue;
        const float ratio = n1 / nrb;
        if (ratio < 0.70f || ratio > 1.35f) continue;
        const double w = 1.0 / (double)(1 + abs(dx) + abs(dy));
        ratio_sum += ratio * w;
        ratio_w += w;
      }
    const float local_ratio = (float)(ratio_w > 0.0 ? ratio_sum / ratio_w : 1.0);
    const float desired_g = rb * sclamp(local_ratio, 0.95f, 1.08f);
    const float g_missing = desired_g - p1;
    if (g_missing <= 0.0f) return;
    const float sat_w = sclamp((l - thr) / smax(1e-6f, smax(1.0f, max_val) - thr), 0.0f, 1.0f);
    const float edge_w = sclamp((local_max - local_min) / 0.08f, 0.0f, 1.0f);
    const float alpha = sclamp(0.30f + 0.55f * sat_w * edge_w, 0.0f, 0.90f);
    const float g_boost = alpha * smin(g_missing, (rb - p1) * 0.90f);
    p1 += g_boost;
    const float rb_residual = smax(0.0f, 0.5f * (p0 + p2) - p1);
    if (rb_residual > 0.0f) {
      const float trim = smin(rb_residual * alpha * 0.45f, 0.5f * (p0 + p2) * 0.12f);
      p0 = smax(0.0f, p0 - trim);
      p2 = smax(0.0f, p2 - trim);
    }
    p1 = smax(0.0f, p1);
    t(0, y, x) = p0;
    t(1, y, x) = p1;
    t(2, y, x) = p2;
  }
};

// Loop 4's scalars for the sweep: aux[0] = threshold, aux[1] = max_val.
__global__ void k_hl_aux(float* scal, float thr) {
  scal[3] = thr;
  scal[4] = scal[2];
}

__global__ void k_hl_interleave(const float* __restrict__ R, const float* __restrict__ G,
                                const float* __restrict__ B, float* __restrict__ out, size_t n) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    out[i * 3] = R[i];
    out[i * 3 + 1] = G[i];
    out[i * 3 + 2] = B[i];
  }
}

size_t plane(size_t n) { return (n * sizeof(float) + 255) & ~size_t(255); }

}  // namespace

size_t ws_bytes_highlights(size_t w, size_t h) {
  const size_t n = w * h;
  const size_t nb = (n + kHlBlock - 1) / kHlBlock;
  const size_t bands = (h + 31) / 32 + 1;
  return 7 * plane(n) + ((n + 255) & ~size_t(255)) + 2 * ((nb + 1) * sizeof(int) + 256) + 256 +
         (kSyncInts + bands) * sizeof(int) + 1024;
}

lre_status launch_recover_highlights(Context* c, const float* in, float* out, size_t w, size_t h,
                                     float saturation_threshold, float* mask_out, const float* wb_rgb,
                                     float* d_max_val_out, int* d_err) {
  const size_t n = w * h;
  const size_t nb = (n + kHlBlock - 1) / kHlBlock;
  if (nb > (size_t)INT_MAX - 1) return fail(c, LRE_ERR_INVALID_ARGUMENT, "recover_highlights: image too large");
  float* R = reinterpret_cast<float*>(c->ws.take(plane(n)));
  float* G = reinterpret_cast<float*>(c->ws.take(plane(n)));
  float* B = reinterpret_cast<float*>(c->ws.take(plane(n)));
  float* R2 = reinterpret_cast<float*>(c->ws.take(plane(n)));
  float* G2 = reinterpret_cast<float*>(c->ws.take(plane(n)));
  float* B2 = reinterpret_cast<float*>(c->ws.take(plane(n)));
  float* HL = reinterpret_cast<float*>(c->ws.take(plane(n)));
  uint8_t* flags = reinterpret_cast<uint8_t*>(c->ws.take((n + 255) & ~size_t(255)));
  int* counts = reinterpret_cast<int*>(c->ws.take((nb + 1) * sizeof(int) + 256));
  int* offs = reinterpret_cast<int*>(c->ws.take((nb + 1) * sizeof(int) + 256));
  float* scal = reinterpret_cast<float*>(c->ws.take(256));
  const int nb_max = (int)((h + 31) / 32 + 1);
  int* sync = reinterpret_cast<int*>(c->ws.take((kSyncInts + nb_max) * sizeof(int)));
  if (!R || !G || !B || !R2 || !G2 || !B2 || !HL || !flags || !counts || !offs || !scal || !sync)
    return fail(c, LRE_ERR_CUDA, "recover_highlights: workspace not reserved");

  HlParams P{};
  P.thr = saturation_threshold;
  P.mask_inv = 1.f / std::max(1e-6f, 1.00f - 0.95f);
  P.chroma_lo = wb_rgb ? 0.30f : 0.50f;
  const float chroma_hi = wb_rgb ? 0.60f : 0.70f;
  P.chroma_inv = 1.f / std::max(1e-6f, chroma_hi - P.chroma_lo);
  for (int k = 0; k < 3; k++) P.inv_wb[k] = wb_rgb ? 1.f / std::max(1e-6f, wb_rgb[k]) : 1.f;

  cudaStream_t s = c->stream;
  auto ck = [&](const char* what) {
    count_launch(c);
    return check_launch(c, what);
  };
  LRE_CUDA_TRY(c, cudaMemsetAsync(scal, 0, 256, s));
  k_hl_pass1<<<(unsigned)nb, kHlBlock, 0, s>>>(in, n, P, mask_out, flags, counts);
  LRE_TRY(ck("recover_highlights"));
  k_hl_scan<<<1, 1024, 0, s>>>(counts, (int)nb, offs);
  LRE_TRY(ck("recover_highlights"));
  // the compacted terms live in R2/G2, which are free until loop 3
  k_hl_compact<<<(unsigned)nb, kHlBlock, 0, s>>>(in, n, flags, offs, R2, G2);
  LRE_TRY(ck("recover_highlights"));
  k_hl_ratio_sums<<<1, 32, 0, s>>>(R2, G2, offs + nb, scal);
  LRE_TRY(ck("recover_highlights"));
  const unsigned g1 = grid_for(n, 256, c->sm_count * 8);
  k_hl_pass2<<<g1, 256, 0, s>>>(in, n, P, flags, R, G, B, HL, scal);
  LRE_TRY(ck("recover_highlights"));
  k_hl_white<<<g1, 256, 0, s>>>(R, G, B, flags, R2, G2, B2, (int)w, (int)h);
  LRE_TRY(ck("recover_highlights"));
  // loop 4 reads the threshold and max_val from the device
  k_hl_aux<<<1, 1, 0, s>>>(scal, P.thr);
  LRE_TRY(ck("recover_highlights"));
  int* err = d_err ? d_err : sync + 1;
  SweepArgs sa{};
  sa.g = Geo{(int)w, (int)h, 0u, 1.0f, scal + 3};
  sa.err = err;
  sa.plane[0] = R2;
  sa.plane[1] = G2;
  sa.plane[2] = B2;
  sa.plane[3] = HL;
  sa.r_lo = 2;
  sa.r_hi = (int)h - 3;
  sa.c_lo = 2;
  sa.c_hi = (int)w - 3;
  if (!d_err) LRE_CUDA_TRY(c, cudaMemsetAsync(err, 0, sizeof(int), s));
  LRE_TRY(sweep<OpLoca>(c, sa, sync, nb_max, "recover_highlights_loca"));
  k_hl_interleave<<<g1, 256, 0, s>>>(R2, G2, B2, out, n);
  LRE_TRY(ck("recover_highlights"));
  if (d_max_val_out) LRE_CUDA_TRY(c, cudaMemcpyAsync(d_max_val_out, scal + 2, sizeof(float), cudaMemcpyDeviceToDevice, s));
  if (d_err) return LRE_OK;  // the caller reads the flag after its own synchronisation
  int e = 0;
  LRE_CUDA_TRY(c, cudaMemcpyAsync(&e, err, sizeof(int), cudaMemcpyDeviceToHost, s));
  LRE_CUDA_TRY(c, cudaStreamSynchronize(s));
  if (e) return fail(c, LRE_ERR_TIMEOUT, "recover_highlights: a sweep band timed out waiting for the band above");
  return LRE_OK;
}

}  // namespace lre
