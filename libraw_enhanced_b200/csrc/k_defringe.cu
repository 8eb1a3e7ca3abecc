// k_defringe.cu -- edge-gated chroma-ratio defringe.
//
// Semantics: core/cpu_accelerator.cpp:3939-5064 (CPUAccelerator::defringe).
// Every per-pixel expression below is the reference's, in the reference's
// operation order (the library is built with --fmad=false), so results match
// bit for bit except where glibc's logf/expf and the device's differ by an
// ulp (see log_cr / exp_cr).
//
// Stage plan on the device (planes are float W x H in the workspace):
//   R0  max(0, G) reduction                       -> max_guide
//   K1  ratios + Sobel on sqrt(G/max)             -> lrg, lbg, edge_raw, max_edge
//   K2  5 separable Gaussian blurs (one kernel)   -> bg, blrg, blbg, be, ber
//   K3  fringe-support seed                       -> fs
//   K4  blur(fs)                                  -> bfs
//   K5  line-linked support + solo seeds          -> lfs, srs, sbs
//   K6  blur(srs), blur(sbs)                      -> srb, sbb
//   K7  classification + correction (in-place safe)
// Blurs stage a (T+2ks)^2 clamped halo tile in shared memory and run both
// passes there; the line-link kernel stages a +-14 px clamped halo.
#include <algorithm>
#include <cmath>

#include "lre_internal.h"
#include "stencil.cuh"

namespace lre {

GaussTaps make_defringe_taps(float radius) {
  GaussTaps t{};
  const float sigma = std::max(radius / 3.f, 0.5f);
  int ks = static_cast<int>(std::ceil(3.f * sigma));
  if (ks > GAUSS_MAX_KS) ks = GAUSS_MAX_KS;  // caller rejects larger radii first
  t.ks = ks;
  float ksum = 0.f;
  for (int k = -ks; k <= ks; k++) {
    float v = std::exp(-0.5f * (float)(k * k) / (sigma * sigma));
    t.w[k + ks] = v;
    ksum += v;
  }
  for (int k = 0; k < 2 * ks + 1; k++) t.w[k] /= ksum;
  return t;
}

namespace {

struct DfScalars {
  float max_guide_raw;  // max(0, G) over the image
  float max_edge;       // max Sobel magnitude (interior)
};

struct DfPlanes {
  float *lrg, *lbg, *er, *bg, *blrg, *blbg, *be, *ber, *fs, *bfs, *lfs, *srs, *sbs, *srb, *sbb;
};

__device__ __forceinline__ float df_max_guide(const DfScalars* s) { return smax(s->max_guide_raw, 1e-6f); }

// ---------------------------------------------------------------- K1
__device__ __forceinline__ float guide_signal_at(const float* __restrict__ src, int x, int y, int W, float max_guide) {
  float g = src[((size_t)y * W + x) * 3 + 1];
  float gg = smax(g, 0.f);
  return sqrtf(sclamp(gg / max_guide, 0.f, 1.f));
}

// K1 on 32 x 8 output tiles: the guide signal (a square root and a divide
// per pixel) is staged once per pixel in shared memory with a 1-px halo and
// the Sobel taps read it from there, instead of recomputing it for each of
// the 8 neighbours that use it.
constexpr int PT_X = 32, PT_Y = 8;

__global__ void __launch_bounds__(256) k_df_prep_tiled(const float* __restrict__ src, int W, int H, DfScalars* sc,
                                                       float* __restrict__ lrg, float* __restrict__ lbg,
                                                       float* __restrict__ er) {
  __shared__ float s_g[PT_Y + 2][PT_X + 3];
  const float max_guide = df_max_guide(sc);
  const float ratio_eps = smax(max_guide * 1e-4f, 1e-6f);
  const int limit_y = (H > 1) ? H - 1 : 1;
  const int limit_x = (W > 1) ? W - 1 : 1;
  const int tiles_x = (W + PT_X - 1) / PT_X;
  const int n_tiles = tiles_x * ((H + PT_Y - 1) / PT_Y);
  float local_max = 0.f;
  // a CTA walks several tiles, so the max-edge reduction costs one atomic
  // per warp in total rather than one per tile
  for (int t = blockIdx.x; t < n_tiles; t += gridDim.x) {
    const int x0 = (t % tiles_x) * PT_X, y0 = (t / tiles_x) * PT_Y;
    __syncthreads();  // the previous tile's readers are done with s_g
    for (int i = threadIdx.x; i < (PT_Y + 2) * (PT_X + 2); i += blockDim.x) {
      const int r = i / (PT_X + 2), q = i % (PT_X + 2);
      const int gy = min(max(y0 - 1 + r, 0), H - 1);
      const int gx = min(max(x0 - 1 + q, 0), W - 1);
      s_g[r][q] = guide_signal_at(src, gx, gy, W, max_guide);
    }
    __syncthreads();
    const int tx = threadIdx.x % PT_X, ty = threadIdx.x / PT_X;
    const int x = x0 + tx, y = y0 + ty;
    if (x < W && y < H) {
      const size_t i = (size_t)y * W + x;
      const float* p = src + i * 3;
      float r = p[0], g = p[1], b = p[2];
      float gg = smax(g, 0.f);
      lrg[i] = log_cr((smax(r, 0.f) + ratio_eps) / (gg + ratio_eps));
      lbg[i] = log_cr((smax(b, 0.f) + ratio_eps) / (gg + ratio_eps));
      float mag = 0.f;
      if (y >= 1 && y < limit_y && x >= 1 && x < limit_x) {
        const int cy = ty + 1, cx = tx + 1;
        float a00 = s_g[cy - 1][cx - 1];
        float a01 = s_g[cy - 1][cx];
        float a02 = s_g[cy - 1][cx + 1];
        float a10 = s_g[cy][cx - 1];
        float a12 = s_g[cy][cx + 1];
        float a20 = s_g[cy + 1][cx - 1];
        float a21 = s_g[cy + 1][cx];
        float a22 = s_g[cy + 1][cx + 1];
        float gx = -a00 + a02 - 2.f * a10 + 2.f * a12 - a20 + a22;
        float gy = -a00 - 2.f * a01 - a02 + a20 + 2.f * a21 + a22;
        mag = sqrtf(gx * gx + gy * gy);
        local_max = smax(local_max, mag);
      }
      er[i] = mag;
    }
  }
  local_max = warp_max(local_max);
  if ((threadIdx.x & 31) == 0) atomic_max_float(&sc->max_edge, local_max);
}

// ---------------------------------------------------------------- blurs
// Source modes for a blur input plane.
enum BlurSrc : int { BS_PLANE = 0, BS_PLANE_EDGE_NORM = 1, BS_GUIDE_LINEAR = 2 };

struct BlurJob {
  const float* in[5];
  float* out[5];
  int mode[5];
  int np;
};

constexpr int BT = 32;  // output tile edge

// Element p of a small parameter array through constant indices only: a
// run-time index into a kernel parameter would copy the whole parameter block
// to local memory.
template <typename T>
__device__ __forceinline__ T pick5(const T (&a)[5], int p) {
  switch (p) {
    case 0: return a[0];
    case 1: return a[1];
    case 2: return a[2];
    case 3: return a[3];
    default: return a[4];
  }
}

__device__ __forceinline__ float blur_src(const float* in, int mode, const DfScalars* sc, int x, int y, int W) {
  size_t i = (size_t)y * W + x;
  switch (mode) {
    case BS_GUIDE_LINEAR:
      return smax(in[i * 3 + 1], 0.f);
    case BS_PLANE_EDGE_NORM: {
      float f = smax(sc->max_edge, 1e-6f);
      float inv = 1.f / f;
      return in[i] * inv;
    }
    default:
      return in[i];
  }
}

// One CTA = BT x BT outputs of every plane in the job; the clamped input halo
// and the horizontal-pass rows live in shared memory.
__global__ void __launch_bounds__(256) k_df_blur(BlurJob job, GaussTaps taps, int W, int H, const DfScalars* sc) {
  extern __shared__ __align__(16) float sm[];
  const int ks = taps.ks;
  const int E = BT + 2 * ks;  // halo tile edge
  const int x0 = blockIdx.x * BT, y0 = blockIdx.y * BT;
  float* s_in = sm;                       // [np][E][E]
  float* s_h = sm + (size_t)job.np * E * E;  // [np][E][BT]
  for (int p = 0; p < job.np; p++) {
    const float* in = pick5(job.in, p);
    const int mode = pick5(job.mode, p);
    for (int i = threadIdx.x; i < E * E; i += blockDim.x) {
      int gy = min(max(y0 - ks + i / E, 0), H - 1);
      int gx = min(max(x0 - ks + i % E, 0), W - 1);
      s_in[(size_t)p * E * E + i] = blur_src(in, mode, sc, gx, gy, W);
    }
  }
  __syncthreads();
  // horizontal pass over all E halo rows (rows are the clamped image rows)
  for (int p = 0; p < job.np; p++) {
    const float* si = s_in + (size_t)p * E * E;
    float* sh = s_h + (size_t)p * E * BT;
    for (int i = threadIdx.x; i < E * BT; i += blockDim.x) {
      int j = i / BT, k = i % BT;
      const float* row = si + j * E + k;
      float acc = 0.f;
      for (int t = 0; t <= 2 * ks; t++) acc += taps.w[t] * row[t];
      sh[i] = acc;
    }
  }
  __syncthreads();
  // vertical pass
  for (int p = 0; p < job.np; p++) {
    const float* sh = s_h + (size_t)p * E * BT;
    float* out = pick5(job.out, p);
    for (int i = threadIdx.x; i < BT * BT; i += blockDim.x) {
      int j = i / BT, k = i % BT;
      int gy = y0 + j, gx = x0 + k;
      if (gx >= W || gy >= H) continue;
      float acc = 0.f;
      for (int t = 0; t <= 2 * ks; t++) acc += taps.w[t] * sh[(j + t) * BT + k];
      out[(size_t)gy * W + gx] = acc;
    }
  }
}

// Register-tiled blur for a compile-time tap radius KS and output tile edge
// TB (32 or 64): planes are processed one after another through the same
// shared memory (18 KB at TB = 32, so 8 CTAs fit on an SM; 50 KB at TB = 64,
// with 1.7x instead of 2.6x halo reads), each thread produces 8 horizontal
// or 4 vertical outputs from operands held in registers.  Tap order and
// clamping are those of k_df_blur.
// Two floats in one 64-bit register: a blur item carries the outputs of two
// rows (horizontal pass) or two adjacent columns (vertical pass) together.
__device__ __forceinline__ unsigned long long f2_pack(float a, float b) {
  unsigned long long r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
  return r;
}
__device__ __forceinline__ void f2_unpack(unsigned long long v, float& a, float& b) {
  asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(v));
}
// acc + w * x per lane, the product and the sum each rounded to nearest
// (the reference's order, no contraction): the two products as IEEE scalar
// multiplies, the two sums as one packed add.rn.f32x2.  A packed multiply
// feeding a packed add is not safe: ptxas contracts that pair into a fused
// multiply-add (one rounding), which on the 51 MP workload flipped one
// pixel's classification by 1.6e-3.  With scalar products between them
// there is nothing to contract: a B200 probe of the 21-tap chain gave 0
// differences from scalar multiply-then-add over 4.2 M outputs, and the
// blurs need a quarter fewer FP instructions than in all-scalar form.
__device__ __forceinline__ unsigned long long f2_madd(unsigned long long acc, unsigned long long w,
                                                      unsigned long long x) {
  float w0, w1, x0, x1;
  f2_unpack(w, w0, w1);
  f2_unpack(x, x0, x1);
  const unsigned long long p = f2_pack(__fmul_rn(w0, x0), __fmul_rn(w1, x1));
  unsigned long long r;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(acc), "l"(p));
  return r;
}

// The two separable passes of one plane on the tile in shared memory.
template <int KS, int TB>
__device__ __forceinline__ void blur_passes(const float* s_in, float* s_h, const float (&w)[2 * KS + 1], float* out,
                                            int x0, int y0, int W, int H) {
  constexpr int E = TB + 2 * KS;
  constexpr int LD = E + 1;
  // horizontal: item = (halo rows 2jp, 2jp + 1; group of 8 output columns)
  for (int item = threadIdx.x; item < (E / 2) * (TB / 8); item += blockDim.x) {
    const int j = (item / (TB / 8)) * 2, k0 = (item % (TB / 8)) * 8;
    unsigned long long x[8 + 2 * KS];
#pragma unroll
    for (int i = 0; i < 8 + 2 * KS; i++) x[i] = f2_pack(s_in[j * LD + k0 + i], s_in[(j + 1) * LD + k0 + i]);
    unsigned long long acc[8];
#pragma unroll
    for (int o = 0; o < 8; o++) acc[o] = 0ull;  // {+0.f, +0.f}
#pragma unroll
    for (int t = 0; t <= 2 * KS; t++) {
      const unsigned long long wt = f2_pack(w[t], w[t]);
#pragma unroll
      for (int o = 0; o < 8; o++) acc[o] = f2_madd(acc[o], wt, x[o + t]);
    }
#pragma unroll
    for (int o = 0; o < 8; o++) f2_unpack(acc[o], s_h[j * TB + k0 + o], s_h[(j + 1) * TB + k0 + o]);
  }
  __syncthreads();
  // vertical: item = (output columns 2kp, 2kp + 1; group of 4 output rows)
  for (int item = threadIdx.x; item < (TB / 2) * (TB / 4); item += blockDim.x) {
    const int k = (item % (TB / 2)) * 2, j0 = (item / (TB / 2)) * 4;
    unsigned long long x[4 + 2 * KS];
#pragma unroll
    for (int i = 0; i < 4 + 2 * KS; i++) x[i] = *reinterpret_cast<const unsigned long long*>(&s_h[(j0 + i) * TB + k]);
    unsigned long long acc[4];
#pragma unroll
    for (int o = 0; o < 4; o++) acc[o] = 0ull;
#pragma unroll
    for (int t = 0; t <= 2 * KS; t++) {
      const unsigned long long wt = f2_pack(w[t], w[t]);
#pragma unroll
      for (int o = 0; o < 4; o++) acc[o] = f2_madd(acc[o], wt, x[o + t]);
    }
    const int gx = x0 + k;
#pragma unroll
    for (int o = 0; o < 4; o++) {
      float a, b;
      f2_unpack(acc[o], a, b);
      const int gy = y0 + j0 + o;
      if (gy < H) {
        if (gx < W) out[(size_t)gy * W + gx] = a;
        if (gx + 1 < W) out[(size_t)gy * W + gx + 1] = b;
      }
    }
  }
  __syncthreads();
}

template <int KS, int TB>
__device__ __forceinline__ void blur_fast_body(const BlurJob& job, const GaussTaps& taps, int W, int H,
                                               const DfScalars* sc) {
  constexpr int E = TB + 2 * KS;
  constexpr int LD = E + 1;  // odd row stride: conflict-light row reads
  extern __shared__ __align__(16) float sm_fast[];
  float* s_in = sm_fast;           // [E][LD]
  float* s_h = sm_fast + E * LD;   // [E][TB]
  const int x0 = blockIdx.x * TB, y0 = blockIdx.y * TB;
  float w[2 * KS + 1];
#pragma unroll
  for (int t = 0; t <= 2 * KS; t++) w[t] = taps.w[t];
  for (int p = 0; p < job.np; p++) {
    const float* in = pick5(job.in, p);
    const int mode = pick5(job.mode, p);
    float* out = pick5(job.out, p);
    for (int i = threadIdx.x; i < E * E; i += blockDim.x) {
      const int r = i / E, q = i % E;
      const int gy = min(max(y0 - KS + r, 0), H - 1);
      const int gx = min(max(x0 - KS + q, 0), W - 1);
      s_in[r * LD + q] = blur_src(in, mode, sc, gx, gy, W);
    }
    __syncthreads();
    // Both passes run two outputs per item and accumulate every output's
    // taps in the reference's order from 0.f, each product and each sum
    // rounded to nearest (f2_madd).
    blur_passes<KS, TB>(s_in, s_h, w, out, x0, y0, W, H);
  }
}

template <int KS, int TB>
__global__ void __launch_bounds__(256) k_df_blur_fast(BlurJob job, GaussTaps taps, int W, int H, const DfScalars* sc) {
  blur_fast_body<KS, TB>(job, taps, W, H, sc);
}

template <int TB>
lre_status run_blur_fast(Context* c, const BlurJob& job, const GaussTaps& taps, int W, int H, const DfScalars* sc) {
  constexpr int E = TB + 2 * 10;
  const size_t smem = ((size_t)E * (E + 1) + (size_t)E * TB) * sizeof(float);
  LRE_CUDA_TRY(c, cudaFuncSetAttribute(k_df_blur_fast<10, TB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  dim3 grid((W + TB - 1) / TB, (H + TB - 1) / TB);
  k_df_blur_fast<10, TB><<<grid, 256, smem, c->stream>>>(job, taps, W, H, sc);
  count_launch(c);
  return check_launch(c, "defringe blur");
}

// ---------------------------------------------------------------- K3
struct DfConst {
  float edge_thr, chroma_thr, strength, green_scale;
  int green;
};

// Fringe-support seed of pixel i (core/cpu_accelerator.cpp:4158-4205).
__device__ __forceinline__ float support_at(const float* __restrict__ src, size_t i, const DfPlanes& P, const DfConst& k,
                                            float inv_s, bool enable_green) {
  const float rg = P.lrg[i];
  const float bgr = P.lbg[i];
  const float dr = rg - P.blrg[i];
  const float db = bgr - P.blbg[i];
  const float* s = src + i * 3;
  const float r0 = smax(s[0], 0.f);
  const float g0 = smax(s[1], 0.f);
  const float b0 = smax(s[2], 0.f);
  const float blur_guide = P.bg[i];
  const float purple_excess = smin(smax(0.f, dr), smax(0.f, db));
  const float denom_support = smax(blur_guide, 0.05f);
  const float g_over_min_support = smax(0.f, g0 - smin(r0, b0)) / denom_support;
  const float green_dom_support = ssmooth(0.010f, 0.060f, g_over_min_support);
  const float green_excess = smax(smax(0.f, -dr), smax(0.f, -db)) * green_dom_support;
  const bool is_purple = purple_excess >= green_excess;
  const float excess_support = is_purple ? purple_excess : green_excess;
  const float min_dir = is_purple ? smax(0.f, smin(rg, bgr)) : smax(0.f, smin(-rg, -bgr));
  const float max_dir = is_purple ? smax(1e-4f, smax(rg, bgr)) : smax(1e-4f, smax(-rg, -bgr));
  const float balance = min_dir / max_dir;
  const float c_edge = ssmooth(k.edge_thr * 0.35f * inv_s, k.edge_thr * 1.50f * inv_s, P.be[i]) *
                       ssmooth(0.55f * inv_s, 1.35f * inv_s, P.ber[i]);
  const float c_bright = ssmooth(0.24f * inv_s, 0.52f * inv_s, blur_guide);
  const float c_chroma = ssmooth(k.chroma_thr * 0.45f * inv_s, k.chroma_thr * 1.60f * inv_s, excess_support);
  const float red_strength = smax(0.f, r0 - smax(g0, b0)) / smax(r0, 1e-4f);
  const float red_blue_balance = b0 / smax(r0, 1e-4f);
  const float blue_lift = smax(0.f, b0 - g0) / smax(r0 - g0, 1e-4f);
  const float red_purple = smax(ssmooth(0.55f, 0.78f, red_blue_balance), ssmooth(0.16f, 0.34f, blue_lift));
  const float red_purple_hue_signal = ssmooth(0.50f, 0.72f, red_blue_balance) * ssmooth(0.24f, 0.42f, blue_lift);
  const float balanced_hue = ssmooth(0.06f * inv_s, 0.22f * inv_s, min_dir) * ssmooth(0.35f, 0.75f, balance);
  const float red_purple_hue = is_purple ? smin(1.f, red_purple_hue_signal * 1.50f) *
                                               ssmooth(0.035f * inv_s, 0.16f * inv_s, min_dir) *
                                               ssmooth(0.18f, 0.58f, balance)
                                         : 0.f;
  const float c_hue = smax(balanced_hue, red_purple_hue);
  const float natural_guard = 1.f - ssmooth(0.08f, 0.25f, red_strength) * (1.f - red_purple);
  const float green_enable = (enable_green || is_purple) ? 1.f : 0.f;
  return c_edge * c_bright * c_hue * c_chroma * natural_guard * green_enable;
}

// Blur of the five first-stage planes with K3 fused after it: once a tile's
// blurred planes are written, the same CTA computes the fringe-support seed
// of the tile's pixels while those values are still in L2.
template <int KS, int TB>
__global__ void __launch_bounds__(256) k_df_blur_support(BlurJob job, GaussTaps taps, int W, int H,
                                                         const DfScalars* sc, const float* __restrict__ src,
                                                         DfPlanes P, DfConst k) {
  blur_fast_body<KS, TB>(job, taps, W, H, sc);  // ends with a CTA barrier
  const float sensitivity = sclamp(sqrtf(smax(k.strength, 1.0f)), 1.0f, 2.5f);
  const float inv_s = 1.0f / sensitivity;
  const bool enable_green = k.green != 0;
  const int x0 = blockIdx.x * TB, y0 = blockIdx.y * TB;
  for (int i = threadIdx.x; i < TB * TB; i += blockDim.x) {
    const int gx = x0 + i % TB, gy = y0 + i / TB;
    if (gx >= W || gy >= H) continue;
    const size_t gi = (size_t)gy * W + gx;
    P.fs[gi] = support_at(src, gi, P, k, inv_s, enable_green);
  }
}

template <int TB>
lre_status run_blur_support(Context* c, const BlurJob& job, const GaussTaps& taps, int W, int H, const DfScalars* sc,
                            const float* src, const DfPlanes& P, const DfConst& k) {
  constexpr int E = TB + 2 * 10;
  const size_t smem = ((size_t)E * (E + 1) + (size_t)E * TB) * sizeof(float);
  LRE_CUDA_TRY(c, cudaFuncSetAttribute(k_df_blur_support<10, TB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  dim3 grid((W + TB - 1) / TB, (H + TB - 1) / TB);
  k_df_blur_support<10, TB><<<grid, 256, smem, c->stream>>>(job, taps, W, H, sc, src, P, k);
  count_launch(c);
  return check_launch(c, "defringe blur + support");
}

__global__ void k_df_support(const float* __restrict__ src, int W, int H, DfPlanes P, DfConst k) {
  const float sensitivity = sclamp(sqrtf(smax(k.strength, 1.0f)), 1.0f, 2.5f);
  const float inv_s = 1.0f / sensitivity;
  const bool enable_green = k.green != 0;
  size_t n = (size_t)W * H;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    P.fs[i] = support_at(src, i, P, k, inv_s, enable_green);
}

// ---------------------------------------------------------------- K5
constexpr int LT = 32;   // line-link output tile
constexpr int LH = 14;   // max step along a line
constexpr int LE = LT + 2 * LH;

// Running max of a line's samples.  `along` starts at 0 and the samples are
// finite or NaN: std::max(along, v) then equals fmaxf(along, v) (neither ever
// yields NaN), so the single-instruction form is exact here.
template <int TX, int TY, int STEPS>
__device__ __forceinline__ float line_along(const float* s_ls, int c) {
  float along = 0.f;
#pragma unroll
  for (int step = 1; step <= STEPS; step++) {
    along = fmaxf(along, s_ls[c + (TY * LE + TX) * step]);
    along = fmaxf(along, s_ls[c - (TY * LE + TX) * step]);
  }
  return along;
}

template <int TX, int TY, int STEPS>
__device__ __forceinline__ void line_dir(const float* s_ls, const float* s_fs, int c, float& best) {
  const float along = line_along<TX, TY, STEPS>(s_ls, c);
  // along == 0 contributes 0 * thin (thin in [0, 1], or NaN which
  // std::max ignores) to a running max that is already >= 0
  if (along == 0.f) return;
  constexpr int NX = -TY, NY = TX;  // across-direction normal
  const float across = smax(s_fs[c + (NY * LE + NX) * 2], s_fs[c - (NY * LE + NX) * 2]);
  const float thin = 1.f - ssmooth(along * 0.45f, along * 0.95f, across);
  best = smax(best, along * thin);
}

__global__ void __launch_bounds__(256) k_df_line(const float* __restrict__ src, int W, int H, DfPlanes P, DfConst k) {
  __shared__ float s_ls[LE * LE];
  __shared__ float s_fs[LE * LE];
  __shared__ int s_any;
  const int x0 = blockIdx.x * LT, y0 = blockIdx.y * LT;
  if (threadIdx.x == 0) s_any = 0;
  __syncthreads();
  int any = 0;
  for (int i = threadIdx.x; i < LE * LE; i += blockDim.x) {
    int gy = min(max(y0 - LH + i / LE, 0), H - 1);
    int gx = min(max(x0 - LH + i % LE, 0), W - 1);
    size_t gi = (size_t)gy * W + gx;
    float f = P.fs[gi];
    s_fs[i] = f;
    const float ls = smax(f, P.bfs[gi] * 0.55f);
    s_ls[i] = ls;
    any |= ls != 0.f;
  }
  if (__any_sync(0xffffffffu, any) && (threadIdx.x & 31) == 0) s_any = 1;
  __syncthreads();
  // a tile whose line sources are all zero has every `along` zero, so every
  // line-linked support value is exactly 0
  const bool tile_active = s_any != 0;
  const float sensitivity = sclamp(sqrtf(smax(k.strength, 1.0f)), 1.0f, 2.5f);
  const float inv_s = 1.0f / sensitivity;
  for (int i = threadIdx.x; i < LT * LT; i += blockDim.x) {
    int ly = i / LT, lx = i % LT;
    int y = y0 + ly, x = x0 + lx;
    if (x >= W || y >= H) continue;
    const int c = (ly + LH) * LE + (lx + LH);
    const size_t gi = (size_t)y * W + x;
    // the solo-seed operands are loaded first, so their latency overlaps
    // the line search (which reads shared memory only); loaded after the
    // lfs store below, they would wait for it
    const float* s = src + gi * 3;
    const float s0 = s[0], s1 = s[1], s2 = s[2];
    const float blur_guide = P.bg[gi];
    const float blrg = P.blrg[gi], blbg = P.blbg[gi];
    const float bfs = P.bfs[gi], be = P.be[gi], ber = P.ber[gi];
    float best = 0.f;
    if (tile_active) {
      // directions and step counts of core/cpu_accelerator.cpp:4290-4318
      line_dir<1, 0, 14>(s_ls, s_fs, c, best);
      line_dir<0, 1, 14>(s_ls, s_fs, c, best);
      line_dir<1, 1, 14>(s_ls, s_fs, c, best);
      line_dir<1, -1, 14>(s_ls, s_fs, c, best);
      line_dir<2, 1, 6>(s_ls, s_fs, c, best);
      line_dir<1, 2, 6>(s_ls, s_fs, c, best);
      line_dir<2, -1, 6>(s_ls, s_fs, c, best);
      line_dir<1, -2, 6>(s_ls, s_fs, c, best);
    }
    P.lfs[gi] = best;

    // solo seeds (core/cpu_accelerator.cpp:4325-4374)
    const float g = smax(s1, 0.f);
    const float target_r = g * exp_cr(blrg);
    const float target_b = g * exp_cr(blbg);
    const float solo_r = smax(0.f, s0 - target_r) / smax(blur_guide, 0.05f);
    const float solo_b = smax(0.f, s2 - target_b) / smax(blur_guide, 0.05f);
    const float linked_fringe = ssmooth(0.004f, 0.045f, smax(bfs, best * 0.90f));
    const float c_edge_solo = ssmooth(k.edge_thr * 0.35f * inv_s, k.edge_thr * 1.50f * inv_s, be) *
                              ssmooth(0.55f * inv_s, 1.35f * inv_s, ber);
    const float c_bright_solo = ssmooth(0.24f * inv_s, 0.52f * inv_s, blur_guide);
    const float solo_enable = ssmooth(1.25f, 3.0f, k.strength);
    const float r0 = smax(s0, 0.f);
    const float g0 = smax(s1, 0.f);
    const float b0 = smax(s2, 0.f);
    const float red_strength_solo = smax(0.f, r0 - smax(g0, b0)) / smax(r0, 1e-4f);
    const float solo_red_guard = 1.f - 0.90f * ssmooth(0.12f, 0.32f, red_strength_solo);
    P.srs[gi] = solo_enable * c_edge_solo * c_bright_solo * linked_fringe * solo_red_guard *
                ssmooth(k.chroma_thr * 0.22f * inv_s, k.chroma_thr * 0.95f * inv_s, solo_r);
    P.sbs[gi] = solo_enable * c_edge_solo * c_bright_solo *
                ssmooth(k.chroma_thr * 0.22f * inv_s, k.chroma_thr * 0.95f * inv_s, solo_b);
  }
}

// ---------------------------------------------------------------- K7
// Constants of the main pass (core/cpu_accelerator.cpp:4376-4706), formed
// once per thread.
struct DfMainK {
  float inv_s, mask_cutoff, scene_highlight_gate, edge_threshold, chroma_threshold, strength, green_strength_scale;
  float e0_edge, e0_raw;
  bool enable_green, can_skip;
};

// The eleven planes the main pass reads at one pixel.
struct DfPx {
  float be, ber, srb, sbb, bg, blrg, blbg, bfs, lfs, lrg, lbg;
};

// Pixels that provably keep their input: with green correction off, either
// edge factor at or below its lower smoothstep edge zeroes both edge weights
// (the other factor is finite, or NaN, and a NaN mask never passes the
// cutoff), so no ratio/direct correction applies; zero solo blurs make the
// solo masks zero.  The output is then the input whatever the other planes
// hold, so those pixels need 4 planes instead of 11 and skip the rest.
__device__ __forceinline__ bool df_keeps_input(const DfMainK& K, float be, float ber, float srb, float sbb) {
  return K.can_skip && (be <= K.e0_edge || ber <= K.e0_raw) && srb == 0.f && sbb == 0.f;
}

// The correction of one pixel (s0, s1, s2) -> (d0, d1, d2).
__device__ __forceinline__ void df_main_px(float s0, float s1, float s2, const DfPx& v, const DfMainK& K, float& d0,
                                           float& d1, float& d2) {
  const float inv_s = K.inv_s;
  const float mask_cutoff = K.mask_cutoff;
  const float scene_highlight_gate = K.scene_highlight_gate;
  const bool enable_green = K.enable_green;
  const float edge_threshold = K.edge_threshold, chroma_threshold = K.chroma_threshold, strength = K.strength;
  const float green_strength_scale = K.green_strength_scale;
  d0 = s0;
  d1 = s1;
  d2 = s2;
  const float blur_guide = v.bg;
  const float blur_log_rg = v.blrg;
  const float blur_log_bg = v.blbg;
  const float blur_fringe_support = v.bfs;
  const float line_support = v.lfs;

  const float rg = v.lrg;
  const float bg = v.lbg;
  const float dr = rg - blur_log_rg;
  const float db = bg - blur_log_bg;
  const float r0 = smax(s0, 0.f);
  const float g0 = smax(s1, 0.f);
  const float b0 = smax(s2, 0.f);
  const float rb_avg_pre = 0.5f * (r0 + b0);
  const float purple_r = smax(0.f, dr);
  const float purple_b = smax(0.f, db);
  const float green_r = smax(0.f, -dr);
  const float green_b = smax(0.f, -db);
  const float purple_excess = smin(purple_r, purple_b);
  const float denom = smax(blur_guide, 0.05f);
  const float g_over_min = smax(0.f, g0 - smin(r0, b0)) / denom;
  const float green_dom = ssmooth(0.010f, 0.060f, g_over_min);
  const float green_excess = smax(green_r, green_b) * green_dom;
  const bool is_purple = purple_excess >= green_excess;
  const float excess = is_purple ? purple_excess : green_excess;
  const float min_dir = is_purple ? smax(0.f, smin(rg, bg)) : smax(0.f, smin(-rg, -bg));
  const float max_dir = is_purple ? smax(1e-4f, smax(rg, bg)) : smax(1e-4f, smax(-rg, -bg));
  const float balance = min_dir / max_dir;
  const float c_edge_core = ssmooth(edge_threshold * 0.35f * inv_s, edge_threshold * 1.50f * inv_s, v.be) *
                            ssmooth(0.55f * inv_s, 1.35f * inv_s, v.ber);
  const float c_edge_low = ssmooth(edge_threshold * 0.10f * inv_s, edge_threshold * 0.80f * inv_s, v.be) *
                           ssmooth(0.20f * inv_s, 0.90f * inv_s, v.ber);
  const float linked_fringe = ssmooth(0.004f, 0.045f, smax(blur_fringe_support, line_support * 0.90f));
  const float c_bright = ssmooth(0.24f * inv_s, 0.52f * inv_s, blur_guide);
  const float c_chroma = ssmooth(chroma_threshold * 0.45f * inv_s, chroma_threshold * 1.60f * inv_s, excess);
  const float red_blue_balance_hue = b0 / smax(r0, 1e-4f);
  const float blue_lift_hue = smax(0.f, b0 - g0) / smax(r0 - g0, 1e-4f);
  const float red_purple_hue_signal = ssmooth(0.50f, 0.72f, red_blue_balance_hue) * ssmooth(0.24f, 0.42f, blue_lift_hue);
  const float balanced_hue = ssmooth(0.06f * inv_s, 0.22f * inv_s, min_dir) * ssmooth(0.35f, 0.75f, balance);
  const float red_purple_hue_gate = is_purple ? smin(1.f, red_purple_hue_signal * 1.50f) *
                                                    ssmooth(0.035f * inv_s, 0.16f * inv_s, min_dir) *
                                                    ssmooth(0.18f, 0.58f, balance)
                                              : 0.f;
  const float green_unbalanced_hue =
      (enable_green && !is_purple) ? ssmooth(0.035f * inv_s, 0.16f * inv_s, max_dir) : 0.f;
  const float c_hue = smax(balanced_hue, smax(red_purple_hue_gate, green_unbalanced_hue));
  const float rb_avg = rb_avg_pre;
  const float purple_abs = smin(smax(0.f, r0 - g0), smax(0.f, b0 - g0)) / smax(blur_guide, 0.05f);
  const float green_abs_base = smax(0.f, g0 - rb_avg) / smax(blur_guide, 0.05f);
  const float green_abs_alt = smax(0.f, g0 - smin(r0, b0)) / smax(blur_guide, 0.05f);
  const float green_abs = smax(green_abs_base, 0.55f * green_abs_alt);
  const bool abs_is_purple = purple_abs >= green_abs;
  const float abs_excess = abs_is_purple ? purple_abs : green_abs;
  const float c_abs = ssmooth(chroma_threshold * 0.35f * inv_s, chroma_threshold * 1.20f * inv_s, abs_excess);
  const float low_contrast_color =
      ssmooth(chroma_threshold * 1.20f * inv_s, chroma_threshold * 2.40f * inv_s, abs_excess);
  const float green_soft_edge_boost =
      (enable_green && !is_purple) ? c_edge_low * ssmooth(0.05f * inv_s, 0.20f * inv_s, max_dir) : 0.f;
  const float c_edge = smax(c_edge_core, smax(c_edge_low * linked_fringe * 1.45f,
                                              smax(c_edge_low * low_contrast_color * 0.35f, green_soft_edge_boost)));
  const float ratio_mask = c_edge * c_bright * c_hue * c_chroma;
  const float direct_mask = c_edge * c_bright * c_hue * c_abs;
  const bool use_direct = direct_mask > ratio_mask;
  float mask = smax(ratio_mask, direct_mask) * scene_highlight_gate;
  const bool correct_purple = use_direct ? abs_is_purple : is_purple;
  float local_gate = 0.f;
  if (correct_purple) {
    local_gate = ssmooth(chroma_threshold * 0.10f * inv_s, chroma_threshold * 0.55f * inv_s, purple_abs);
    mask *= local_gate;
  } else {
    local_gate = ssmooth(chroma_threshold * 0.10f * inv_s, chroma_threshold * 0.55f * inv_s, green_abs);
    if (enable_green) {
      const float peak_chroma_signal =
          ssmooth(chroma_threshold * 0.80f * inv_s, chroma_threshold * 2.50f * inv_s, green_abs);
      const float peak_neighbourhood = ssmooth(0.005f, 0.030f, blur_fringe_support);
      const float green_peak_mask = peak_chroma_signal * peak_neighbourhood * c_bright * c_hue;
      mask = smax(mask, green_peak_mask * scene_highlight_gate);
    }
    const float green_highlight_protect = 1.f - 0.85f * ssmooth(0.62f, 0.88f, blur_guide);
    const float rb_to_green = rb_avg / smax(g0, 1e-4f);
    const float natural_green_highlight = ssmooth(0.22f, 0.46f, rb_to_green) * ssmooth(0.30f, 0.55f, g0);
    const float natural_green_suppress = 1.f - 0.99f * natural_green_highlight;
    const float natural_green_suppress_sq = natural_green_suppress * natural_green_suppress;
    const float green_halo_strength =
        ssmooth(chroma_threshold * 0.55f * inv_s, chroma_threshold * 1.65f * inv_s, green_abs);
    const float green_gain_base = enable_green ? 0.60f : 0.35f;
    const float green_gain_slope = enable_green ? 1.10f : 0.95f;
    const float green_gain = green_gain_base + green_gain_slope * green_halo_strength;
    const float min_ratio_ref = smin(blur_log_rg, blur_log_bg);
    const float green_neighbour = ssmooth(0.02f, 0.10f, smax(0.f, -min_ratio_ref));
    const float src_max = smax(r0, smax(g0, b0));
    const float src_min = smin(r0, smin(g0, b0));
    const float src_chroma = src_max - src_min;
    const float src_sat = src_chroma / smax(src_max, 1e-4f);
    const float whiteish = 1.f - ssmooth(0.05f, 0.13f, src_sat);
    const float foliage_guard =
        green_neighbour * whiteish * ssmooth(0.35f, 0.75f, blur_guide) * (1.f - green_halo_strength);
    const float strength_release = enable_green ? ssmooth(2.0f, 6.0f, strength) : 0.f;
    const float green_line_evidence = ssmooth(0.004f, 0.030f, line_support) *
                                      ssmooth(0.20f, 0.55f, green_halo_strength) * ssmooth(0.05f, 0.15f, src_sat);
    const float not_natural_green = 1.f - natural_green_highlight;
    const float guard_release = strength_release * green_line_evidence * not_natural_green;
    const float released_highlight_protect = green_highlight_protect + (1.f - green_highlight_protect) * guard_release;
    const float released_natural_suppress =
        natural_green_suppress_sq + (1.f - natural_green_suppress_sq) * guard_release;
    const float foliage_term = 1.f - 0.999f * foliage_guard;
    const float released_foliage_term = foliage_term + (1.f - foliage_term) * guard_release;
    mask *= local_gate * green_gain * released_highlight_protect * released_natural_suppress * released_foliage_term;
    const float line_kill_evidence = ssmooth(0.04f, 0.15f, line_support);
    const float natural_blob =
        sqrtf(smax(0.f, natural_green_highlight)) * (1.f - line_kill_evidence) * green_neighbour;
    mask *= 1.f - 0.999f * natural_blob;
    if (!enable_green) mask = 0.f;
  }

  bool skip_rest = false;
  if (mask > mask_cutoff) {
    const float g = smax(s1, 0.f);
    const float red_strength = smax(0.f, r0 - smax(g0, b0)) / smax(r0, 1e-4f);
    const float red_blue_balance = b0 / smax(r0, 1e-4f);
    const float blue_lift = smax(0.f, b0 - g0) / smax(r0 - g0, 1e-4f);
    const float red_purple_balance = ssmooth(0.55f, 0.78f, red_blue_balance);
    const float red_purple_lift = ssmooth(0.16f, 0.34f, blue_lift);
    const float red_purple = smax(red_purple_balance, red_purple_lift);
    const float red_strength_guard = ssmooth(0.08f, 0.25f, red_strength);
    float red_purple_context = 0.f;
    float contextual_red_purple = 0.f;
    float red_magenta_surface = 0.f;
    if (red_purple > 0.50f) {
      red_purple_context = linked_fringe;
      contextual_red_purple = red_purple * red_purple_context;
      if (red_purple_context < 0.20f && red_strength_guard < 0.50f && red_purple > 0.50f) {
        red_magenta_surface = ssmooth(0.02f, 0.12f, purple_abs) * (1.f - red_purple_context);
      }
    }
    float neutral_gray_surface = 0.f;
    if (strength > 3.f && red_purple_context > 0.80f && line_support > 0.012f && red_strength_guard < 0.98f &&
        blue_lift > 1.10f && red_blue_balance > 0.82f && purple_abs > 0.015f) {
      const float neutral_gray_edge = ssmooth(1.10f, 1.80f, blue_lift) * ssmooth(0.82f, 1.05f, red_blue_balance) *
                                      (1.f - red_strength_guard);
      neutral_gray_surface = neutral_gray_edge * ssmooth(0.015f, 0.08f, purple_abs) * ssmooth(3.f, 8.f, strength);
    }
    const float red_object_strength = smax(red_strength_guard, red_magenta_surface);
    const float natural_warm_guard_base = 1.f - red_object_strength * (1.f - contextual_red_purple);
    const float natural_warm_guard_sq =
        natural_warm_guard_base * natural_warm_guard_base * natural_warm_guard_base * natural_warm_guard_base;
    const float natural_warm_guard = natural_warm_guard_sq * natural_warm_guard_sq;
    const float line_purple_relief = ssmooth(0.012f, 0.06f, line_support) * ssmooth(0.10f, 0.24f, blue_lift);
    const float red_object_guard = ssmooth(0.55f, 0.90f, red_object_strength);
    const float linked_override = linked_fringe * 1.05f * (1.f - 0.85f * red_object_guard);
    const float line_override = line_purple_relief * (1.f - 0.85f * red_object_guard);
    const bool force_warm_guard = (red_object_guard > 0.75f) && (linked_fringe < 0.65f) && (line_purple_relief < 0.45f);
    const float warm_protect = correct_purple
                                   ? (force_warm_guard ? natural_warm_guard
                                                       : smax(natural_warm_guard, smax(linked_override, line_override)))
                                   : 1.f;
    const float red_without_support =
        ssmooth(0.22f, 0.45f, red_strength) * (1.f - ssmooth(0.02f, 0.12f, blur_fringe_support));
    const float protect = correct_purple ? red_without_support : 0.f;
    const float smooth_mask = ssmooth(mask_cutoff, mask_cutoff * 5.0f, mask);
    const float threshold_soften = 1.f - 0.86f * ssmooth(0.22f, 0.40f, chroma_threshold);
    const float src_max = smax(r0, smax(g0, b0));
    const float src_min = smin(r0, smin(g0, b0));
    const float src_chroma = src_max - src_min;
    const float src_sat = src_chroma / smax(src_max, 1e-4f);
    const float neutral_guard_base = ssmooth(0.008f, 0.030f, src_sat);
    const float neutral_guard = 1.f - (1.f - neutral_guard_base) * ssmooth(0.35f, 0.80f, red_object_strength);
    float amount = sclamp(smooth_mask * strength * 1.90f * (1.f - protect) * warm_protect * neutral_guard *
                              threshold_soften,
                          0.f, 1.f);
    const float warm_edge_surface = ssmooth(0.006f, 0.035f, purple_abs) * ssmooth(0.25f, 0.65f, red_purple) *
                                    ssmooth(0.15f, 0.65f, red_purple_context) * (1.f - 0.55f * red_strength_guard) *
                                    ssmooth(3.f, 8.f, strength);
    const float safe_surface = smax(neutral_gray_surface, warm_edge_surface);
    if (correct_purple && safe_surface > 1e-4f) {
      const float safe_amount_cap = 1.f - 0.99f * safe_surface;
      amount = smin(amount, safe_amount_cap);
    }
    if (amount <= 1e-4f) {
      skip_rest = true;
    } else {
      const float e_rg = exp_cr(blur_log_rg);
      const float e_bg = exp_cr(blur_log_bg);
      const float target_r = smin(g, g * e_rg);
      const float target_b = smin(g, g * e_bg);
      if (correct_purple) {
        float corrected_r = sclamp(s0 * (1.f - amount) + target_r * amount, 0.f, s0);
        float corrected_g = s1;
        float corrected_b = sclamp(s2 * (1.f - amount) + target_b * amount, 0.f, s2);
        if (safe_surface > 1e-4f) {
          const float luma_before = 0.2126f * s0 + 0.7152f * s1 + 0.0722f * s2;
          const float luma_after = 0.2126f * corrected_r + 0.7152f * corrected_g + 0.0722f * corrected_b;
          const float max_luma_drop = luma_before * 0.02f * (1.f - neutral_gray_surface);
          const float min_luma = smax(0.f, luma_before - max_luma_drop);
          if (luma_after < min_luma) {
            const float lift = min_luma - luma_after;
            const float channel_ceil = smax(s0, smax(s1, s2));
            corrected_r = smin(s0, corrected_r + lift);
            corrected_g = smin(channel_ceil, corrected_g + lift);
            corrected_b = smin(s2, corrected_b + lift);
          }
          const float smx = smax(s0, smax(s1, s2));
          const float smn = smin(s0, smin(s1, s2));
          const float cmx = smax(corrected_r, smax(corrected_g, corrected_b));
          const float cmn = smin(corrected_r, smin(corrected_g, corrected_b));
          const float sch = smx - smn;
          const float cch = cmx - cmn;
          const float min_chroma = sch * (1.f - 0.12f * safe_surface);
          if (sch > 1e-4f && cch < min_chroma) {
            const float dn = smax(sch - cch, 1e-4f);
            const float keep = sclamp((sch - min_chroma) / dn, 0.f, 1.f);
            corrected_r = s0 * (1.f - keep) + corrected_r * keep;
            corrected_g = s1 * (1.f - keep) + corrected_g * keep;
            corrected_b = s2 * (1.f - keep) + corrected_b * keep;
          }
        }
        d0 = corrected_r;
        d1 = corrected_g;
        d2 = corrected_b;
      } else {
        float target_g = s1;
        const float rg_ref = e_rg;
        const float bg_ref = e_bg;
        if (rg_ref > 1e-4f && bg_ref > 1e-4f) {
          const float g_from_r = smax(s0, 0.f) / rg_ref;
          const float g_from_b = smax(s2, 0.f) / bg_ref;
          target_g = 0.5f * (g_from_r + g_from_b);
        }
        const float rb_avg_target = 0.5f * (smax(s0, 0.f) + smax(s2, 0.f));
        target_g = smax(target_g, rb_avg_target);
        const float green_amount = sclamp(amount * green_strength_scale, 0.f, 1.f);
        d0 = s0;
        d1 = sclamp(s1 * (1.f - green_amount) + target_g * green_amount, 0.f, s1);
        d2 = s2;
      }
    }
  }

  if (!skip_rest) {
    const float solo_enable = ssmooth(1.25f, 3.0f, strength);
    if (solo_enable > 0.f) {
      const float g = smax(s1, 0.f);
      const float target_r = g * exp_cr(blur_log_rg);
      const float target_b = g * exp_cr(blur_log_bg);
      const float solo_r = smax(0.f, s0 - target_r) / smax(blur_guide, 0.05f);
      const float solo_b = smax(0.f, s2 - target_b) / smax(blur_guide, 0.05f);
      const float local_solo_r =
          ssmooth(chroma_threshold * 0.12f * inv_s, chroma_threshold * 0.65f * inv_s, solo_r);
      const float local_solo_b =
          ssmooth(chroma_threshold * 0.12f * inv_s, chroma_threshold * 0.65f * inv_s, solo_b);
      const float rr0 = smax(s0, 0.f);
      const float gg0 = g;
      const float bb0 = smax(s2, 0.f);
      const float g_over_min2 = smax(0.f, gg0 - smin(rr0, bb0)) / smax(blur_guide, 0.05f);
      const float green_dom2 = ssmooth(0.010f, 0.060f, g_over_min2);
      const float denom_solo = smax(blur_guide, 0.05f);
      const float purpleish =
          ssmooth(0.010f, 0.060f, smax(smax(0.f, rr0 - gg0), smax(0.f, bb0 - gg0)) / denom_solo);
      const float solo_allow = 1.f - green_dom2 * (1.f - purpleish);
      const float solo_r_mask = v.srb * local_solo_r * solo_allow;
      const float solo_b_mask = v.sbb * local_solo_b * solo_allow;
      if (solo_r_mask > mask_cutoff) {
        const float amount = sclamp(solo_r_mask * strength * 0.85f, 0.f, 0.85f);
        d0 = sclamp(d0 * (1.f - amount) + target_r * amount, 0.f, d0);
      }
      if (solo_b_mask > mask_cutoff) {
        const float amount = sclamp(solo_b_mask * strength * 0.95f, 0.f, 0.90f);
        d2 = sclamp(d2 * (1.f - amount) + target_b * amount, 0.f, d2);
      }
    }
  }
}

__device__ __forceinline__ void ld4(const float* p, float* o) {
  const float4 t = *reinterpret_cast<const float4*>(p);
  o[0] = t.x;
  o[1] = t.y;
  o[2] = t.z;
  o[3] = t.w;
}
__device__ __forceinline__ void st4(float* p, const float* o) {
  *reinterpret_cast<float4*>(p) = make_float4(o[0], o[1], o[2], o[3]);
}

// Four consecutive pixels per thread and step, read and written as float4
// (src/dst 16-byte aligned; the planes are 256-byte aligned), so every load
// of a step is issued before the first use; the one-pixel loop was bound by
// load latency.  The keep-input test reads 4 planes; the other 7 are read
// only when a pixel of the group needs them.  The group's operands are then
// staged in shared memory (one column per thread) and one copy of the
// per-pixel code runs over the four pixels.
constexpr int DFM_THREADS = 128;
constexpr int DFM_VALS = 14;  // s0 s1 s2 be ber srb sbb bg blrg blbg bfs lfs lrg lbg

__global__ void __launch_bounds__(DFM_THREADS, 6) k_df_main(const float* src, float* dst, int W, int H, DfPlanes P,
                                                           DfConst k, const DfScalars* sc, float* out_max_g) {
  __shared__ float S[DFM_VALS * 4][DFM_THREADS];
  DfMainK K;
  const float sensitivity = sclamp(sqrtf(smax(k.strength, 1.0f)), 1.0f, 2.5f);
  K.inv_s = 1.0f / sensitivity;
  K.mask_cutoff = 0.02f * K.inv_s;
  const float max_guide = df_max_guide(sc);
  K.scene_highlight_gate = ssmooth(0.55f, 0.75f, max_guide);
  K.enable_green = k.green != 0;
  K.edge_threshold = k.edge_thr;
  K.chroma_threshold = k.chroma_thr;
  K.strength = k.strength;
  K.green_strength_scale = sclamp(k.green_scale, 0.f, 1.f);
  K.e0_edge = K.edge_threshold * 0.10f * K.inv_s;
  K.e0_raw = 0.20f * K.inv_s;
  K.can_skip = !K.enable_green && K.edge_threshold > 0.f;  // smoothstep edges strictly ordered
  const size_t n = (size_t)W * H;
  const bool vec = ((reinterpret_cast<uintptr_t>(src) | reinterpret_cast<uintptr_t>(dst)) & 15) == 0;
  const size_t n4 = vec ? n / 4 : 0;
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  const int tid = threadIdx.x;
  float mg = 0.f;  // max(0, G) of what this thread writes (fmaxf drops NaN)
  for (size_t q = blockIdx.x * (size_t)blockDim.x + tid; q < n4; q += stride) {
    const size_t i = q * 4;
    float s[12], be[4], ber[4], srb[4], sbb[4];
    ld4(src + i * 3, s);
    ld4(src + i * 3 + 4, s + 4);
    ld4(src + i * 3 + 8, s + 8);
    ld4(P.be + i, be);
    ld4(P.ber + i, ber);
    ld4(P.srb + i, srb);
    ld4(P.sbb + i, sbb);
    unsigned keep = 0;
#pragma unroll
    for (int t = 0; t < 4; t++) keep |= df_keeps_input(K, be[t], ber[t], srb[t], sbb[t]) ? 1u << t : 0u;
    if (keep == 0xFu) {
      st4(dst + i * 3, s);
      st4(dst + i * 3 + 4, s + 4);
      st4(dst + i * 3 + 8, s + 8);
      mg = fmaxf(mg, fmaxf(fmaxf(s[1], s[4]), fmaxf(s[7], s[10])));
      continue;
    }
    float pl[7][4];
    ld4(P.bg + i, pl[0]);
    ld4(P.blrg + i, pl[1]);
    ld4(P.blbg + i, pl[2]);
    ld4(P.bfs + i, pl[3]);
    ld4(P.lfs + i, pl[4]);
    ld4(P.lrg + i, pl[5]);
    ld4(P.lbg + i, pl[6]);
    // S[v * 4 + t][tid]: value v of pixel t
#pragma unroll
    for (int t = 0; t < 4; t++) {
      S[0 * 4 + t][tid] = s[3 * t];
      S[1 * 4 + t][tid] = s[3 * t + 1];
      S[2 * 4 + t][tid] = s[3 * t + 2];
      S[3 * 4 + t][tid] = be[t];
      S[4 * 4 + t][tid] = ber[t];
      S[5 * 4 + t][tid] = srb[t];
      S[6 * 4 + t][tid] = sbb[t];
#pragma unroll
      for (int v = 0; v < 7; v++) S[(7 + v) * 4 + t][tid] = pl[v][t];
    }
#pragma unroll 1
    for (int t = 0; t < 4; t++) {
      if (keep >> t & 1u) continue;
      const DfPx v{S[3 * 4 + t][tid],  S[4 * 4 + t][tid],  S[5 * 4 + t][tid],  S[6 * 4 + t][tid],
                   S[7 * 4 + t][tid],  S[8 * 4 + t][tid],  S[9 * 4 + t][tid],  S[10 * 4 + t][tid],
                   S[11 * 4 + t][tid], S[12 * 4 + t][tid], S[13 * 4 + t][tid]};
      float r0, r1, r2;
      df_main_px(S[0 * 4 + t][tid], S[1 * 4 + t][tid], S[2 * 4 + t][tid], v, K, r0, r1, r2);
      S[0 * 4 + t][tid] = r0;
      S[1 * 4 + t][tid] = r1;
      S[2 * 4 + t][tid] = r2;
    }
    float d[12];
#pragma unroll
    for (int t = 0; t < 4; t++) {
      d[3 * t] = S[0 * 4 + t][tid];
      d[3 * t + 1] = S[1 * 4 + t][tid];
      d[3 * t + 2] = S[2 * 4 + t][tid];
    }
    st4(dst + i * 3, d);
    st4(dst + i * 3 + 4, d + 4);
    st4(dst + i * 3 + 8, d + 8);
    mg = fmaxf(mg, fmaxf(fmaxf(d[1], d[4]), fmaxf(d[7], d[10])));
  }
  for (size_t i = n4 * 4 + blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += stride) {
    const float s0 = src[i * 3 + 0], s1 = src[i * 3 + 1], s2 = src[i * 3 + 2];
    float d0 = s0, d1 = s1, d2 = s2;
    if (!df_keeps_input(K, P.be[i], P.ber[i], P.srb[i], P.sbb[i])) {
      const DfPx v{P.be[i], P.ber[i], P.srb[i], P.sbb[i], P.bg[i],  P.blrg[i],
                   P.blbg[i], P.bfs[i], P.lfs[i], P.lrg[i], P.lbg[i]};
      df_main_px(s0, s1, s2, v, K, d0, d1, d2);
    }
    dst[i * 3 + 0] = d0;
    dst[i * 3 + 1] = d1;
    dst[i * 3 + 2] = d2;
    mg = fmaxf(mg, d1);
  }
  if (out_max_g) {  // every thread of the block gets here
    mg = warp_max(mg);
    if ((tid & 31) == 0) atomic_max_float(out_max_g, mg);
  }
}

__global__ void k_df_init(DfScalars* sc, const float* in_max_g, float* out_max_g) {
  sc->max_guide_raw = in_max_g ? *in_max_g : 0.f;
  sc->max_edge = 0.f;
  if (out_max_g) *out_max_g = 0.f;
}

__global__ void k_df_maxg(const float* __restrict__ src, size_t n, DfScalars* sc) {
  float m = 0.f;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    m = smax(m, smax(0.f, src[i * 3 + 1]));
  m = warp_max(m);
  if ((threadIdx.x & 31) == 0) atomic_max_float(&sc->max_guide_raw, m);
}

lre_status run_blur(Context* c, const BlurJob& job, const GaussTaps& taps, int W, int H, const DfScalars* sc) {
  if (taps.ks == 10)  // radius 10 (the reference default): sigma 10/3, 21 taps
    return c->tune.blur_tile == 64 ? run_blur_fast<64>(c, job, taps, W, H, sc) : run_blur_fast<32>(c, job, taps, W, H, sc);
  const int E = BT + 2 * taps.ks;
  size_t smem = ((size_t)job.np * E * E + (size_t)job.np * E * BT) * sizeof(float);
  LRE_CUDA_TRY(c, cudaFuncSetAttribute(k_df_blur, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  dim3 grid((W + BT - 1) / BT, (H + BT - 1) / BT);
  k_df_blur<<<grid, 256, smem, c->stream>>>(job, taps, W, H, sc);
  count_launch(c);
  return check_launch(c, "defringe blur");
}

}  // namespace

size_t ws_bytes_defringe(size_t w, size_t h, float radius) {
  (void)radius;
  return 15 * ((w * h * sizeof(float) + 255) & ~size_t(255)) + 256;
}

lre_status launch_defringe(Context* c, const float* in, float* out, size_t w, size_t h, float radius,
                           float edge_thr, float chroma_thr, float strength, bool green, float green_scale,
                           const float* in_max_g, float* out_max_g) {
  GaussTaps taps = make_defringe_taps(radius);
  {
    const float sigma = std::max(radius / 3.f, 0.5f);
    if (static_cast<int>(std::ceil(3.f * sigma)) > GAUSS_MAX_KS)
      return fail(c, LRE_ERR_INVALID_ARGUMENT, "defringe: radius > 32 is not supported");
  }
  const int W = (int)w, H = (int)h;
  const size_t plane = (w * h * sizeof(float) + 255) & ~size_t(255);
  DfPlanes P;
  float** slots[15] = {&P.lrg, &P.lbg, &P.er, &P.bg, &P.blrg, &P.blbg, &P.be, &P.ber,
                       &P.fs,  &P.bfs, &P.lfs, &P.srs, &P.sbs, &P.srb, &P.sbb};
  for (int i = 0; i < 15; i++) {
    *slots[i] = reinterpret_cast<float*>(c->ws.take(plane));
    if (!*slots[i]) return fail(c, LRE_ERR_OUT_OF_MEMORY, "defringe: workspace too small");
  }
  DfScalars* sc = reinterpret_cast<DfScalars*>(c->ws.take(sizeof(DfScalars)));
  if (!sc) return fail(c, LRE_ERR_OUT_OF_MEMORY, "defringe: workspace too small");
  DfConst k{edge_thr, chroma_thr, strength, green_scale, green ? 1 : 0};
  const size_t n = w * h;
  const unsigned gstream = grid_for(n, 256, c->sm_count * 8);

  k_df_init<<<1, 1, 0, c->stream>>>(sc, in_max_g, out_max_g);
  count_launch(c);
  if (!in_max_g) {
    k_df_maxg<<<grid_for(n, 256, c->sm_count * 4), 256, 0, c->stream>>>(in, n, sc);
    count_launch(c);
  }
  const size_t prep_tiles = (size_t)((W + PT_X - 1) / PT_X) * ((H + PT_Y - 1) / PT_Y);
  k_df_prep_tiled<<<(unsigned)std::min<size_t>(prep_tiles, (size_t)c->sm_count * 8), 256, 0, c->stream>>>(
      in, W, H, sc, P.lrg, P.lbg, P.er);
  count_launch(c);
  LRE_TRY(check_launch(c, "defringe prep"));

  BlurJob j1{};
  j1.np = 5;
  j1.in[0] = in;    j1.mode[0] = BS_GUIDE_LINEAR;    j1.out[0] = P.bg;
  j1.in[1] = P.lrg; j1.mode[1] = BS_PLANE;           j1.out[1] = P.blrg;
  j1.in[2] = P.lbg; j1.mode[2] = BS_PLANE;           j1.out[2] = P.blbg;
  j1.in[3] = P.er;  j1.mode[3] = BS_PLANE_EDGE_NORM; j1.out[3] = P.be;
  j1.in[4] = P.er;  j1.mode[4] = BS_PLANE;           j1.out[4] = P.ber;
  if (taps.ks == 10) {  // radius 10: the register-tiled blur with K3 fused
    LRE_TRY(c->tune.blur_tile == 64 ? run_blur_support<64>(c, j1, taps, W, H, sc, in, P, k)
                                    : run_blur_support<32>(c, j1, taps, W, H, sc, in, P, k));
  } else {
    LRE_TRY(run_blur(c, j1, taps, W, H, sc));
    k_df_support<<<gstream, 256, 0, c->stream>>>(in, W, H, P, k);
    count_launch(c);
    LRE_TRY(check_launch(c, "defringe support"));
  }

  BlurJob j2{};
  j2.np = 1;
  j2.in[0] = P.fs; j2.mode[0] = BS_PLANE; j2.out[0] = P.bfs;
  LRE_TRY(run_blur(c, j2, taps, W, H, sc));

  dim3 lgrid((W + LT - 1) / LT, (H + LT - 1) / LT);
  k_df_line<<<lgrid, 256, 0, c->stream>>>(in, W, H, P, k);
  count_launch(c);
  LRE_TRY(check_launch(c, "defringe line"));

  BlurJob j3{};
  j3.np = 2;
  j3.in[0] = P.srs; j3.mode[0] = BS_PLANE; j3.out[0] = P.srb;
  j3.in[1] = P.sbs; j3.mode[1] = BS_PLANE; j3.out[1] = P.sbb;
  LRE_TRY(run_blur(c, j3, taps, W, H, sc));

  k_df_main<<<grid_for((n + 3) / 4, DFM_THREADS, c->sm_count * 6), DFM_THREADS, 0, c->stream>>>(in, out, W, H, P, k,
                                                                                                sc, out_max_g);
  count_launch(c);
  return check_launch(c, "defringe main");
}

}  // namespace lre
