// k_amaze.cu -- AMaZE Bayer demosaic (RawTherapee's algorithm as ported in
// libraw_enhanced) followed by the 4-px LibRaw border interpolation.
//
// Semantics: core/cpu_accelerator.cpp:1145-1630 (AMaZE_Processor_RT) and
// :1635-1653 (demosaic_bayer_amaze -> border_interpolate(4), :2984-3028).
//
// The reference's result depends on its tiling, not only on the image:
//   * tiles are 160 x 160 (TS) with a 16-px apron, stepping 128 px, starting
//     at -16 (:1243-1246); the last tile row/column is shorter;
//   * stage 3 updates hcd / vcd in place while scanning, so each row (hcd)
//     and each column (vcd) of a tile is a sequential chain (:1376-1398);
//   * stage 6 (hvwt) and stage 9 (pmwt) are in-place Gauss-Seidel sweeps:
//     row rr reads the already-updated row rr-1 (:1456-1464, :1537-1542);
//   * pmwt is stored half-indexed in dirwts1's memory (:1507), and stage 9
//     later reads dirwts1 full-indexed (:1556), so part of what it reads is
//     pmwt -- that aliasing is reproduced explicitly below (dirwts1_eff).
//
// Device design: a persistent CTA per SM pulls the reference's tiles from a
// counter and runs each one stage by stage.
//   * Scratch: one slab per CTA of 6 full planes (160x160 floats) plus one
//     half plane; the reference's ~20 planes are mapped onto it by lifetime
//     (a plane is reused once its last reader has run), the cheap gradient
//     planes (dirwts0/1, delhvsqsum) are recomputed from cfa where read, and
//     R/B-only quantities are stored half-indexed.  148 slabs (~95 MB) sit
//     in L2.
//   * cfa (read by nearly every stage) lives in shared memory (102 KB).
//   * hvwt and pmwt live in shared memory (2 x 51 KB), so both Gauss-Seidel
//     sweeps chase their row-to-row dependency through SMEM; the work that
//     only needs a site's final weight runs in a parallel pass afterwards.
//   * Stage-3 chains run one chain per thread with the next step's operands
//     loaded ahead of the dependent arithmetic.
// Positions the reference reads without writing in the same tile read zeros
// (a freshly allocated buffer): the 4-px frame of vcd/hcd/vcdalt/hcdalt, the
// nyquist maps, Dgrb1, and the unfilled apron corners of corner tiles.
#include "common.cuh"
#include "lre_internal.h"

namespace lre {

namespace {

constexpr int TS = 160;
constexpr int TSH = TS / 2;
constexpr int TS2 = TS * TS;
constexpr int HALF = TS * TSH;
constexpr int AMZ_THREADS = 1024;

constexpr float eps = 1e-5f;
constexpr float epssq = 1e-10f;
constexpr float arthresh = 0.75f;
constexpr float nyqthresh = 0.5f;

// Stencil weights of the reference (:1155-1161).
__constant__ float gaussodd[4] = {0.14659727707323927f, 0.103592713382435f, 0.0732036125103057f, 0.0365543548389495f};
__constant__ float gaussgrad[6] = {nyqthresh * 0.07384411893421103f, nyqthresh * 0.06207511968171489f,
                                   nyqthresh * 0.0521818194747806f,  nyqthresh * 0.03687419286733595f,
                                   nyqthresh * 0.03099732204057846f, nyqthresh * 0.018413194161458882f};
__constant__ float gausseven[2] = {0.13719494435797422f, 0.05640252782101291f};
__constant__ float gquinc[4] = {0.169917f, 0.108947f, 0.069855f, 0.0287182f};

__device__ __forceinline__ float SQR(float x) { return x * x; }
__device__ __forceinline__ float xmul2f(float x) { return x + x; }
__device__ __forceinline__ float xdiv2f(float x) { return x * 0.5f; }

constexpr size_t kFull = 6;
constexpr size_t kSlabBytes = kFull * TS2 * 4 + 2 * HALF + 256;  // + nyquist, nyquist2 bytes
constexpr size_t kSmemBytes = 2 * HALF * 4 + TS2 * 4;            // hvwt + pmwt + cfa

// Lifetime map of the reference's planes onto the slab (F0..F5 full planes;
// "a"/"b" = first/second half of a full plane):
//   F0 vcd  (S2..S6)     -> a rbm, b rbp     (S8..S9)
//   F1 hcd  (S2..S6)     -> a pmwt copy-out unused, b rbint (S9)
//   F2 vcdalt (S2..S3)   -> a cddiffsq (S3..S5) then Dgrb0 (S6..S10), b rgbgreen@R/B (S6..S10)
//   F3 hcdalt (S2..S3)   -> a Dgrb2h, b Dgrb2v (S6) -> a Dgrb1 (S9..S10)
//   F4 dgintv (S2..S5)   -> a delp, b delm (S7..S8)
//   F5 dginth (S2..S5)   -> a Dgrbsq1p, b Dgrbsq1m (S7..S8)
//   SMEM: cfa (fill..S10), hvwt (S4..S10), pmwt (S8..S9)
struct Slab {
  float *cfa, *vcd, *hcd, *vcdalt, *hcdalt, *dgintv, *dginth;
  float *rbm, *rbp, *rbint, *cddiffsq, *Dgrb0, *rgbg, *Dgrb2h, *Dgrb2v, *Dgrb1, *delp, *delm, *Dq1p, *Dq1m;
  unsigned char *nyquist, *nyquist2;
};

__device__ Slab make_slab(unsigned char* base, float* cfa_smem) {
  Slab s;
  float* F = reinterpret_cast<float*>(base);
  s.cfa = cfa_smem;
  s.vcd = F + 0 * TS2;
  s.hcd = F + 1 * TS2;
  s.vcdalt = F + 2 * TS2;
  s.hcdalt = F + 3 * TS2;
  s.dgintv = F + 4 * TS2;
  s.dginth = F + 5 * TS2;
  s.rbm = s.vcd;
  s.rbp = s.vcd + HALF;
  s.rbint = s.hcd + HALF;
  s.cddiffsq = s.vcdalt;
  s.Dgrb0 = s.vcdalt;
  s.rgbg = s.vcdalt + HALF;
  s.Dgrb2h = s.hcdalt;
  s.Dgrb2v = s.hcdalt + HALF;
  s.Dgrb1 = s.hcdalt;
  s.delp = s.dgintv;
  s.delm = s.dgintv + HALF;
  s.Dq1p = s.dginth;
  s.Dq1m = s.dginth + HALF;
  s.nyquist = reinterpret_cast<unsigned char*>(F + kFull * TS2);
  s.nyquist2 = s.nyquist + HALF;
  return s;
}

struct AmazeArgs {
  const float* raw;
  int cstride;  // 1: dense CFA mosaic, 3: sparse (H,W,3) raw buffer
  float* rgb;
  int W, H;
  uint32_t filters;
  unsigned cfarray[2][2];
  unsigned cfpack;  // cfarray packed 2 bits per site: bit 2*((r&1)*2+(c&1))
  int ex, ey;
  float clip_pt, clip_pt8, scale;
  int n_top, n_left;
  int tile_lo, tile_hi;  // tiles [tile_lo, tile_hi) of the n_top x n_left grid
  unsigned char* scratch;
  int* tile_counter;
  float* max_g;  // nullable: max(0, G) of the interior outputs (the 4-px frame is left to the border pass)
};

// (a packed lookup: indexing the parameter's array at run time would copy the
// whole parameter block to local memory)
__device__ __forceinline__ unsigned fc_rt(const AmazeArgs& a, int r, int c) {
  return (a.cfpack >> (2 * (((r & 1) << 1) | (c & 1)))) & 3u;
}

__device__ __forceinline__ float raw_at(const AmazeArgs& a, int row, int col) {
  size_t i = (size_t)row * a.W + col;
  if (a.cstride == 1) return a.raw[i];
  return a.raw[i * 3 + fc_rt(a, row, col)];
}

// n / d for 0 <= n < 2^16 by a multiply-high (exact in that range): the
// per-stage site loops map a flat index to (row, site) every iteration.
struct FDiv {
  unsigned m;
  int d;
  __device__ explicit FDiv(int d_) : m(d_ > 1 ? 0xFFFFFFFFu / (unsigned)d_ + 1u : 0u), d(d_) {}
  __device__ __forceinline__ int div(int n) const { return (int)__umulhi((unsigned)n, m) + (d == 1 ? n : 0); }
};

// The reference's stage-1 planes (:1330-1339), recomputed from cfa.
__device__ __forceinline__ float dirwts0_at(const float* cfa, int idx) {
  const float delv = fabsf(cfa[idx + TS] - cfa[idx - TS]);
  return eps + fabsf(cfa[idx + 2 * TS] - cfa[idx]) + fabsf(cfa[idx] - cfa[idx - 2 * TS]) + delv;
}
__device__ __forceinline__ float dirwts1_at(const float* cfa, int idx) {
  const float delh = fabsf(cfa[idx + 1] - cfa[idx - 1]);
  return eps + fabsf(cfa[idx + 2] - cfa[idx]) + fabsf(cfa[idx] - cfa[idx - 2]) + delh;
}
__device__ __forceinline__ float delhvsqsum_at(const float* cfa, int idx) {
  const float delh = fabsf(cfa[idx + 1] - cfa[idx - 1]);
  const float delv = fabsf(cfa[idx + TS] - cfa[idx - TS]);
  return SQR(delh) + SQR(delv);
}

// Stage 3 (:1375-1398) after the step has chosen h (the stage-2 value or its
// alternate): the clamp against the site's Gint and its two neighbours along
// the chain direction.  A pure function of h, so both candidates can be
// finished before the chain recurrence decides between them.
__device__ __forceinline__ float s3_finish(float h, float c, float cm, float cp, bool green, float clip_pt) {
  float Gint;
  if (green) {
    Gint = -h + c;
    if (h > 0) {
      if (3.f * h > (Gint + c)) {
        h = -median3(Gint, cm, cp) + c;
      } else {
        const float wt2 = 1.f - 3.f * h / (eps + Gint + c);
        h = wt2 * h + (1.f - wt2) * (-median3(Gint, cm, cp) + c);
      }
    }
  } else {
    Gint = h + c;
    if (h < 0) {
      if (3.f * h < -(Gint + c)) {
        h = median3(Gint, cm, cp) - c;
      } else {
        const float wt2 = 1.f + 3.f * h / (eps + Gint + c);
        h = wt2 * h + (1.f - wt2) * (median3(Gint, cm, cp) - c);
      }
    }
  }
  if (Gint > clip_pt) h = (float)(green ? -1 : 1) * (median3(Gint, cm, cp) - c);
  return h;
}

// Directional variance of three consecutive chain values (:1380-1381).
__device__ __forceinline__ float s3_var(float a, float b, float c) {
  return 3.f * (SQR(a) + SQR(b) + SQR(c)) - SQR(a + b + c);
}

__global__ void __launch_bounds__(AMZ_THREADS, 1) k_amaze(AmazeArgs A) {
  const int v1 = TS, v2 = 2 * TS, v3 = 3 * TS, p1 = -TS + 1, p2 = -2 * TS + 2, p3 = -3 * TS + 3, m1 = TS + 1,
            m2 = 2 * TS + 2, m3 = 3 * TS + 3;
  extern __shared__ __align__(16) float smem[];
  float* hvwt = smem;         // [HALF]
  float* pmwt = smem + HALF;  // [HALF]
  float* cfa = smem + 2 * HALF;  // [TS2], read by nearly every stage
  const int tid = threadIdx.x, nth = blockDim.x;
  const int W = A.W, H = A.H;
  const Slab S = make_slab(A.scratch + (size_t)blockIdx.x * kSlabBytes, cfa);
  __shared__ int s_tile;
  __shared__ int s_doNyq;
  float mg = 0.f;  // max G of this thread's interior outputs

  for (;;) {
    if (tid == 0) s_tile = atomicAdd(A.tile_counter, 1);
    __syncthreads();
    const int tile = A.tile_lo + s_tile;
    if (tile >= A.tile_hi) break;
    const int top = -16 + (tile / A.n_left) * (TS - 32);
    const int left = -16 + (tile % A.n_left) * (TS - 32);
    const int bottom = min(top + TS, H + 16);
    const int right = min(left + TS, W + 16);
    const int rr1 = bottom - top;
    const int cc1 = right - left;
    const int rrmin = (top < 0) ? 16 : 0;
    const int ccmin = (left < 0) ? 16 : 0;
    const int rrmax = (bottom > H) ? H - top : rr1;
    const int ccmax = (right > W) ? W - left : cc1;
    const FDiv fdc(cc1), fd8(cc1 - 8), fd32(cc1 - 32);

    // ---- zero what this tile reads before writing (fresh-buffer semantics)
    for (int i = tid; i < 2 * HALF / 16; i += nth)
      reinterpret_cast<float4*>(S.nyquist)[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    for (int i = tid; i < rr1 * cc1; i += nth) {
      const int rr = fdc.div(i), cc = i - rr * cc1;
      if (rr >= 4 && rr < rr1 - 4 && cc >= 4 && cc < cc1 - 4) continue;
      const int idx = rr * TS + cc;
      S.vcd[idx] = 0.f;
      S.hcd[idx] = 0.f;
      S.vcdalt[idx] = 0.f;
      S.hcdalt[idx] = 0.f;
    }
    if ((rrmin > 0 || rrmax < rr1) && (ccmin > 0 || ccmax < cc1)) {
      // unfilled 16x16 apron corners (:1326)
      for (int i = tid; i < rr1 * cc1; i += nth) {
        const int rr = fdc.div(i), cc = i - rr * cc1;
        const bool rc = (rrmin > 0 && rr < 16) || (rrmax < rr1 && rr >= rrmax);
        const bool cc_ = (ccmin > 0 && cc < 16) || (ccmax < cc1 && cc >= ccmax);
        if (rc && cc_) cfa[rr * TS + cc] = 0.f;
      }
    }
    __syncthreads();

    // ---- fill (:1254-1326); the right apron is written last, wrapping into
    // the next row when ccmax + 16 exceeds the tile width, as the reference's
    // flat buffer does
    const float scale = A.scale;
    for (int i = tid; i < rr1 * cc1; i += nth) {
      const int rr = fdc.div(i), cc = i - rr * cc1;
      int srow = -1, scol = -1;
      if (rr >= rrmin && rr < rrmax && cc >= ccmin && cc < ccmax) {
        srow = rr + top;
        scol = cc + left;
      } else if (rrmin > 0 && rr < 16 && cc >= ccmin && cc < ccmax) {
        srow = min(max(32 - rr + top, 0), H - 1);
        scol = min(max(cc + left, 0), W - 1);
      } else if (rrmax < rr1 && rr >= rrmax && rr < rrmax + 16 && cc >= ccmin && cc < ccmax) {
        srow = min(max(H - (rr - rrmax) - 2, 0), H - 1);
        scol = min(max(left + cc, 0), W - 1);
      } else if (ccmin > 0 && cc < 16 && rr >= rrmin && rr < rrmax) {
        srow = min(max(rr + top, 0), H - 1);
        scol = min(max(32 - cc + left, 0), W - 1);
      } else if (ccmax < cc1 && cc >= ccmax && cc < ccmax + 16 && rr >= rrmin && rr < rrmax) {
        srow = min(max(top + rr, 0), H - 1);
        scol = min(max(W - (cc - ccmax) - 2, 0), W - 1);
      }
      if (srow >= 0) cfa[rr * TS + cc] = raw_at(A, srow, scol) * scale;
    }
    if (ccmax < cc1 && ccmax + 16 > TS) {
      __syncthreads();
      for (int i = tid; i < (rrmax - rrmin) * 16; i += nth) {
        const int rr = rrmin + i / 16, k = i % 16;
        if (ccmax + k < TS || rr + 1 >= TS) continue;
        const int srow = min(max(top + rr, 0), H - 1);
        const int scol = min(max(W - k - 2, 0), W - 1);
        cfa[(rr + 1) * TS + (ccmax + k - TS)] = raw_at(A, srow, scol) * scale;
      }
    }
    __syncthreads();

    // ---- S2 colour differences (:1341-1373); S1 planes recomputed
    for (int i = tid; i < (rr1 - 8) * (cc1 - 8); i += nth) {
      const int q_ = fd8.div(i), rr = 4 + q_, cc = 4 + i - q_ * (cc1 - 8);
      const int idx = rr * TS + cc;
      const int sgn = (fc_rt(A, rr, cc) & 1) ? -1 : 1;
      const float d0m2 = dirwts0_at(cfa, idx - v2), d00 = dirwts0_at(cfa, idx), d0p2 = dirwts0_at(cfa, idx + v2);
      const float d1m2 = dirwts1_at(cfa, idx - 2), d10 = dirwts1_at(cfa, idx), d1p2 = dirwts1_at(cfa, idx + 2);
      const float cru = cfa[idx - v1] * (d0m2 + d00) / (d0m2 * (eps + cfa[idx]) + d00 * (eps + cfa[idx - v2]));
      const float crd = cfa[idx + v1] * (d0p2 + d00) / (d0p2 * (eps + cfa[idx]) + d00 * (eps + cfa[idx + v2]));
      const float crl = cfa[idx - 1] * (d1m2 + d10) / (d1m2 * (eps + cfa[idx]) + d10 * (eps + cfa[idx - 2]));
      const float crr = cfa[idx + 1] * (d1p2 + d10) / (d1p2 * (eps + cfa[idx]) + d10 * (eps + cfa[idx + 2]));
      const float guha = cfa[idx - v1] + xdiv2f(cfa[idx] - cfa[idx - v2]);
      const float gdha = cfa[idx + v1] + xdiv2f(cfa[idx] - cfa[idx + v2]);
      const float glha = cfa[idx - 1] + xdiv2f(cfa[idx] - cfa[idx - 2]);
      const float grha = cfa[idx + 1] + xdiv2f(cfa[idx] - cfa[idx + 2]);
      float guar = fabsf(1.f - cru) < arthresh ? cfa[idx] * cru : guha;
      float gdar = fabsf(1.f - crd) < arthresh ? cfa[idx] * crd : gdha;
      float glar = fabsf(1.f - crl) < arthresh ? cfa[idx] * crl : glha;
      float grar = fabsf(1.f - crr) < arthresh ? cfa[idx] * crr : grha;
      const float d1m1 = dirwts1_at(cfa, idx - 1), d1p1 = dirwts1_at(cfa, idx + 1);
      const float d0m1 = dirwts0_at(cfa, idx - v1), d0p1 = dirwts0_at(cfa, idx + v1);
      const float hwt = d1m1 / (d1m1 + d1p1);
      const float vwt = d0m1 / (d0p1 + d0m1);
      const float Gintvha = vwt * gdha + (1.f - vwt) * guha;
      const float Ginthha = hwt * grha + (1.f - hwt) * glha;
      const float fs = (float)sgn;
      const float va = fs * (Gintvha - cfa[idx]);
      const float ha = fs * (Ginthha - cfa[idx]);
      S.vcdalt[idx] = va;
      S.hcdalt[idx] = ha;
      if (cfa[idx] > A.clip_pt8 || Gintvha > A.clip_pt8 || Ginthha > A.clip_pt8) {
        S.vcd[idx] = va;
        S.hcd[idx] = ha;
        guar = guha;
        gdar = gdha;
        glar = glha;
        grar = grha;
      } else {
        S.vcd[idx] = fs * (vwt * gdar + (1.f - vwt) * guar - cfa[idx]);
        S.hcd[idx] = fs * (hwt * grar + (1.f - hwt) * glar - cfa[idx]);
      }
      S.dgintv[idx] = fminf(SQR(guha - gdha), SQR(guar - gdar));
      S.dginth[idx] = fminf(SQR(glha - grha), SQR(glar - grar));
    }
    __syncthreads();

    // ---- S3 (:1375-1398): hcd chains along rows, vcd chains down columns,
    // each in the reference's scan order.  Every operand of a step except
    // the previous (already updated) site is an original value, so each
    // group of G sites loads its operands together.
    {
      // transposed cfa in the (not yet used) hvwt/pmwt region, so that the
      // row chains of a warp read distinct banks; diagonal order keeps both
      // the reads and the writes of each 32x32 block conflict-free
      float* cfaT = smem;
      {
        const int lane = tid & 31, warp = tid >> 5, nwarp = nth >> 5;
        const int bx = (cc1 + 31) >> 5, by = (rr1 + 31) >> 5;
        for (int b = warp; b < bx * by; b += nwarp) {
          const int r0 = (b / bx) << 5, c0 = (b % bx) << 5;
          const int r = r0 + lane;
#pragma unroll 4
          for (int k = 0; k < 32; k++) {
            const int c = c0 + ((lane + k) & 31);
            if (r < rr1 && c < cc1) cfaT[c * TS + r] = cfa[r * TS + c];
          }
        }
      }
      __syncthreads();
      const int nlh = rr1 - 8, nlv = cc1 - 8;
      const int n_h = 2 * nlh, n_v = 2 * nlv;
      for (int item = tid; item < n_h + n_v; item += nth) {
        const bool horiz = item < n_h;
        const int it = horiz ? item : item - n_h;
        const int nl = horiz ? nlh : nlv;
        // row chains: the two chains of a row on neighbouring lanes (their
        // sites share cache lines); column chains: grouped by the parity of
        // line + start, i.e. by CFA colour, so a warp's lanes take the same
        // branches and read consecutive columns of one row
        int line, par;
        if (horiz) {
          line = 4 + (it >> 1);
          par = it & 1;
        } else {
          const int grp = it >= nl;
          line = 4 + (grp ? it - nl : it);
          par = grp ? 1 - (line & 1) : (line & 1);
        }
        const int stride = horiz ? 2 : v2;      // chain step in the flat tile
        const int len = horiz ? cc1 : rr1;
        float* d = horiz ? S.hcd : S.vcd;
        const float* alt = horiz ? S.hcdalt : S.vcdalt;
        const float* cf = horiz ? cfaT : cfa;   // cf[pos * TS + line] / cf[line + pos * TS]
        const int pos0 = 4 + par;
        if (pos0 >= len - 4) continue;
        const bool green = (fc_rt(A, horiz ? line : pos0, horiz ? pos0 : line) & 1) != 0;
        const int K = (len - 4 - pos0 + 1) / 2;  // sites pos0, pos0 + 2, ... < len - 4
        int idx = horiz ? line * TS + pos0 : pos0 * TS + line;
        int cidx = pos0 * TS + line;  // site in cf (both layouts: position-major)
        float prev = d[idx - stride], altp = alt[idx - stride];
        constexpr int G = 8;
        for (int s0 = 0; s0 < K; s0 += G) {
          const int g = min(G, K - s0);
          float dv[G + 1], av[G + 1];
#pragma unroll
          for (int k = 0; k <= G; k++) {
            dv[k] = k <= g ? d[idx + k * stride] : 0.f;
            av[k] = k <= g ? alt[idx + k * stride] : 0.f;
          }
#pragma unroll
          for (int k = 0; k < G; k++) {
            if (k < g) {
              const int ci = cidx + k * v2;
              const float altvar = s3_var(altp, av[k], av[k + 1]);
              const float h0 = (altvar < s3_var(prev, dv[k], dv[k + 1])) ? av[k] : dv[k];
              const float h = s3_finish(h0, cf[ci], cf[ci - TS], cf[ci + TS], green, A.clip_pt);
              d[idx + k * stride] = h;
              prev = h;
              altp = av[k];
            }
          }
          idx += g * stride;
          cidx += g * v2;
        }
      }
    }
    __syncthreads();
    // cddiffsq at R/B sites (read only there by stage 4/5), half-indexed
    auto rb_count = [&](int a) { return (cc1 - a - a + 1) / 2 + 1; };
    {
      const int per_row = rb_count(4);
      const FDiv fdr(per_row);
      for (int i = tid; i < (rr1 - 8) * per_row; i += nth) {
        const int q_ = fdr.div(i), rr = 4 + q_;
        const int cc = 4 + (fc_rt(A, rr, 2) & 1) + 2 * (i - q_ * per_row);
        if (cc >= cc1 - 4) continue;
        const int idx = rr * TS + cc;
        S.cddiffsq[idx >> 1] = SQR(S.vcd[idx] - S.hcd[idx]);
      }
    }
    if (tid == 0) s_doNyq = 0;
    __syncthreads();

    // ---- S4/5 directional variance + Nyquist test (:1400-1433)
    {
      const int a = 6;
      const int per_row = rb_count(a);
      const FDiv fdr(per_row);
      for (int i = tid; i < (rr1 - 2 * a) * per_row; i += nth) {
        const int q_ = fdr.div(i), rr = a + q_;
        const int cc = a + (fc_rt(A, rr, 2) & 1) + 2 * (i - q_ * per_row);
        if (cc >= cc1 - a) continue;
        const int idx = rr * TS + cc;
        const float* vcd = S.vcd;
        const float* hcd = S.hcd;
        const float uave = vcd[idx] + vcd[idx - v1] + vcd[idx - v2] + vcd[idx - v3];
        const float dave = vcd[idx] + vcd[idx + v1] + vcd[idx + v2] + vcd[idx + v3];
        const float lave = hcd[idx] + hcd[idx - 1] + hcd[idx - 2] + hcd[idx - 3];
        const float rave = hcd[idx] + hcd[idx + 1] + hcd[idx + 2] + hcd[idx + 3];
        const float Dgrbvvaru = SQR(vcd[idx] - uave) + SQR(vcd[idx - v1] - uave) + SQR(vcd[idx - v2] - uave) + SQR(vcd[idx - v3] - uave);
        const float Dgrbvvard = SQR(vcd[idx] - dave) + SQR(vcd[idx + v1] - dave) + SQR(vcd[idx + v2] - dave) + SQR(vcd[idx + v3] - dave);
        const float Dgrbhvarl = SQR(hcd[idx] - lave) + SQR(hcd[idx - 1] - lave) + SQR(hcd[idx - 2] - lave) + SQR(hcd[idx - 3] - lave);
        const float Dgrbhvarr = SQR(hcd[idx] - rave) + SQR(hcd[idx + 1] - rave) + SQR(hcd[idx + 2] - rave) + SQR(hcd[idx + 3] - rave);
        const float d1m1 = dirwts1_at(cfa, idx - 1), d1p1 = dirwts1_at(cfa, idx + 1);
        const float d0m1 = dirwts0_at(cfa, idx - v1), d0p1 = dirwts0_at(cfa, idx + v1);
        const float hwt = d1m1 / (d1m1 + d1p1);
        const float vwt = d0m1 / (d0p1 + d0m1);
        const float vcdvar = epssq + vwt * Dgrbvvard + (1.f - vwt) * Dgrbvvaru;
        const float hcdvar = epssq + hwt * Dgrbhvarr + (1.f - hwt) * Dgrbhvarl;
        const float* dgintv = S.dgintv;
        const float* dginth = S.dginth;
        const float Dgrbvvaru2 = dgintv[idx] + dgintv[idx - v1] + dgintv[idx - v2];
        const float Dgrbvvard2 = dgintv[idx] + dgintv[idx + v1] + dgintv[idx + v2];
        const float Dgrbhvarl2 = dginth[idx] + dginth[idx - 1] + dginth[idx - 2];
        const float Dgrbhvarr2 = dginth[idx] + dginth[idx + 1] + dginth[idx + 2];
        const float vcdvar1 = epssq + vwt * Dgrbvvard2 + (1.f - vwt) * Dgrbvvaru2;
        const float hcdvar1 = epssq + hwt * Dgrbhvarr2 + (1.f - hwt) * Dgrbhvarl2;
        const float varwt = hcdvar / (vcdvar + hcdvar);
        const float diffwt = hcdvar1 / (vcdvar1 + hcdvar1);
        hvwt[idx >> 1] =
            ((0.5f - varwt) * (0.5f - diffwt) > 0.f && fabsf(0.5f - diffwt) < fabsf(0.5f - varwt)) ? varwt : diffwt;
        const float* cdd = S.cddiffsq;  // half-indexed; every tap is an R/B site
        auto dh = [&](int o) { return delhvsqsum_at(cfa, idx + o); };
        const float nt =
            (gaussodd[0] * cdd[idx >> 1] +
             gaussodd[1] * (cdd[(idx - m1) >> 1] + cdd[(idx + p1) >> 1] + cdd[(idx - p1) >> 1] + cdd[(idx + m1) >> 1]) +
             gaussodd[2] * (cdd[(idx - v2) >> 1] + cdd[(idx - 2) >> 1] + cdd[(idx + 2) >> 1] + cdd[(idx + v2) >> 1]) +
             gaussodd[3] * (cdd[(idx - m2) >> 1] + cdd[(idx + p2) >> 1] + cdd[(idx - p2) >> 1] + cdd[(idx + m2) >> 1])) -
            (gaussgrad[0] * dh(0) + gaussgrad[1] * (dh(-v1) + dh(1) + dh(-1) + dh(v1)) +
             gaussgrad[2] * (dh(-m1) + dh(p1) + dh(-p1) + dh(m1)) + gaussgrad[3] * (dh(-v2) + dh(-2) + dh(2) + dh(v2)) +
             gaussgrad[4] * (dh(-v2 - 1) + dh(-v2 + 1) + dh(-TS - 2) + dh(-TS + 2) + dh(TS - 2) + dh(TS + 2) +
                             dh(v2 - 1) + dh(v2 + 1)) +
             gaussgrad[5] * (dh(-m2) + dh(p2) + dh(-p2) + dh(m2)));
        if (nt > 0.f) {
          S.nyquist[idx >> 1] = 1;
          s_doNyq = 1;
        }
      }
    }
    __syncthreads();
    const bool doNyquist = s_doNyq != 0;

    // ---- S6 Nyquist refinement + green (:1435-1481)
    if (doNyquist) {
      const int a = 8;
      const int per_row = rb_count(a);
      const FDiv fdr(per_row);
      for (int i = tid; i < (rr1 - 2 * a) * per_row; i += nth) {
        const int q_ = fdr.div(i), rr = a + q_;
        const int cc = a + (fc_rt(A, rr, 2) & 1) + 2 * (i - q_ * per_row);
        if (cc >= cc1 - a) continue;
        const int idx = rr * TS + cc;
        const unsigned char* nq = S.nyquist;
        const unsigned nqsum = nq[(idx - v2) >> 1] + nq[(idx - m1) >> 1] + nq[(idx + p1) >> 1] + nq[(idx - 2) >> 1] +
                               nq[(idx + 2) >> 1] + nq[(idx - p1) >> 1] + nq[(idx + m1) >> 1] + nq[(idx + v2) >> 1];
        S.nyquist2[idx >> 1] = nqsum > 4 ? 1 : (nqsum < 4 ? 0 : nq[idx >> 1]);
      }
      __syncthreads();
      for (int i = tid; i < (rr1 - 2 * a) * per_row; i += nth) {
        const int q_ = fdr.div(i), rr = a + q_;
        const int cc = a + (fc_rt(A, rr, 2) & 1) + 2 * (i - q_ * per_row);
        if (cc >= cc1 - a) continue;
        const int idx = rr * TS + cc;
        if (!S.nyquist2[idx >> 1]) continue;
        float sumcfa = 0, sumh = 0, sumv = 0, sumsqh = 0, sumsqv = 0, areawt = 0;
        for (int ii = -6; ii < 7; ii += 2)
          for (int jj = -6; jj < 7; jj += 2) {
            const int idx1 = idx + ii * TS + jj;
            if ((idx1 >= 0) && (idx1 < TS * TS) && S.nyquist2[idx1 >> 1]) {
              const float cfatemplate = cfa[idx1];
              sumcfa += cfatemplate;
              sumh += (cfa[idx1 - 1] + cfa[idx1 + 1]);
              sumv += (cfa[idx1 - v1] + cfa[idx1 + v1]);
              sumsqh += SQR(cfatemplate - cfa[idx1 - 1]) + SQR(cfatemplate - cfa[idx1 + 1]);
              sumsqv += SQR(cfatemplate - cfa[idx1 - v1]) + SQR(cfatemplate - cfa[idx1 + v1]);
              areawt += 1;
            }
          }
        sumh = sumcfa - xdiv2f(sumh);
        sumv = sumcfa - xdiv2f(sumv);
        areawt = xdiv2f(areawt);
        const float hcdvar2 = epssq + fabsf(areawt * sumsqh - sumh * sumh);
        const float vcdvar2 = epssq + fabsf(areawt * sumsqv - sumv * sumv);
        hvwt[idx >> 1] = hcdvar2 / (vcdvar2 + hcdvar2);
      }
      __syncthreads();
    }
    // Gauss-Seidel sweep of hvwt in shared memory (row rr reads row rr-1
    // already updated), then the per-site green / Dgrb2 in parallel.
    {
      const int a = 8;
      const int per_row = rb_count(a);
      const FDiv fdr(per_row);
      for (int rr = a; rr < rr1 - a; rr++) {
        for (int k = tid; k < per_row; k += nth) {
          const int cc = a + (fc_rt(A, rr, 2) & 1) + 2 * k;
          if (cc >= cc1 - a) continue;
          const int idx = rr * TS + cc;
          const float hvwtalt =
              0.25f * (hvwt[(idx - m1) >> 1] + hvwt[(idx + p1) >> 1] + hvwt[(idx - p1) >> 1] + hvwt[(idx + m1) >> 1]);
          const float cur = hvwt[idx >> 1];
          hvwt[idx >> 1] = fabsf(0.5f - cur) < fabsf(0.5f - hvwtalt) ? hvwtalt : cur;
        }
        __syncthreads();
      }
      for (int i = tid; i < (rr1 - 2 * a) * per_row; i += nth) {
        const int q_ = fdr.div(i), rr = a + q_;
        const int cc = a + (fc_rt(A, rr, 2) & 1) + 2 * (i - q_ * per_row);
        if (cc >= cc1 - a) continue;
        const int idx = rr * TS + cc;
        const float hv = hvwt[idx >> 1];
        const float d0 = hv * S.vcd[idx] + (1.f - hv) * S.hcd[idx];
        S.Dgrb0[idx >> 1] = d0;
        const float g = cfa[idx] + d0;
        S.rgbg[idx >> 1] = g;
        const bool nq2 = S.nyquist2[idx >> 1] != 0;
        // horizontal / vertical neighbours are G sites: their green is cfa
        S.Dgrb2h[idx >> 1] = nq2 ? SQR(g - xdiv2f(cfa[idx - 1] + cfa[idx + 1])) : 0.f;
        S.Dgrb2v[idx >> 1] = nq2 ? SQR(g - xdiv2f(cfa[idx - v1] + cfa[idx + v1])) : 0.f;
      }
      __syncthreads();
    }
    if (doNyquist) {
      const int a = 8;
      const int per_row = rb_count(a);
      const FDiv fdr(per_row);
      const float* D2h = S.Dgrb2h;
      const float* D2v = S.Dgrb2v;
      for (int i = tid; i < (rr1 - 2 * a) * per_row; i += nth) {
        const int q_ = fdr.div(i), rr = a + q_;
        const int cc = a + (fc_rt(A, rr, 2) & 1) + 2 * (i - q_ * per_row);
        if (cc >= cc1 - a) continue;
        const int idx = rr * TS + cc;
        if (!S.nyquist2[idx >> 1]) continue;
        const float gvarh =
            epssq + (gquinc[0] * D2h[idx >> 1] +
                     gquinc[1] * (D2h[(idx - m1) >> 1] + D2h[(idx + p1) >> 1] + D2h[(idx - p1) >> 1] + D2h[(idx + m1) >> 1]) +
                     gquinc[2] * (D2h[(idx - v2) >> 1] + D2h[(idx - 2) >> 1] + D2h[(idx + 2) >> 1] + D2h[(idx + v2) >> 1]) +
                     gquinc[3] * (D2h[(idx - m2) >> 1] + D2h[(idx + p2) >> 1] + D2h[(idx - p2) >> 1] + D2h[(idx + m2) >> 1]));
        const float gvarv =
            epssq + (gquinc[0] * D2v[idx >> 1] +
                     gquinc[1] * (D2v[(idx - m1) >> 1] + D2v[(idx + p1) >> 1] + D2v[(idx - p1) >> 1] + D2v[(idx + m1) >> 1]) +
                     gquinc[2] * (D2v[(idx - v2) >> 1] + D2v[(idx - 2) >> 1] + D2v[(idx + 2) >> 1] + D2v[(idx + v2) >> 1]) +
                     gquinc[3] * (D2v[(idx - m2) >> 1] + D2v[(idx + p2) >> 1] + D2v[(idx - p2) >> 1] + D2v[(idx + m2) >> 1]));
        const float d0 = (S.hcd[idx] * gvarv + S.vcd[idx] * gvarh) / (gvarv + gvarh);
        S.Dgrb0[idx >> 1] = d0;
        S.rgbg[idx >> 1] = cfa[idx] + d0;
      }
      __syncthreads();
    }

    // ---- S7 R/B gradients (:1483-1502)
    const int per7 = (cc1 - 12 + 1) / 2;
    const FDiv fd7(per7);
    for (int i = tid; i < (rr1 - 12) * per7; i += nth) {
      const int q_ = fd7.div(i);
      const int rr = 6 + q_;
      const int cc = 6 + 2 * (i - q_ * per7);
      const int idx = rr * TS + cc;
      if ((fc_rt(A, rr, 2) & 1) == 0) {
        S.delp[idx >> 1] = fabsf(cfa[idx + p1] - cfa[idx - p1]);
        S.delm[idx >> 1] = fabsf(cfa[idx + m1] - cfa[idx - m1]);
        S.Dq1p[idx >> 1] = SQR(cfa[idx + 1] - cfa[idx + 1 - p1]) + SQR(cfa[idx + 1] - cfa[idx + 1 + p1]);
        S.Dq1m[idx >> 1] = SQR(cfa[idx + 1] - cfa[idx + 1 - m1]) + SQR(cfa[idx + 1] - cfa[idx + 1 + m1]);
      } else {
        S.Dq1p[idx >> 1] = SQR(cfa[idx] - cfa[idx - p1]) + SQR(cfa[idx] - cfa[idx + p1]);
        S.Dq1m[idx >> 1] = SQR(cfa[idx] - cfa[idx - m1]) + SQR(cfa[idx] - cfa[idx + m1]);
        S.delp[idx >> 1] = fabsf(cfa[idx + 1 + p1] - cfa[idx + 1 - p1]);
        S.delm[idx >> 1] = fabsf(cfa[idx + 1 + m1] - cfa[idx + 1 - m1]);
      }
    }
    __syncthreads();

    // ---- S8 diagonal R/B interpolation (:1504-1532); pmwt into SMEM
    {
      const int a = 8;
      const int per_row = rb_count(a);
      const FDiv fdr(per_row);
      const float* delp = S.delp;
      const float* delm = S.delm;
      const float* Dq1m = S.Dq1m;
      const float* Dq1p = S.Dq1p;
      for (int i = tid; i < (rr1 - 2 * a) * per_row; i += nth) {
        const int q_ = fdr.div(i), rr = a + q_;
        const int cc = a + (fc_rt(A, rr, 2) & 1) + 2 * (i - q_ * per_row);
        if (cc >= cc1 - a) continue;
        const int idx = rr * TS + cc, idx1 = idx >> 1;
        const float crse = xmul2f(cfa[idx + m1]) / (eps + cfa[idx] + cfa[idx + m2]);
        const float crnw = xmul2f(cfa[idx - m1]) / (eps + cfa[idx] + cfa[idx - m2]);
        const float crne = xmul2f(cfa[idx + p1]) / (eps + cfa[idx] + cfa[idx + p2]);
        const float crsw = xmul2f(cfa[idx - p1]) / (eps + cfa[idx] + cfa[idx - p2]);
        const float rbse = fabsf(1.f - crse) < arthresh ? cfa[idx] * crse : (cfa[idx + m1]) + xdiv2f(cfa[idx] - cfa[idx + m2]);
        const float rbnw = fabsf(1.f - crnw) < arthresh ? cfa[idx] * crnw : (cfa[idx - m1]) + xdiv2f(cfa[idx] - cfa[idx - m2]);
        const float rbne = fabsf(1.f - crne) < arthresh ? cfa[idx] * crne : (cfa[idx + p1]) + xdiv2f(cfa[idx] - cfa[idx + p2]);
        const float rbsw = fabsf(1.f - crsw) < arthresh ? cfa[idx] * crsw : (cfa[idx - p1]) + xdiv2f(cfa[idx] - cfa[idx - p2]);
        const float wtse = eps + delm[idx1] + delm[(idx + m1) >> 1] + delm[(idx + m2) >> 1];
        const float wtnw = eps + delm[idx1] + delm[(idx - m1) >> 1] + delm[(idx - m2) >> 1];
        const float wtne = eps + delp[idx1] + delp[(idx + p1) >> 1] + delp[(idx + p2) >> 1];
        const float wtsw = eps + delp[idx1] + delp[(idx - p1) >> 1] + delp[(idx - p2) >> 1];
        float rbm = (wtse * rbnw + wtnw * rbse) / (wtse + wtnw);
        float rbp = (wtne * rbsw + wtsw * rbne) / (wtne + wtsw);
        if (rbp < cfa[idx]) {
          if (xmul2f(rbp) < cfa[idx]) {
            rbp = median3(rbp, cfa[idx - p1], cfa[idx + p1]);
          } else {
            const float pwt = xmul2f(cfa[idx] - rbp) / (eps + rbp + cfa[idx]);
            rbp = pwt * rbp + (1.f - pwt) * median3(rbp, cfa[idx - p1], cfa[idx + p1]);
          }
        }
        if (rbm < cfa[idx]) {
          if (xmul2f(rbm) < cfa[idx]) {
            rbm = median3(rbm, cfa[idx - m1], cfa[idx + m1]);
          } else {
            const float mwt = xmul2f(cfa[idx] - rbm) / (eps + rbm + cfa[idx]);
            rbm = mwt * rbm + (1.f - mwt) * median3(rbm, cfa[idx - m1], cfa[idx + m1]);
          }
        }
        if (rbp > A.clip_pt) rbp = median3(rbp, cfa[idx - p1], cfa[idx + p1]);
        if (rbm > A.clip_pt) rbm = median3(rbm, cfa[idx - m1], cfa[idx + m1]);
        S.rbm[idx1] = rbm;
        S.rbp[idx1] = rbp;
        const float rbvarm =
            epssq + (gausseven[0] * (Dq1m[(idx - v1) >> 1] + Dq1m[(idx - 1) >> 1] + Dq1m[(idx + 1) >> 1] + Dq1m[(idx + v1) >> 1]) +
                     gausseven[1] * (Dq1m[(idx - v2 - 1) >> 1] + Dq1m[(idx - v2 + 1) >> 1] + Dq1m[(idx - 2 - v1) >> 1] +
                                     Dq1m[(idx + 2 - v1) >> 1] + Dq1m[(idx - 2 + v1) >> 1] + Dq1m[(idx + 2 + v1) >> 1] +
                                     Dq1m[(idx + v2 - 1) >> 1] + Dq1m[(idx + v2 + 1) >> 1]));
        const float rbvarp =
            epssq + (gausseven[0] * (Dq1p[(idx - v1) >> 1] + Dq1p[(idx - 1) >> 1] + Dq1p[(idx + 1) >> 1] + Dq1p[(idx + v1) >> 1]) +
                     gausseven[1] * (Dq1p[(idx - v2 - 1) >> 1] + Dq1p[(idx - v2 + 1) >> 1] + Dq1p[(idx - 2 - v1) >> 1] +
                                     Dq1p[(idx + 2 - v1) >> 1] + Dq1p[(idx - 2 + v1) >> 1] + Dq1p[(idx + 2 + v1) >> 1] +
                                     Dq1p[(idx + v2 - 1) >> 1] + Dq1p[(idx + v2 + 1) >> 1]));
        pmwt[idx1] = rbvarm / (rbvarp + rbvarm);
      }
    }
    __syncthreads();

    // ---- S9 (:1534-1592): Gauss-Seidel pmwt sweep in SMEM, then rbint
    {
      const int a = 10;
      const int per_row = rb_count(a);
      const FDiv fdr(per_row);
      for (int rr = a; rr < rr1 - a; rr++) {
        for (int k = tid; k < per_row; k += nth) {
          const int cc = a + (fc_rt(A, rr, 2) & 1) + 2 * k;
          if (cc >= cc1 - a) continue;
          const int idx = rr * TS + cc, idx1 = idx >> 1;
          const float pmwtalt =
              0.25f * (pmwt[(idx - m1) >> 1] + pmwt[(idx + p1) >> 1] + pmwt[(idx - p1) >> 1] + pmwt[(idx + m1) >> 1]);
          const float pw = pmwt[idx1];
          if (fabsf(0.5f - pw) < fabsf(0.5f - pmwtalt)) pmwt[idx1] = pmwtalt;
        }
        __syncthreads();
      }
      for (int i = tid; i < (rr1 - 2 * a) * per_row; i += nth) {
        const int q_ = fdr.div(i), rr = a + q_;
        const int cc = a + (fc_rt(A, rr, 2) & 1) + 2 * (i - q_ * per_row);
        if (cc >= cc1 - a) continue;
        const int idx = rr * TS + cc, idx1 = idx >> 1;
        const float pw = pmwt[idx1];
        S.rbint[idx1] = xdiv2f(cfa[idx] + S.rbm[idx1] * (1.f - pw) + S.rbp[idx1] * pw);
      }
    }
    // Dgrb1 starts as zeros (its unwritten cells are read by the diagonal
    // step); it occupies Dgrb2h's half plane, dead after stage 6
    for (int i = tid; i < HALF / 4; i += nth) reinterpret_cast<float4*>(S.Dgrb1)[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    __syncthreads();
    // dirwts1 as the reference reads it after pmwt was stored over it
    // (half index k of pmwt == float offset k of dirwts1).
    auto pm_written = [&](int p) -> bool {
      if (p < 0 || p >= HALF) return false;
      const int r2 = (2 * p) / TS;
      const int c0 = (2 * p) % TS;
      const int crb = c0 + (int)(fc_rt(A, r2, 2) & 1);
      return r2 >= 8 && r2 < rr1 - 8 && crb >= 8 && crb < cc1 - 8;
    };
    auto dirwts1_eff = [&](int p) -> float { return pm_written(p) ? pmwt[p] : dirwts1_at(cfa, p); };
    {
      const int a = 12;
      const int per_row = rb_count(a);
      const FDiv fdr(per_row);
      const float* rbint = S.rbint;
      for (int i = tid; i < (rr1 - 2 * a) * per_row; i += nth) {
        const int q_ = fdr.div(i), rr = a + q_;
        const int cc = a + (fc_rt(A, rr, 2) & 1) + 2 * (i - q_ * per_row);
        if (cc >= cc1 - a) continue;
        const int idx = rr * TS + cc, idx1 = idx >> 1;
        if (fabsf(0.5f - pmwt[idx1]) >= fabsf(0.5f - hvwt[idx1])) continue;
        const float cru = xmul2f(cfa[idx - v1]) / (eps + rbint[idx1] + rbint[idx1 - v1]);
        const float crd = xmul2f(cfa[idx + v1]) / (eps + rbint[idx1] + rbint[idx1 + v1]);
        const float crl = xmul2f(cfa[idx - 1]) / (eps + rbint[idx1] + rbint[idx1 - 1]);
        const float crr = xmul2f(cfa[idx + 1]) / (eps + rbint[idx1] + rbint[idx1 + 1]);
        const float gu = fabsf(1.f - cru) < arthresh ? rbint[idx1] * cru : cfa[idx - v1] + xdiv2f(rbint[idx1] - rbint[idx1 - v1]);
        const float gd = fabsf(1.f - crd) < arthresh ? rbint[idx1] * crd : cfa[idx + v1] + xdiv2f(rbint[idx1] - rbint[idx1 + v1]);
        const float gl = fabsf(1.f - crl) < arthresh ? rbint[idx1] * crl : cfa[idx - 1] + xdiv2f(rbint[idx1] - rbint[idx1 - 1]);
        const float gr = fabsf(1.f - crr) < arthresh ? rbint[idx1] * crr : cfa[idx + 1] + xdiv2f(rbint[idx1] - rbint[idx1 + 1]);
        const float d0m = dirwts0_at(cfa, idx - v1), d0p = dirwts0_at(cfa, idx + v1);
        float Gintv = (d0m * gd + d0p * gu) / (d0p + d0m);
        const float d1m = dirwts1_eff(idx - 1), d1p = dirwts1_eff(idx + 1);
        float Ginth = (d1m * gr + d1p * gl) / (d1m + d1p);
        if (Gintv < rbint[idx1]) {
          if (xmul2f(Gintv) < rbint[idx1]) {
            Gintv = median3(Gintv, cfa[idx - v1], cfa[idx + v1]);
          } else {
            const float vwt2 = xmul2f(rbint[idx1] - Gintv) / (eps + Gintv + rbint[idx1]);
            Gintv = vwt2 * Gintv + (1.f - vwt2) * median3(Gintv, cfa[idx - v1], cfa[idx + v1]);
          }
        }
        if (Ginth < rbint[idx1]) {
          if (xmul2f(Ginth) < rbint[idx1]) {
            Ginth = median3(Ginth, cfa[idx - 1], cfa[idx + 1]);
          } else {
            const float hwt2 = xmul2f(rbint[idx1] - Ginth) / (eps + Ginth + rbint[idx1]);
            Ginth = hwt2 * Ginth + (1.f - hwt2) * median3(Ginth, cfa[idx - 1], cfa[idx + 1]);
          }
        }
        if (Ginth > A.clip_pt) Ginth = median3(Ginth, cfa[idx - 1], cfa[idx + 1]);
        if (Gintv > A.clip_pt) Gintv = median3(Gintv, cfa[idx - v1], cfa[idx + v1]);
        const float hv = hvwt[idx1];
        const float g = Ginth * (1.f - hv) + Gintv * hv;
        S.rgbg[idx1] = g;
        S.Dgrb0[idx1] = g - cfa[idx];
      }
    }
    __syncthreads();

    // Dgrb1 initialisation (:1563-1569): move the B-row values to Dgrb1.
    {
      const int r0 = 13 - A.ey;
      const int nrows = (rr1 - 12 - r0 + 1) / 2;
      const int k0 = 13 - A.ex;
      for (int i = tid; i < nrows * TSH; i += nth) {
        const int rr = r0 + 2 * (i / TSH);
        if (rr >= rr1 - 12) continue;
        const int lo = (rr * TS + k0) >> 1, hi = (rr * TS + cc1 - 12) >> 1;
        const int idx1 = lo + (i % TSH);
        if (idx1 >= hi) continue;
        S.Dgrb1[idx1] = S.Dgrb0[idx1];
        S.Dgrb0[idx1] = 0;
      }
    }
    __syncthreads();
    // Diagonal chroma interpolation (:1570-1587).
    {
      const int a = 14;
      const int per_row = rb_count(a);
      const FDiv fdr(per_row);
      for (int i = tid; i < (rr1 - 2 * a) * per_row; i += nth) {
        const int q_ = fdr.div(i), rr = a + q_;
        const int cc = a + (fc_rt(A, rr, 2) & 1) + 2 * (i - q_ * per_row);
        if (cc >= cc1 - a) continue;
        const int idx = rr * TS + cc;
        const int c = 1 - (int)fc_rt(A, rr, cc) / 2;
        float* D = c ? S.Dgrb1 : S.Dgrb0;
        const float wtnw = 1.f / (eps + fabsf(D[(idx - m1) >> 1] - D[(idx + m1) >> 1]) + fabsf(D[(idx - m1) >> 1] - D[(idx - m3) >> 1]) +
                                  fabsf(D[(idx + m1) >> 1] - D[(idx - m3) >> 1]));
        const float wtne = 1.f / (eps + fabsf(D[(idx + p1) >> 1] - D[(idx - p1) >> 1]) + fabsf(D[(idx + p1) >> 1] - D[(idx + p3) >> 1]) +
                                  fabsf(D[(idx - p1) >> 1] - D[(idx + p3) >> 1]));
        const float wtsw = 1.f / (eps + fabsf(D[(idx - p1) >> 1] - D[(idx + p1) >> 1]) + fabsf(D[(idx - p1) >> 1] - D[(idx + m3) >> 1]) +
                                  fabsf(D[(idx + p1) >> 1] - D[(idx - p3) >> 1]));
        const float wtse = 1.f / (eps + fabsf(D[(idx + m1) >> 1] - D[(idx - m1) >> 1]) + fabsf(D[(idx + m1) >> 1] - D[(idx - p3) >> 1]) +
                                  fabsf(D[(idx - m1) >> 1] - D[(idx + m3) >> 1]));
        D[idx >> 1] =
            (wtnw * (1.325f * D[(idx - m1) >> 1] - 0.175f * D[(idx - m3) >> 1] - 0.075f * (D[(idx - m1 - 2) >> 1] + D[(idx - m1 - v2) >> 1])) +
             wtne * (1.325f * D[(idx + p1) >> 1] - 0.175f * D[(idx + p3) >> 1] - 0.075f * (D[(idx + p1 + 2) >> 1] + D[(idx + p1 + v2) >> 1])) +
             wtsw * (1.325f * D[(idx - p1) >> 1] - 0.175f * D[(idx - p3) >> 1] - 0.075f * (D[(idx - p1 - 2) >> 1] + D[(idx - p1 - v2) >> 1])) +
             wtse * (1.325f * D[(idx + m1) >> 1] - 0.175f * D[(idx + m3) >> 1] - 0.075f * (D[(idx + m1 + 2) >> 1] + D[(idx + m1 + v2) >> 1]))) /
            (wtnw + wtne + wtsw + wtse);
      }
    }
    __syncthreads();

    // ---- S10 output (:1594-1625)
    for (int i = tid; i < (rr1 - 32) * (cc1 - 32); i += nth) {
      const int q_ = fd32.div(i), rr = 16 + q_, cc = 16 + i - q_ * (cc1 - 32);
      const int row = rr + top, col = cc + left;
      if (row < 0 || row >= H || col < 0 || col >= W) continue;
      const int t = rr * TS + cc;
      float r, g, b;
      const float* D0 = S.Dgrb0;
      const float* D1 = S.Dgrb1;
      if (fc_rt(A, row, col) == 1) {
        g = cfa[t];
        const float wsum_inv =
            1.0f / (hvwt[(t - v1) >> 1] + 2.f - hvwt[(t + 1) >> 1] - hvwt[(t - 1) >> 1] + hvwt[(t + v1) >> 1]);
        const float r_diff = (hvwt[(t - v1) >> 1] * D0[(t - v1) >> 1] + (1.f - hvwt[(t + 1) >> 1]) * D0[(t + 1) >> 1] +
                              (1.f - hvwt[(t - 1) >> 1]) * D0[(t - 1) >> 1] + hvwt[(t + v1) >> 1] * D0[(t + v1) >> 1]) *
                             wsum_inv;
        const float b_diff = (hvwt[(t - v1) >> 1] * D1[(t - v1) >> 1] + (1.f - hvwt[(t + 1) >> 1]) * D1[(t + 1) >> 1] +
                              (1.f - hvwt[(t - 1) >> 1]) * D1[(t - 1) >> 1] + hvwt[(t + v1) >> 1] * D1[(t + v1) >> 1]) *
                             wsum_inv;
        r = g - r_diff;
        b = g - b_diff;
      } else {
        g = S.rgbg[t >> 1];
        r = g - D0[t >> 1];
        b = g - D1[t >> 1];
      }
      // streaming stores: the output is not re-read by this kernel, so it
      // should not evict the slab planes from L2
      float* o = A.rgb + ((size_t)row * W + col) * 3;
      __stcs(o + 0, fmaxf(0.f, r));
      __stcs(o + 1, fmaxf(0.f, g));
      __stcs(o + 2, fmaxf(0.f, b));
      if (row >= 4 && row < H - 4 && col >= 4 && col < W - 4) mg = fmaxf(mg, fmaxf(0.f, g));
    }
    __syncthreads();
  }
  // every thread leaves the tile loop together (s_tile is shared)
  if (A.max_g) {
    mg = warp_max(mg);
    if ((tid & 31) == 0) atomic_max_float(A.max_g, mg);
  }
}

// LibRaw-style border interpolation (core/cpu_accelerator.cpp:2984-3028):
// only pixels within `border` of the frame; non-native channels become the
// mean of that colour's samples in the clipped 3x3 neighbourhood.
__global__ void k_border_interp(float* rgb, int W, int H, uint32_t filters, int border, float* max_g) {
  float mg = 0.f;  // max of the final G of this thread's border pixels
  // enumerate only border pixels: top/bottom bands then left/right bands
  const int band = border;
  const long long n_tb = 2LL * band * W;
  const long long n_lr = 2LL * band * (H - 2 * band > 0 ? H - 2 * band : 0);
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n_tb + n_lr;
       k += (long long)gridDim.x * blockDim.x) {
    int row, col;
    if (k < n_tb) {
      const int b = (int)(k / W);
      col = (int)(k % W);
      row = b < band ? b : H - 2 * band + b;
    } else {
      const long long q = k - n_tb;
      const int b = (int)(q % (2 * band));
      row = band + (int)(q / (2 * band));
      col = b < band ? b : W - 2 * band + b;
    }
    if (row < 0 || row >= H || col < 0 || col >= W) continue;
    if (col >= border && col < W - border && row >= border && row < H - border) continue;
    float sum[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int y = row > 0 ? row - 1 : 0; y < row + 2 && y < H; y++)
      for (int x = col > 0 ? col - 1 : 0; x < col + 2 && x < W; x++) {
        const unsigned f = fcol3((unsigned)y, (unsigned)x, filters);
        sum[f] += rgb[((size_t)y * W + x) * 3 + f];
        sum[f + 4]++;
      }
    const unsigned f = fcol3((unsigned)row, (unsigned)col, filters);
    for (unsigned c = 0; c < 3; c++)
      if (c != f && sum[c + 4] > 0) rgb[((size_t)row * W + col) * 3 + c] = sum[c] / sum[c + 4];
    if (max_g) {
      // G as this pass leaves it: a G site keeps its own sample, an R/B site
      // takes the neighbours' mean when it has G neighbours
      const float gv = (f != 1 && sum[5] > 0) ? sum[1] / sum[5] : rgb[((size_t)row * W + col) * 3 + 1];
      mg = fmaxf(mg, fmaxf(0.f, gv));
    }
  }
  if (max_g) {
    mg = warp_max(mg);
    if ((threadIdx.x & 31) == 0) atomic_max_float(max_g, mg);
  }
}

}  // namespace

size_t ws_bytes_amaze(size_t w, size_t h) {
  (void)w;
  (void)h;
  return 160u * kSlabBytes + 4096;
}

namespace {

AmazeArgs amaze_args(const float* raw, int cstride, float* rgb, size_t w, size_t h, uint32_t filters,
                     const float cam_mul[4], float maximum_value) {
  AmazeArgs A;
  A.raw = raw;
  A.cstride = cstride;
  A.rgb = rgb;
  A.W = (int)w;
  A.H = (int)h;
  A.filters = filters;
  // core/cpu_accelerator.cpp:1183-1206
  const float max_mul = std::max(cam_mul[0], cam_mul[2]);
  const float min_mul = std::min(cam_mul[0], cam_mul[2]);
  const float initialGain = (min_mul > 1e-6f) ? (max_mul / min_mul) : 1.0f;
  A.clip_pt = 1.0f / initialGain;
  A.clip_pt8 = 0.8f / initialGain;
  for (int r = 0; r < 2; r++)
    for (int q = 0; q < 2; q++) A.cfarray[r][q] = fcol3((unsigned)r, (unsigned)q, filters);
  A.cfpack = 0;
  for (int r = 0; r < 2; r++)
    for (int q = 0; q < 2; q++) A.cfpack |= A.cfarray[r][q] << (2 * (r * 2 + q));
  if (A.cfarray[0][0] == 1) {
    if (A.cfarray[0][1] == 0) { A.ey = 0; A.ex = 1; } else { A.ey = 1; A.ex = 0; }
  } else {
    if (A.cfarray[0][0] == 0) { A.ey = 0; A.ex = 0; } else { A.ey = 1; A.ex = 1; }
  }
  A.scale = 1.0f / maximum_value;
  // tile grid of :1243-1246
  A.n_top = 0;
  for (int top = -16; top < (int)h; top += TS - 32) A.n_top++;
  A.n_left = 0;
  for (int left = -16; left < (int)w; left += TS - 32) A.n_left++;
  A.tile_lo = 0;
  A.tile_hi = A.n_top * A.n_left;
  A.scratch = nullptr;
  A.tile_counter = nullptr;
  A.max_g = nullptr;
  return A;
}

// One persistent launch over the tile rows [row_lo, row_hi) of the grid.
lre_status launch_amaze_rows(Context* c, AmazeArgs A, int row_lo, int row_hi) {
  A.tile_lo = row_lo * A.n_left;
  A.tile_hi = row_hi * A.n_left;
  const int tiles = A.tile_hi - A.tile_lo;
  if (tiles <= 0) return LRE_OK;
  int nblk = std::min(tiles, c->sm_count);
  if (nblk < 1) nblk = 1;
  const size_t mark = c->ws.used();
  A.scratch = reinterpret_cast<unsigned char*>(c->ws.take((size_t)nblk * kSlabBytes));
  A.tile_counter = reinterpret_cast<int*>(c->ws.take(256));
  if (!A.scratch || !A.tile_counter) return fail(c, LRE_ERR_OUT_OF_MEMORY, "demosaic_bayer_amaze: workspace too small");
  LRE_CUDA_TRY(c, cudaMemsetAsync(A.tile_counter, 0, sizeof(int), c->stream));
  LRE_CUDA_TRY(c, cudaFuncSetAttribute(k_amaze, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemBytes));
  k_amaze<<<nblk, AMZ_THREADS, kSmemBytes, c->stream>>>(A);
  count_launch(c);
  c->ws.rewind(mark);
  return check_launch(c, "demosaic_bayer_amaze");
}

}  // namespace

lre_status launch_amaze(Context* c, const float* raw, int cstride, float* rgb, size_t w, size_t h, uint32_t filters,
                        const float cam_mul[4], float maximum_value, float* max_g) {
  AmazeArgs A = amaze_args(raw, cstride, rgb, w, h, filters, cam_mul, maximum_value);
  A.max_g = max_g;
  if (max_g) LRE_CUDA_TRY(c, cudaMemsetAsync(max_g, 0, sizeof(float), c->stream));
  LRE_TRY(launch_amaze_rows(c, A, 0, A.n_top));
  return launch_border_interp(c, rgb, w, h, filters, 4, max_g);
}

lre_status launch_amaze_from_host(Context* c, const float* h_mosaic, float* d_mosaic, float* rgb, size_t w,
                                  size_t h, uint32_t filters, const float cam_mul[4], float maximum_value,
                                  cudaStream_t copy_stream, cudaEvent_t* events, int n_events, float* max_g) {
  AmazeArgs A = amaze_args(d_mosaic, 1, rgb, w, h, filters, cam_mul, maximum_value);
  A.max_g = max_g;
  if (max_g) LRE_CUDA_TRY(c, cudaMemsetAsync(max_g, 0, sizeof(float), c->stream));
  const int bands = std::max(1, std::min(n_events, A.n_top / 4));
  size_t copied = 0;  // mosaic rows already queued for upload
  for (int b = 0; b < bands; b++) {
    const int row_lo = A.n_top * b / bands, row_hi = A.n_top * (b + 1) / bands;
    // a tile row k reads mosaic rows [128k - 16, 128k + 144) (clamped)
    const size_t need = std::min(h, (size_t)std::max(0, -16 + (row_hi - 1) * (TS - 32) + TS));
    if (need > copied) {
      LRE_TRY(copy_h2d(c, d_mosaic + copied * w, h_mosaic + copied * w, (need - copied) * w * sizeof(float),
                       copy_stream));
      copied = need;
    }
    LRE_CUDA_TRY(c, cudaEventRecord(events[b], copy_stream));
    LRE_CUDA_TRY(c, cudaStreamWaitEvent(c->stream, events[b], 0));
    LRE_TRY(launch_amaze_rows(c, A, row_lo, row_hi));
  }
  if (copied < h) {  // rows no tile reads still belong to the resident mosaic
    LRE_TRY(copy_h2d(c, d_mosaic + copied * w, h_mosaic + copied * w, (h - copied) * w * sizeof(float),
                     copy_stream));
    LRE_CUDA_TRY(c, cudaEventRecord(events[bands - 1], copy_stream));
    LRE_CUDA_TRY(c, cudaStreamWaitEvent(c->stream, events[bands - 1], 0));
  }
  return launch_border_interp(c, rgb, w, h, filters, 4, max_g);
}

lre_status launch_border_interp(Context* c, float* rgb, size_t w, size_t h, uint32_t filters, int band, float* max_g) {
  const long long nb = 2LL * band * (long long)w + 2LL * band * (long long)(h > (size_t)(2 * band) ? h - 2 * band : 0);
  k_border_interp<<<grid_for((size_t)nb, 256, c->sm_count * 2), 256, 0, c->stream>>>(rgb, (int)w, (int)h, filters, band,
                                                                                     max_g);
  count_launch(c);
  return check_launch(c, "border_interpolate");
}

}  // namespace lre
