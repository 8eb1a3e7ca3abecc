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
// This kernel therefore runs the reference's tiles one CTA per tile, stage by
// stage, with the sequential chains on individual threads and the
// Gauss-Seidel sweeps as row-synchronous wavefronts.  Per-tile planes live in
// a per-CTA global scratch slab (they do not fit in shared memory: ~20 planes
// of 160x160).  Scratch positions the reference reads without writing in the
// same tile hold zeros (a fresh, zero-initialised buffer), and the unfilled
// 16x16 apron corners at the image corners are zero as well.
#include "common.cuh"
#include "lre_internal.h"

namespace lre {

namespace {

constexpr int TS = 160;
constexpr int TSH = TS / 2;
constexpr int TS2 = TS * TS;
constexpr int AMZ_THREADS = 512;

constexpr float eps = 1e-5f;
constexpr float epssq = 1e-10f;
constexpr float arthresh = 0.75f;
constexpr float nyqthresh = 0.5f;

__device__ __forceinline__ float SQR(float x) { return x * x; }
__device__ __forceinline__ float xmul2f(float x) { return x + x; }
__device__ __forceinline__ float xdiv2f(float x) { return x * 0.5f; }

// Scratch slab layout (floats unless noted).
struct Slab {
  float *cfa, *rgbgreen, *delhvsqsum, *dirwts0, *dirwts1, *vcd, *hcd, *vcdalt, *hcdalt, *cddiffsq, *dgintv, *dginth;
  float *hvwt, *nyqutest, *Dgrb0, *Dgrb1, *Dgrb2h, *Dgrb2v, *delp, *delm, *Dgrbsq1p, *Dgrbsq1m, *rbm, *rbp, *pmwt, *rbint;
  unsigned char *nyquist, *nyquist2;
};
constexpr size_t kFullPlanes = 12;
constexpr size_t kHalfPlanes = 14;
constexpr size_t kSlabBytes = (kFullPlanes * TS2 + kHalfPlanes * TS * TSH) * 4 + 2 * TS * TSH + 256;

__device__ Slab make_slab(unsigned char* base) {
  Slab s;
  float* f = reinterpret_cast<float*>(base);
  float** full[kFullPlanes] = {&s.cfa, &s.rgbgreen, &s.delhvsqsum, &s.dirwts0, &s.dirwts1, &s.vcd,
                               &s.hcd, &s.vcdalt,   &s.hcdalt,     &s.cddiffsq, &s.dgintv, &s.dginth};
  for (size_t i = 0; i < kFullPlanes; i++) *full[i] = f + i * TS2;
  f += kFullPlanes * TS2;
  float** half[kHalfPlanes] = {&s.hvwt, &s.nyqutest, &s.Dgrb0,    &s.Dgrb1,    &s.Dgrb2h, &s.Dgrb2v, &s.delp,
                               &s.delm, &s.Dgrbsq1p, &s.Dgrbsq1m, &s.rbm,      &s.rbp,    &s.pmwt,   &s.rbint};
  for (size_t i = 0; i < kHalfPlanes; i++) *half[i] = f + i * TS * TSH;
  f += kHalfPlanes * TS * TSH;
  s.nyquist = reinterpret_cast<unsigned char*>(f);
  s.nyquist2 = s.nyquist + TS * TSH;
  return s;
}

struct AmazeArgs {
  const float* raw;
  int cstride;  // 1: dense CFA mosaic, 3: sparse (H,W,3) raw buffer
  float* rgb;
  int W, H;
  uint32_t filters;
  unsigned cfarray[2][2];
  int ex, ey;
  float clip_pt, clip_pt8, scale;
  int n_top, n_left;
  unsigned char* scratch;
  int* tile_counter;
};

__device__ __forceinline__ unsigned fc_rt(const AmazeArgs& a, int r, int c) { return a.cfarray[r & 1][c & 1]; }

__device__ __forceinline__ float raw_at(const AmazeArgs& a, int row, int col) {
  size_t i = (size_t)row * a.W + col;
  if (a.cstride == 1) return a.raw[i];
  return a.raw[i * 3 + fc_rt(a, row, col)];
}

__global__ void __launch_bounds__(AMZ_THREADS, 1) k_amaze(AmazeArgs A) {
  const int v1 = TS, v2 = 2 * TS, v3 = 3 * TS, p1 = -TS + 1, p2 = -2 * TS + 2, p3 = -3 * TS + 3, m1 = TS + 1,
            m2 = 2 * TS + 2, m3 = 3 * TS + 3;
  const float gaussodd[4] = {0.14659727707323927f, 0.103592713382435f, 0.0732036125103057f, 0.0365543548389495f};
  const float gaussgrad[6] = {nyqthresh * 0.07384411893421103f, nyqthresh * 0.06207511968171489f,
                              nyqthresh * 0.0521818194747806f,  nyqthresh * 0.03687419286733595f,
                              nyqthresh * 0.03099732204057846f, nyqthresh * 0.018413194161458882f};
  const float gausseven[2] = {0.13719494435797422f, 0.05640252782101291f};
  const float gquinc[4] = {0.169917f, 0.108947f, 0.069855f, 0.0287182f};
  const int tid = threadIdx.x, nth = blockDim.x;
  const int W = A.W, H = A.H;
  Slab S = make_slab(A.scratch + (size_t)blockIdx.x * kSlabBytes);
  __shared__ int s_tile;
  __shared__ int s_doNyq;

  for (;;) {
    if (tid == 0) s_tile = atomicAdd(A.tile_counter, 1);
    __syncthreads();
    const int tile = s_tile;
    __syncthreads();
    if (tile >= A.n_top * A.n_left) break;
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

    // ---- fresh scratch: zero every plane (reads outside a stage's written
    // range see zeros, as in a newly allocated reference buffer).
    {
      float4* z = reinterpret_cast<float4*>(S.cfa);
      const size_t n4 = (kSlabBytes - 256) / 16;
      for (size_t i = tid; i < n4; i += nth) z[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    __syncthreads();

    // ---- fill (:1254-1326)
    const float scale = A.scale;
    for (int i = tid; i < rr1 * cc1; i += nth) {
      const int rr = i / cc1, cc = i % cc1;
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
      if (srow >= 0) {
        const float val = raw_at(A, srow, scol) * scale;
        S.cfa[rr * TS + cc] = val;
        S.rgbgreen[rr * TS + cc] = val;
      }
    }
    __syncthreads();

    float* cfa = S.cfa;
    float* dirwts0 = S.dirwts0;
    float* dirwts1 = S.dirwts1;
    // ---- S1 gradients (:1330-1339)
    for (int i = tid; i < (rr1 - 4) * (cc1 - 4); i += nth) {
      const int rr = 2 + i / (cc1 - 4), cc = 2 + i % (cc1 - 4);
      const int idx = rr * TS + cc;
      const float delh = fabsf(cfa[idx + 1] - cfa[idx - 1]);
      const float delv = fabsf(cfa[idx + v1] - cfa[idx - v1]);
      dirwts0[idx] = eps + fabsf(cfa[idx + v2] - cfa[idx]) + fabsf(cfa[idx] - cfa[idx - v2]) + delv;
      dirwts1[idx] = eps + fabsf(cfa[idx + 2] - cfa[idx]) + fabsf(cfa[idx] - cfa[idx - 2]) + delh;
      S.delhvsqsum[idx] = SQR(delh) + SQR(delv);
    }
    __syncthreads();

    // ---- S2 colour differences (:1341-1373)
    for (int i = tid; i < (rr1 - 8) * (cc1 - 8); i += nth) {
      const int rr = 4 + i / (cc1 - 8), cc = 4 + i % (cc1 - 8);
      const int idx = rr * TS + cc;
      const int sgn = (fc_rt(A, rr, cc) & 1) ? -1 : 1;
      const float cru = cfa[idx - v1] * (dirwts0[idx - v2] + dirwts0[idx]) /
                        (dirwts0[idx - v2] * (eps + cfa[idx]) + dirwts0[idx] * (eps + cfa[idx - v2]));
      const float crd = cfa[idx + v1] * (dirwts0[idx + v2] + dirwts0[idx]) /
                        (dirwts0[idx + v2] * (eps + cfa[idx]) + dirwts0[idx] * (eps + cfa[idx + v2]));
      const float crl = cfa[idx - 1] * (dirwts1[idx - 2] + dirwts1[idx]) /
                        (dirwts1[idx - 2] * (eps + cfa[idx]) + dirwts1[idx] * (eps + cfa[idx - 2]));
      const float crr = cfa[idx + 1] * (dirwts1[idx + 2] + dirwts1[idx]) /
                        (dirwts1[idx + 2] * (eps + cfa[idx]) + dirwts1[idx] * (eps + cfa[idx + 2]));
      const float guha = cfa[idx - v1] + xdiv2f(cfa[idx] - cfa[idx - v2]);
      const float gdha = cfa[idx + v1] + xdiv2f(cfa[idx] - cfa[idx + v2]);
      const float glha = cfa[idx - 1] + xdiv2f(cfa[idx] - cfa[idx - 2]);
      const float grha = cfa[idx + 1] + xdiv2f(cfa[idx] - cfa[idx + 2]);
      float guar = fabsf(1.f - cru) < arthresh ? cfa[idx] * cru : guha;
      float gdar = fabsf(1.f - crd) < arthresh ? cfa[idx] * crd : gdha;
      float glar = fabsf(1.f - crl) < arthresh ? cfa[idx] * crl : glha;
      float grar = fabsf(1.f - crr) < arthresh ? cfa[idx] * crr : grha;
      const float hwt = dirwts1[idx - 1] / (dirwts1[idx - 1] + dirwts1[idx + 1]);
      const float vwt = dirwts0[idx - v1] / (dirwts0[idx + v1] + dirwts0[idx - v1]);
      const float Gintvha = vwt * gdha + (1.f - vwt) * guha;
      const float Ginthha = hwt * grha + (1.f - hwt) * glha;
      const float fs = (float)sgn;
      S.vcdalt[idx] = fs * (Gintvha - cfa[idx]);
      S.hcdalt[idx] = fs * (Ginthha - cfa[idx]);
      if (cfa[idx] > A.clip_pt8 || Gintvha > A.clip_pt8 || Ginthha > A.clip_pt8) {
        S.vcd[idx] = S.vcdalt[idx];
        S.hcd[idx] = S.hcdalt[idx];
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

    // ---- S3 variance + bounding (:1375-1398): hcd chains along rows,
    // vcd chains along columns (stride 2, in place, as the reference scans).
    {
      const int nrows = rr1 - 8, ncols = cc1 - 8;
      const int n_h = nrows * 2, n_v = ncols * 2;
      for (int item = tid; item < n_h + n_v; item += nth) {
        if (item < n_h) {
          const int rr = 4 + item / 2, par = item % 2;
          float* hcd = S.hcd;
          const float* hcdalt = S.hcdalt;
          for (int cc = 4 + par; cc < cc1 - 4; cc += 2) {
            const int idx = rr * TS + cc;
            const float hcdvar = 3.f * (SQR(hcd[idx - 2]) + SQR(hcd[idx]) + SQR(hcd[idx + 2])) -
                                 SQR(hcd[idx - 2] + hcd[idx] + hcd[idx + 2]);
            const float hcdaltvar = 3.f * (SQR(hcdalt[idx - 2]) + SQR(hcdalt[idx]) + SQR(hcdalt[idx + 2])) -
                                    SQR(hcdalt[idx - 2] + hcdalt[idx] + hcdalt[idx + 2]);
            float h = hcd[idx];
            if (hcdaltvar < hcdvar) h = hcdalt[idx];
            float Ginth;
            if (fc_rt(A, rr, cc) & 1) {
              Ginth = -h + cfa[idx];
              if (h > 0) {
                if (3.f * h > (Ginth + cfa[idx])) {
                  h = -median3(Ginth, cfa[idx - 1], cfa[idx + 1]) + cfa[idx];
                } else {
                  const float hwt2 = 1.f - 3.f * h / (eps + Ginth + cfa[idx]);
                  h = hwt2 * h + (1.f - hwt2) * (-median3(Ginth, cfa[idx - 1], cfa[idx + 1]) + cfa[idx]);
                }
              }
            } else {
              Ginth = h + cfa[idx];
              if (h < 0) {
                if (3.f * h < -(Ginth + cfa[idx])) {
                  h = median3(Ginth, cfa[idx - 1], cfa[idx + 1]) - cfa[idx];
                } else {
                  const float hwt2 = 1.f + 3.f * h / (eps + Ginth + cfa[idx]);
                  h = hwt2 * h + (1.f - hwt2) * (median3(Ginth, cfa[idx - 1], cfa[idx + 1]) - cfa[idx]);
                }
              }
            }
            if (Ginth > A.clip_pt)
              h = (float)((fc_rt(A, rr, cc) & 1) ? -1 : 1) * (median3(Ginth, cfa[idx - 1], cfa[idx + 1]) - cfa[idx]);
            hcd[idx] = h;
          }
        } else {
          const int it = item - n_h;
          const int cc = 4 + it / 2, par = it % 2;
          float* vcd = S.vcd;
          const float* vcdalt = S.vcdalt;
          for (int rr = 4 + par; rr < rr1 - 4; rr += 2) {
            const int idx = rr * TS + cc;
            const float vcdvar = 3.f * (SQR(vcd[idx - v2]) + SQR(vcd[idx]) + SQR(vcd[idx + v2])) -
                                 SQR(vcd[idx - v2] + vcd[idx] + vcd[idx + v2]);
            const float vcdaltvar = 3.f * (SQR(vcdalt[idx - v2]) + SQR(vcdalt[idx]) + SQR(vcdalt[idx + v2])) -
                                    SQR(vcdalt[idx - v2] + vcdalt[idx] + vcdalt[idx + v2]);
            float v = vcd[idx];
            if (vcdaltvar < vcdvar) v = vcdalt[idx];
            float Gintv;
            if (fc_rt(A, rr, cc) & 1) {
              Gintv = -v + cfa[idx];
              if (v > 0) {
                if (3.f * v > (Gintv + cfa[idx])) {
                  v = -median3(Gintv, cfa[idx - v1], cfa[idx + v1]) + cfa[idx];
                } else {
                  const float vwt2 = 1.f - 3.f * v / (eps + Gintv + cfa[idx]);
                  v = vwt2 * v + (1.f - vwt2) * (-median3(Gintv, cfa[idx - v1], cfa[idx + v1]) + cfa[idx]);
                }
              }
            } else {
              Gintv = v + cfa[idx];
              if (v < 0) {
                if (3.f * v < -(Gintv + cfa[idx])) {
                  v = median3(Gintv, cfa[idx - v1], cfa[idx + v1]) - cfa[idx];
                } else {
                  const float vwt2 = 1.f + 3.f * v / (eps + Gintv + cfa[idx]);
                  v = vwt2 * v + (1.f - vwt2) * (median3(Gintv, cfa[idx - v1], cfa[idx + v1]) - cfa[idx]);
                }
              }
            }
            if (Gintv > A.clip_pt)
              v = (float)((fc_rt(A, rr, cc) & 1) ? -1 : 1) * (median3(Gintv, cfa[idx - v1], cfa[idx + v1]) - cfa[idx]);
            vcd[idx] = v;
          }
        }
      }
    }
    __syncthreads();
    for (int i = tid; i < (rr1 - 8) * (cc1 - 8); i += nth) {
      const int rr = 4 + i / (cc1 - 8), cc = 4 + i % (cc1 - 8);
      const int idx = rr * TS + cc;
      S.cddiffsq[idx] = SQR(S.vcd[idx] - S.hcd[idx]);
    }
    __syncthreads();

    // R/B-site iteration helper: rows [a, rr1-a), cc = a + (fc(rr,2)&1) step 2, cc < cc1 - a.
    auto rb_count = [&](int a) { return (cc1 - a - a + 1) / 2 + 1; };

    // ---- S4/5 directional variance + Nyquist test (:1400-1433)
    if (tid == 0) s_doNyq = 0;
    {
      const int a = 6;
      const int per_row = rb_count(a);
      for (int i = tid; i < (rr1 - 2 * a) * per_row; i += nth) {
        const int rr = a + i / per_row;
        const int cc = a + (fc_rt(A, rr, 2) & 1) + 2 * (i % per_row);
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
        const float hwt = dirwts1[idx - 1] / (dirwts1[idx - 1] + dirwts1[idx + 1]);
        const float vwt = dirwts0[idx - v1] / (dirwts0[idx + v1] + dirwts0[idx - v1]);
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
        S.hvwt[idx >> 1] =
            ((0.5f - varwt) * (0.5f - diffwt) > 0.f && fabsf(0.5f - diffwt) < fabsf(0.5f - varwt)) ? varwt : diffwt;
        const float* cdd = S.cddiffsq;
        const float* dhv = S.delhvsqsum;
        const float nt =
            (gaussodd[0] * cdd[idx] + gaussodd[1] * (cdd[idx - m1] + cdd[idx + p1] + cdd[idx - p1] + cdd[idx + m1]) +
             gaussodd[2] * (cdd[idx - v2] + cdd[idx - 2] + cdd[idx + 2] + cdd[idx + v2]) +
             gaussodd[3] * (cdd[idx - m2] + cdd[idx + p2] + cdd[idx - p2] + cdd[idx + m2])) -
            (gaussgrad[0] * dhv[idx] + gaussgrad[1] * (dhv[idx - v1] + dhv[idx + 1] + dhv[idx - 1] + dhv[idx + v1]) +
             gaussgrad[2] * (dhv[idx - m1] + dhv[idx + p1] + dhv[idx - p1] + dhv[idx + m1]) +
             gaussgrad[3] * (dhv[idx - v2] + dhv[idx - 2] + dhv[idx + 2] + dhv[idx + v2]) +
             gaussgrad[4] * (dhv[idx - v2 - 1] + dhv[idx - v2 + 1] + dhv[idx - TS - 2] + dhv[idx - TS + 2] +
                             dhv[idx + TS - 2] + dhv[idx + TS + 2] + dhv[idx + v2 - 1] + dhv[idx + v2 + 1]) +
             gaussgrad[5] * (dhv[idx - m2] + dhv[idx + p2] + dhv[idx - p2] + dhv[idx + m2]));
        S.nyqutest[idx >> 1] = nt;
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
      for (int i = tid; i < (rr1 - 2 * a) * per_row; i += nth) {
        const int rr = a + i / per_row;
        const int cc = a + (fc_rt(A, rr, 2) & 1) + 2 * (i % per_row);
        if (cc >= cc1 - a) continue;
        const int idx = rr * TS + cc;
        const unsigned char* nq = S.nyquist;
        const unsigned nqsum = nq[(idx - v2) >> 1] + nq[(idx - m1) >> 1] + nq[(idx + p1) >> 1] + nq[(idx - 2) >> 1] +
                               nq[(idx + 2) >> 1] + nq[(idx - p1) >> 1] + nq[(idx + m1) >> 1] + nq[(idx + v2) >> 1];
        S.nyquist2[idx >> 1] = nqsum > 4 ? 1 : (nqsum < 4 ? 0 : nq[idx >> 1]);
      }
      __syncthreads();
      for (int i = tid; i < (rr1 - 2 * a) * per_row; i += nth) {
        const int rr = a + i / per_row;
        const int cc = a + (fc_rt(A, rr, 2) & 1) + 2 * (i % per_row);
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
        S.hvwt[idx >> 1] = hcdvar2 / (vcdvar2 + hcdvar2);
      }
      __syncthreads();
    }
    // Gauss-Seidel sweep over rows (row rr reads the updated row rr-1).
    {
      const int a = 8;
      const int per_row = rb_count(a);
      float* hvwt = S.hvwt;
      float* rgbgreen = S.rgbgreen;
      for (int rr = a; rr < rr1 - a; rr++) {
        for (int k = tid; k < per_row; k += nth) {
          const int cc = a + (fc_rt(A, rr, 2) & 1) + 2 * k;
          if (cc >= cc1 - a) continue;
          const int idx = rr * TS + cc;
          const float hvwtalt =
              0.25f * (hvwt[(idx - m1) >> 1] + hvwt[(idx + p1) >> 1] + hvwt[(idx - p1) >> 1] + hvwt[(idx + m1) >> 1]);
          const float hv = fabsf(0.5f - hvwt[idx >> 1]) < fabsf(0.5f - hvwtalt) ? hvwtalt : hvwt[idx >> 1];
          hvwt[idx >> 1] = hv;
          const float d0 = hv * S.vcd[idx] + (1.f - hv) * S.hcd[idx];
          S.Dgrb0[idx >> 1] = d0;
          const float g = cfa[idx] + d0;
          rgbgreen[idx] = g;
          const bool nq2 = S.nyquist2[idx >> 1] != 0;
          S.Dgrb2h[idx >> 1] = nq2 ? SQR(g - xdiv2f(rgbgreen[idx - 1] + rgbgreen[idx + 1])) : 0.f;
          S.Dgrb2v[idx >> 1] = nq2 ? SQR(g - xdiv2f(rgbgreen[idx - v1] + rgbgreen[idx + v1])) : 0.f;
        }
        __syncthreads();
      }
    }
    if (doNyquist) {
      const int a = 8;
      const int per_row = rb_count(a);
      const float* D2h = S.Dgrb2h;
      const float* D2v = S.Dgrb2v;
      for (int i = tid; i < (rr1 - 2 * a) * per_row; i += nth) {
        const int rr = a + i / per_row;
        const int cc = a + (fc_rt(A, rr, 2) & 1) + 2 * (i % per_row);
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
        S.rgbgreen[idx] = cfa[idx] + d0;
      }
      __syncthreads();
    }

    // ---- S7 R/B gradients (:1483-1502)
    for (int i = tid; i < (rr1 - 12) * ((cc1 - 12 + 1) / 2); i += nth) {
      const int per_row = (cc1 - 12 + 1) / 2;
      const int rr = 6 + i / per_row;
      const int cc = 6 + 2 * (i % per_row);
      const int idx = rr * TS + cc;
      if ((fc_rt(A, rr, 2) & 1) == 0) {
        S.delp[idx >> 1] = fabsf(cfa[idx + p1] - cfa[idx - p1]);
        S.delm[idx >> 1] = fabsf(cfa[idx + m1] - cfa[idx - m1]);
        S.Dgrbsq1p[idx >> 1] = SQR(cfa[idx + 1] - cfa[idx + 1 - p1]) + SQR(cfa[idx + 1] - cfa[idx + 1 + p1]);
        S.Dgrbsq1m[idx >> 1] = SQR(cfa[idx + 1] - cfa[idx + 1 - m1]) + SQR(cfa[idx + 1] - cfa[idx + 1 + m1]);
      } else {
        S.Dgrbsq1p[idx >> 1] = SQR(cfa[idx] - cfa[idx - p1]) + SQR(cfa[idx] - cfa[idx + p1]);
        S.Dgrbsq1m[idx >> 1] = SQR(cfa[idx] - cfa[idx - m1]) + SQR(cfa[idx] - cfa[idx + m1]);
        S.delp[idx >> 1] = fabsf(cfa[idx + 1 + p1] - cfa[idx + 1 - p1]);
        S.delm[idx >> 1] = fabsf(cfa[idx + 1 + m1] - cfa[idx + 1 - m1]);
      }
    }
    __syncthreads();

    // ---- S8 diagonal R/B interpolation (:1504-1532)
    {
      const int a = 8;
      const int per_row = rb_count(a);
      const float* delp = S.delp;
      const float* delm = S.delm;
      const float* Dq1m = S.Dgrbsq1m;
      const float* Dq1p = S.Dgrbsq1p;
      for (int i = tid; i < (rr1 - 2 * a) * per_row; i += nth) {
        const int rr = a + i / per_row;
        const int cc = a + (fc_rt(A, rr, 2) & 1) + 2 * (i % per_row);
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
        S.pmwt[idx1] = rbvarm / (rbvarp + rbvarm);
      }
    }
    __syncthreads();

    // ---- S9 (:1534-1592): Gauss-Seidel pmwt sweep + rbint
    {
      const int a = 10;
      const int per_row = rb_count(a);
      float* pmwt = S.pmwt;
      for (int rr = a; rr < rr1 - a; rr++) {
        for (int k = tid; k < per_row; k += nth) {
          const int cc = a + (fc_rt(A, rr, 2) & 1) + 2 * k;
          if (cc >= cc1 - a) continue;
          const int idx = rr * TS + cc, idx1 = idx >> 1;
          const float pmwtalt =
              0.25f * (pmwt[(idx - m1) >> 1] + pmwt[(idx + p1) >> 1] + pmwt[(idx - p1) >> 1] + pmwt[(idx + m1) >> 1]);
          float pw = pmwt[idx1];
          if (fabsf(0.5f - pw) < fabsf(0.5f - pmwtalt)) pw = pmwtalt;
          pmwt[idx1] = pw;
          S.rbint[idx1] = xdiv2f(cfa[idx] + S.rbm[idx1] * (1.f - pw) + S.rbp[idx1] * pw);
        }
        __syncthreads();
      }
    }
    // dirwts1 as the reference reads it after pmwt was stored over it
    // (half index k of pmwt == float offset k of dirwts1).
    auto pm_written = [&](int p) -> bool {
      if (p < 0 || p >= TS * TSH) return false;
      const int r2 = (2 * p) / TS;
      const int c0 = (2 * p) % TS;
      const int crb = c0 + (int)(fc_rt(A, r2, 2) & 1);
      return r2 >= 8 && r2 < rr1 - 8 && crb >= 8 && crb < cc1 - 8;
    };
    auto dirwts1_eff = [&](int p) -> float { return pm_written(p) ? S.pmwt[p] : dirwts1[p]; };
    {
      const int a = 12;
      const int per_row = rb_count(a);
      const float* rbint = S.rbint;
      for (int i = tid; i < (rr1 - 2 * a) * per_row; i += nth) {
        const int rr = a + i / per_row;
        const int cc = a + (fc_rt(A, rr, 2) & 1) + 2 * (i % per_row);
        if (cc >= cc1 - a) continue;
        const int idx = rr * TS + cc, idx1 = idx >> 1;
        if (fabsf(0.5f - S.pmwt[idx1]) >= fabsf(0.5f - S.hvwt[idx1])) continue;
        const float cru = xmul2f(cfa[idx - v1]) / (eps + rbint[idx1] + rbint[idx1 - v1]);
        const float crd = xmul2f(cfa[idx + v1]) / (eps + rbint[idx1] + rbint[idx1 + v1]);
        const float crl = xmul2f(cfa[idx - 1]) / (eps + rbint[idx1] + rbint[idx1 - 1]);
        const float crr = xmul2f(cfa[idx + 1]) / (eps + rbint[idx1] + rbint[idx1 + 1]);
        const float gu = fabsf(1.f - cru) < arthresh ? rbint[idx1] * cru : cfa[idx - v1] + xdiv2f(rbint[idx1] - rbint[idx1 - v1]);
        const float gd = fabsf(1.f - crd) < arthresh ? rbint[idx1] * crd : cfa[idx + v1] + xdiv2f(rbint[idx1] - rbint[idx1 + v1]);
        const float gl = fabsf(1.f - crl) < arthresh ? rbint[idx1] * crl : cfa[idx - 1] + xdiv2f(rbint[idx1] - rbint[idx1 - 1]);
        const float gr = fabsf(1.f - crr) < arthresh ? rbint[idx1] * crr : cfa[idx + 1] + xdiv2f(rbint[idx1] - rbint[idx1 + 1]);
        float Gintv = (dirwts0[idx - v1] * gd + dirwts0[idx + v1] * gu) / (dirwts0[idx + v1] + dirwts0[idx - v1]);
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
        const float hv = S.hvwt[idx1];
        const float g = Ginth * (1.f - hv) + Gintv * hv;
        S.rgbgreen[idx] = g;
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
      for (int i = tid; i < (rr1 - 2 * a) * per_row; i += nth) {
        const int rr = a + i / per_row;
        const int cc = a + (fc_rt(A, rr, 2) & 1) + 2 * (i % per_row);
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
      const int rr = 16 + i / (cc1 - 32), cc = 16 + i % (cc1 - 32);
      const int row = rr + top, col = cc + left;
      if (row < 0 || row >= H || col < 0 || col >= W) continue;
      const int t = rr * TS + cc;
      float r, g, b;
      const float* hvwt = S.hvwt;
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
        g = S.rgbgreen[t];
        r = g - D0[t >> 1];
        b = g - D1[t >> 1];
      }
      float* o = A.rgb + ((size_t)row * W + col) * 3;
      o[0] = fmaxf(0.f, r);
      o[1] = fmaxf(0.f, g);
      o[2] = fmaxf(0.f, b);
    }
    __syncthreads();
  }
}

// LibRaw-style border interpolation (core/cpu_accelerator.cpp:2984-3028):
// only pixels within `border` of the frame; non-native channels become the
// mean of that colour's samples in the clipped 3x3 neighbourhood.
__global__ void k_border_interp(float* rgb, int W, int H, uint32_t filters, int border) {
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
  }
}

}  // namespace

size_t ws_bytes_amaze(size_t w, size_t h) {
  (void)w;
  (void)h;
  return 148u * 2u * kSlabBytes + 4096;
}

lre_status launch_amaze(Context* c, const float* raw, int cstride, float* rgb, size_t w, size_t h, uint32_t filters,
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
  if (A.cfarray[0][0] == 1) {
    if (A.cfarray[0][1] == 0) { A.ey = 0; A.ex = 1; } else { A.ey = 1; A.ex = 0; }
  } else {
    if (A.cfarray[0][0] == 0) { A.ey = 0; A.ex = 0; } else { A.ey = 1; A.ex = 1; }
  }
  A.scale = 1.0f / maximum_value;
  A.n_top = (int)((h + 16 + (TS - 32) - 1) / (TS - 32));
  A.n_left = (int)((w + 16 + (TS - 32) - 1) / (TS - 32));
  // verify the tile count matches the reference's loop bounds
  while (A.n_top > 0 && -16 + (A.n_top - 1) * (TS - 32) >= (int)h) A.n_top--;
  while (A.n_left > 0 && -16 + (A.n_left - 1) * (TS - 32) >= (int)w) A.n_left--;
  const int tiles = A.n_top * A.n_left;
  int nblk = std::min(tiles, c->sm_count);
  if (nblk < 1) nblk = 1;
  A.scratch = reinterpret_cast<unsigned char*>(c->ws.take((size_t)nblk * kSlabBytes));
  A.tile_counter = reinterpret_cast<int*>(c->ws.take(256));
  if (!A.scratch || !A.tile_counter) return fail(c, LRE_ERR_OUT_OF_MEMORY, "demosaic_bayer_amaze: workspace too small");
  LRE_CUDA_TRY(c, cudaMemsetAsync(A.tile_counter, 0, sizeof(int), c->stream));
  k_amaze<<<nblk, AMZ_THREADS, 0, c->stream>>>(A);
  const int band = 4;
  const long long nb = 2LL * band * (long long)w + 2LL * band * (long long)(h > 8 ? h - 8 : 0);
  k_border_interp<<<grid_for((size_t)nb, 256, c->sm_count * 2), 256, 0, c->stream>>>(rgb, (int)w, (int)h, filters, band);
  count_launch(c, 2);
  return check_launch(c, "demosaic_bayer_amaze");
}

}  // namespace lre
