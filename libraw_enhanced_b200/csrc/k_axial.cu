// k_axial.cu -- axial chromatic-aberration cleanup: cross-channel guided
// filter of R and B with G as the guide, edge-gated blend.
//
// Semantics follow core/cpu_accelerator.cpp:3799-3928
// (CPUAccelerator::ca_axial_cleanup) with guided_filter_with_shared_guide
// (:3725-3777) and box_mean (:3703-3716):
//   * R, G, B are normalised by norm = max(1e-6, max G) (float multiply by
//     1/norm, exactly as the reference);
//   * box means use an edge-truncated (2r+1)^2 window; the reference builds
//     double summed-area tables, here every window sum is accumulated in
//     double directly (sliding sums), which equals the SAT difference up to
//     double rounding;
//   * a = cov(G,X) / (var(G) + eps), b = mean(X) - a mean(G) in double, stored
//     as float; q = mean(a) * G + mean(b) in double, stored as float;
//   * edge weight w = smoothstep(0.01, 0.06, boxmean_r(|central grad G|));
//   * out = (X (1 - s w) + q s w) * norm, G passes through.
//
// B200 design: after the global max(G) reduction, two streaming passes over
// column strips (k_ax_ab: guide statistics and the a/b solve for R and B;
// k_ax_q: second box level, edge gate and blend), each pixel's window sums
// computed once, with the a/b planes (16 B/px) passing through HBM.  The
// older single fused tile kernel (k_axial_fused: both box levels out of
// shared memory, the level-one statistics recomputed over each tile's halo)
// remains for the allocation-free entry point at the end of this file.
#include <mutex>

#include <functional>

#include "common.cuh"
#include "lre_internal.h"

namespace lre {

namespace {

struct AxGeom {
  int T, r, IN, AB;
  size_t off_g, off_r, off_b, off_h0, off_h1, off_mi, off_vi, off_ar, off_br, off_ab, off_bb, off_er, bytes;
};

__host__ __device__ inline AxGeom ax_geom(int T, int r) {
  AxGeom g;
  g.T = T;
  g.r = r;
  g.IN = T + 4 * r;
  g.AB = T + 2 * r;
  size_t o = 0;
  auto take = [&](size_t b) {
    size_t cur = o;
    o += (b + 15) & ~size_t(15);
    return cur;
  };
  // odd row strides (IN+1 floats, AB+1 doubles) keep warp accesses that walk
  // down rows on distinct shared-memory banks
  size_t in2 = (size_t)g.IN * (g.IN + 1), hb = (size_t)g.IN * (g.AB + 1), ab2 = (size_t)g.AB * g.AB;
  g.off_h0 = take(hb * 8);
  g.off_h1 = take(hb * 8);
  g.off_mi = take(ab2 * 8);
  g.off_vi = take(ab2 * 8);
  g.off_g = take(in2 * 4);
  g.off_r = take(in2 * 4);
  g.off_b = take(in2 * 4);
  const size_t abp = (size_t)g.AB * (g.AB + 1);  // float planes, row stride AB + 1
  g.off_ar = take(abp * 4);
  g.off_br = take(abp * 4);
  g.off_ab = take(abp * 4);
  g.off_bb = take(abp * 4);
  g.off_er = take(abp * 4);
  g.bytes = o;
  return g;
}

// Sliding horizontal window sums: dst[j][k] = sum_{t=0..2r} val(j, k + t)
// for j < rows, k < cols_out, stored with row stride cols_out + 1.  Rows are
// split into segments so every thread has work; inside a segment the sum
// slides with one add and one subtract.  Consecutive threads take
// consecutive rows of the same segment (distinct banks with odd strides).
template <typename F>
__device__ void hsum(double* dst, int rows, int cols_out, int r, F val) {
  const int seg = max(1, (rows * cols_out + (int)blockDim.x - 1) / (int)blockDim.x);
  const int nseg = (cols_out + seg - 1) / seg;
  const int ld = cols_out + 1;
  for (int item = threadIdx.x; item < rows * nseg; item += blockDim.x) {
    int j = item % rows, s = item / rows;
    int k0 = s * seg, k1 = min(cols_out, k0 + seg);
    double acc = 0.0;
    for (int t = 0; t <= 2 * r; t++) acc += val(j, k0 + t);
    dst[j * ld + k0] = acc;
    for (int k = k0 + 1; k < k1; k++) {
      acc += val(j, k + 2 * r);
      acc -= val(j, k - 1);
      dst[j * ld + k] = acc;
    }
  }
}

// Two horizontal window sums in one sweep (two independent accumulators per
// thread, for quantities that are always consumed together).
template <typename F0, typename F1>
__device__ void hsum2(double* d0, double* d1, int rows, int cols_out, int r, F0 v0, F1 v1) {
  // segment length chosen so one pass of the block covers every row segment
  const int seg = max(1, (rows * cols_out + (int)blockDim.x - 1) / (int)blockDim.x);
  const int nseg = (cols_out + seg - 1) / seg;
  const int ld = cols_out + 1;
  for (int item = threadIdx.x; item < rows * nseg; item += blockDim.x) {
    int j = item % rows, s = item / rows;
    int k0 = s * seg, k1 = min(cols_out, k0 + seg);
    double a0 = 0.0, a1 = 0.0;
    for (int t = 0; t <= 2 * r; t++) {
      a0 += v0(j, k0 + t);
      a1 += v1(j, k0 + t);
    }
    d0[j * ld + k0] = a0;
    d1[j * ld + k0] = a1;
    for (int k = k0 + 1; k < k1; k++) {
      a0 += v0(j, k + 2 * r);
      a1 += v1(j, k + 2 * r);
      a0 -= v0(j, k - 1);
      a1 -= v1(j, k - 1);
      d0[j * ld + k] = a0;
      d1[j * ld + k] = a1;
    }
  }
}

__device__ __forceinline__ int win_count(int p, int r, int n) {
  int lo = p - r < 0 ? 0 : p - r;
  int hi = p + r > n - 1 ? n - 1 : p + r;
  return hi - lo + 1;
}

template <int T, int NT>
__global__ void __launch_bounds__(NT, NT <= 256 ? 2 : 1)
    k_axial_fused(const float* __restrict__ src, float* __restrict__ dst, int W, int H, int r, float eps,
                  float strength, const float* __restrict__ d_maxg) {
  extern __shared__ __align__(16) unsigned char smem[];
  const AxGeom g = ax_geom(T, r);
  double* h0 = reinterpret_cast<double*>(smem + g.off_h0);
  double* h1 = reinterpret_cast<double*>(smem + g.off_h1);
  double* mI = reinterpret_cast<double*>(smem + g.off_mi);
  double* vI = reinterpret_cast<double*>(smem + g.off_vi);
  float* sG = reinterpret_cast<float*>(smem + g.off_g);
  float* sR = reinterpret_cast<float*>(smem + g.off_r);
  float* sB = reinterpret_cast<float*>(smem + g.off_b);
  float* aR = reinterpret_cast<float*>(smem + g.off_ar);
  float* bR = reinterpret_cast<float*>(smem + g.off_br);
  float* aB = reinterpret_cast<float*>(smem + g.off_ab);
  float* bB = reinterpret_cast<float*>(smem + g.off_bb);
  float* er = reinterpret_cast<float*>(smem + g.off_er);

  const int IN = g.IN, AB = g.AB;
  const int x0 = blockIdx.x * T, y0 = blockIdx.y * T;
  const int ix0 = x0 - 2 * r, iy0 = y0 - 2 * r;  // global coords of input region origin
  const int ax0 = x0 - r, ay0 = y0 - r;          // global coords of a/b region origin

  const float norm_ref = fmaxf(*d_maxg, 1e-6f);
  const float inv_norm = 1.f / norm_ref;

  // Reciprocal window counts along x and y for every column / row of the
  // input region (0 outside the image): a box mean is sum * inv_x * inv_y,
  // within two double ulps of the reference's sum / area.
  __shared__ double inv_x[T + 4 * 16], inv_y[T + 4 * 16];
  for (int i = threadIdx.x; i < IN; i += blockDim.x) {
    const int gx = ix0 + i, gy = iy0 + i;
    inv_x[i] = (gx >= 0 && gx < W) ? 1.0 / (double)win_count(gx, r, W) : 0.0;
    inv_y[i] = (gy >= 0 && gy < H) ? 1.0 / (double)win_count(gy, r, H) : 0.0;
  }

  const int SP = IN + 1;   // row stride of the staged planes (odd)
  const int LDH = AB + 1;  // row stride of the level-1 window sums (odd)
  const int LDB = AB + 1;  // row stride of the a/b/edge planes (odd)

  // 1. stage normalised R, G, B (zeros outside the image).
  for (int i = threadIdx.x; i < IN * IN; i += blockDim.x) {
    const int j = i / IN, k = i % IN;
    int gy = iy0 + j, gx = ix0 + k;
    float r_ = 0.f, g_ = 0.f, b_ = 0.f;
    if (gx >= 0 && gx < W && gy >= 0 && gy < H) {
      const float* p = src + ((size_t)gy * W + gx) * 3;
      r_ = p[0] * inv_norm;
      g_ = p[1] * inv_norm;
      b_ = p[2] * inv_norm;
    }
    sR[j * SP + k] = r_;
    sG[j * SP + k] = g_;
    sB[j * SP + k] = b_;
  }
  __syncthreads();

  // 2. guide statistics mean(G), var(G) over the a/b region.
  hsum2(
      h0, h1, IN, AB, r, [&](int j, int k) { return (double)sG[j * SP + k]; },
      [&](int j, int k) {
        float v = sG[j * SP + k];
        return (double)(v * v);
      });
  __syncthreads();
  // a/b-region cell (j, k) sits at input-region index (j + r, k + r)
  {
    const int seg = 8;
    const int nseg = (AB + seg - 1) / seg;
    for (int item = threadIdx.x; item < AB * nseg; item += blockDim.x) {
      const int k = item % AB, s = item / AB;
      const int j0 = s * seg, j1 = min(AB, j0 + seg);
      double s0 = 0.0, s1 = 0.0;
      for (int t = 0; t <= 2 * r; t++) {
        s0 += h0[(j0 + t) * LDH + k];
        s1 += h1[(j0 + t) * LDH + k];
      }
      for (int j = j0; j < j1; j++) {
        if (j > j0) {
          s0 += h0[(j + 2 * r) * LDH + k];
          s1 += h1[(j + 2 * r) * LDH + k];
          s0 -= h0[(j - 1) * LDH + k];
          s1 -= h1[(j - 1) * LDH + k];
        }
        const double inv_area = inv_x[k + r] * inv_y[j + r];
        const double m = s0 * inv_area;
        mI[j * AB + k] = m;
        vI[j * AB + k] = s1 * inv_area - m * m;
      }
    }
  }
  __syncthreads();

  // 3. per-channel a, b (R then B), sharing the guide statistics.
  for (int ch = 0; ch < 2; ch++) {
    const float* sX = ch == 0 ? sR : sB;
    float* aX = ch == 0 ? aR : aB;
    float* bX = ch == 0 ? bR : bB;
    hsum2(
        h0, h1, IN, AB, r, [&](int j, int k) { return (double)sX[j * SP + k]; },
        [&](int j, int k) { return (double)(sG[j * SP + k] * sX[j * SP + k]); });
    __syncthreads();
    // mean(X) into aX temporarily as double is not possible (float); keep the
    // double mean in vI's sibling: reuse h0's first AB*AB doubles after the
    // vertical pass would clobber its input, so compute both sums per pixel
    // in one vertical sweep over the two buffers.
    {
      const int seg = 8;
      const int nseg = (AB + seg - 1) / seg;
      for (int item = threadIdx.x; item < AB * nseg; item += blockDim.x) {
        int k = item % AB, s = item / AB;
        int j0 = s * seg, j1 = min(AB, j0 + seg);
        double sp = 0.0, sip = 0.0;
        for (int t = 0; t <= 2 * r; t++) {
          sp += h0[(j0 + t) * LDH + k];
          sip += h1[(j0 + t) * LDH + k];
        }
        for (int j = j0; j < j1; j++) {
          if (j > j0) {
            sp += h0[(j + 2 * r) * LDH + k];
            sp -= h0[(j - 1) * LDH + k];
            sip += h1[(j + 2 * r) * LDH + k];
            sip -= h1[(j - 1) * LDH + k];
          }
          int gy = ay0 + j, gx = ax0 + k;
          float a_f = 0.f, b_f = 0.f;
          if (gx >= 0 && gx < W && gy >= 0 && gy < H) {
            const double inv_area = inv_x[k + r] * inv_y[j + r];
            double mp = sp * inv_area, mIp = sip * inv_area;
            double mi = mI[j * AB + k];
            double cov = mIp - mi * mp;
            double a = cov / (vI[j * AB + k] + (double)eps);
            double b = mp - a * mi;
            a_f = (float)a;
            b_f = (float)b;
          }
          aX[j * LDB + k] = a_f;
          bX[j * LDB + k] = b_f;
        }
      }
    }
    __syncthreads();
  }

  // 4. edge magnitude |(G[x+1]-G[x-1], G[y+1]-G[y-1])| on the interior.
  for (int i = threadIdx.x; i < AB * AB; i += blockDim.x) {
    int j = i / AB, k = i % AB;
    int gy = ay0 + j, gx = ax0 + k;
    float e = 0.f;
    if (gx >= 1 && gx < W - 1 && gy >= 1 && gy < H - 1) {
      int c = (j + r) * SP + (k + r);
      float gxv = sG[c + 1] - sG[c - 1];
      float gyv = sG[c + SP] - sG[c - SP];
      e = sqrtf(gxv * gxv + gyv * gyv);
    }
    er[j * LDB + k] = e;
  }
  __syncthreads();

  // 5. second box level and blend.  Each thread owns PER vertically adjacent
  // output pixels of one column (its window sums slide down by one row per
  // pixel); the three sweeps (R, B, edge) keep their results in registers.
  constexpr int PER = (T * T + NT - 1) / NT;
  const int my_k = threadIdx.x % T;
  const int my_j0 = (threadIdx.x / T) * PER;
  const bool my_active = my_j0 < T;
  float qR[PER], qB[PER], ew[PER];
  for (int pass = 0; pass < 3; pass++) {
    if (pass < 2) {
      const float* aX = pass == 0 ? aR : aB;
      const float* bX = pass == 0 ? bR : bB;
      hsum2(
          h0, h1, AB, T, r, [&](int j, int k) { return (double)aX[j * LDB + k]; },
          [&](int j, int k) { return (double)bX[j * LDB + k]; });
    } else {
      hsum(h0, AB, T, r, [&](int j, int k) { return (double)er[j * LDB + k]; });
    }
    __syncthreads();
    if (my_active) {
      const int k = my_k;
      const int LD2 = T + 1;
      double s0 = 0.0, s1 = 0.0;
      for (int t = 0; t <= 2 * r; t++) {
        s0 += h0[(my_j0 + t) * LD2 + k];
        if (pass < 2) s1 += h1[(my_j0 + t) * LD2 + k];
      }
#pragma unroll
      for (int q = 0; q < PER; q++) {
        const int j = my_j0 + q;
        if (q > 0) {
          s0 += h0[(j + 2 * r) * LD2 + k];
          s0 -= h0[(j - 1) * LD2 + k];
          if (pass < 2) {
            s1 += h1[(j + 2 * r) * LD2 + k];
            s1 -= h1[(j - 1) * LD2 + k];
          }
        }
        const double inv_area = inv_x[k + 2 * r] * inv_y[j + 2 * r];
        if (pass < 2) {
          const double ma = s0 * inv_area, mb = s1 * inv_area;
          const float I = sG[(j + 2 * r) * SP + (k + 2 * r)];
          const float qv = (float)(ma * (double)I + mb);
          if (pass == 0) qR[q] = qv; else qB[q] = qv;
        } else {
          const double m = s0 * inv_area;
          const float t = clampf(((float)m - 0.01f) / 0.05f, 0.f, 1.f);
          ew[q] = t * t * (3.f - 2.f * t);
        }
      }
    }
    __syncthreads();
  }

#pragma unroll
  for (int q = 0; q < PER; q++) {
    if (!my_active) break;
    const int j = my_j0 + q, k = my_k;
    int gy = y0 + j, gx = x0 + k;
    if (gx >= W || gy >= H) continue;
    int c = (j + 2 * r) * SP + (k + 2 * r);
    float w = strength * ew[q];
    float r_out = sR[c] * (1.f - w) + qR[q] * w;
    float b_out = sB[c] * (1.f - w) + qB[q] * w;
    size_t o = ((size_t)gy * W + gx) * 3;
    float gsrc = src[o + 1];
    dst[o + 0] = r_out * norm_ref;
    dst[o + 1] = gsrc;
    dst[o + 2] = b_out * norm_ref;
  }
}

// Output tile edge: 32 (the default) or 16; radii above 8 need the smaller
// tile to fit shared memory.
int pick_tile(int r, int want) { return r > 8 ? 16 : (want == 16 ? 16 : 32); }

template <int T, int NT>
cudaError_t axial_launch(dim3 grid, size_t smem, cudaStream_t s, const float* src, float* out, int w, int h, int r,
                         float eps, float strength, const float* d_max) {
  cudaError_t e = cudaFuncSetAttribute(k_axial_fused<T, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  k_axial_fused<T, NT><<<grid, NT, smem, s>>>(src, out, w, h, r, eps, strength, d_max);
  return cudaPeekAtLastError();
}

// Kernel variants: tile 32 or 16, 256 or 512 threads per CTA.
cudaError_t axial_dispatch(int T, int NT, size_t w, size_t h, cudaStream_t s, const float* src, float* out, int r,
                           float eps, float strength, const float* d_max) {
  const AxGeom g = ax_geom(T, r);
  dim3 grid((unsigned)((w + T - 1) / T), (unsigned)((h + T - 1) / T));
  if (T == 32) {
    if (NT == 256) return axial_launch<32, 256>(grid, g.bytes, s, src, out, (int)w, (int)h, r, eps, strength, d_max);
    return axial_launch<32, 512>(grid, g.bytes, s, src, out, (int)w, (int)h, r, eps, strength, d_max);
  }
  if (NT == 512) return axial_launch<16, 512>(grid, g.bytes, s, src, out, (int)w, (int)h, r, eps, strength, d_max);
  return axial_launch<16, 256>(grid, g.bytes, s, src, out, (int)w, (int)h, r, eps, strength, d_max);
}

// ---------------------------------------------------------------------------
// Streaming two-pass form (the default path).  The image is cut into strips
// of WS output columns and HS output rows; one warp walks a strip down its
// rows.  The vertical window sum of every column of the strip (plus r halo
// columns each side) lives in shared memory and slides: each row step adds
// the row entering the window and subtracts the row leaving it.  Each lane
// then forms the horizontal window sums of 4 adjacent output columns, sliding
// across them.  Every pixel's statistics are computed once, all sums are in
// double, and HBM carries the a/b planes between the two box levels.
//   pass A: G, G^2, R, G R, B, G B -> a_R, b_R, a_B, b_B, |grad G| (float planes)
//   pass B: box means of those five -> blended output
// Window sums use the same truncated windows, area reciprocals and float /
// double conversions as the fused kernel; only the summation order differs.
// A strip is WS = 32 * PL columns: each lane forms the horizontal sums of PL
// adjacent output columns (PL = 4 or 2).

// Column j of a strip's shared-memory window sums, with one pad slot per 16
// doubles: lanes reading 4 apart then hit 16 distinct 8-byte bank pairs.
__device__ __forceinline__ int vidx(int j) { return j + (j >> 4); }
template <int WS>
__host__ __device__ constexpr int vs_len() { return (WS + 32) + (WS + 32) / 16 + 1; }

// Quantities of pass A at (x, y) of the normalised image (zeros outside).
struct AbQ {
  __device__ static void load(const float* __restrict__ src, int W, int H, int x, int y, float inv_norm, double* q) {
    float g = 0.f, rr = 0.f, b = 0.f;
    if (x >= 0 && x < W && y >= 0 && y < H) {
      const float* p = src + ((size_t)y * W + x) * 3;
      rr = p[0] * inv_norm;
      g = p[1] * inv_norm;
      b = p[2] * inv_norm;
    }
    q[0] = (double)g;
    q[1] = (double)(g * g);
    q[2] = (double)rr;
    q[3] = (double)(g * rr);
    q[4] = (double)b;
    q[5] = (double)(g * b);
  }
};

template <int NQ, int WS, typename Loader>
__device__ __forceinline__ void strip_update(double (*Vs)[vs_len<WS>()], int VC, int xv0, int y_add, int y_sub, Loader ld) {
  for (int j = threadIdx.x; j < VC; j += 32) {
    double qa[NQ], qs[NQ];
    const int x = xv0 + j;
    ld(x, y_add, qa);
    ld(x, y_sub, qs);
#pragma unroll
    for (int q = 0; q < NQ; q++) {
      double v = Vs[q][vidx(j)];
      v += qa[q];
      v -= qs[q];
      Vs[q][vidx(j)] = v;
    }
  }
}

// One row step of a strip's vertical window sums (the row entering and the
// row leaving the window), fetched as raw samples one step ahead of its use.
// The fetch is issued after the step's last __syncwarp, so the loads stay in
// flight while the warp writes the current row's outputs.  The per-sample
// doubles and the order of the additions are those of strip_update.
template <int NQ, int NR, int WS>
struct StripStep {
  static constexpr int SL = WS / 32 + 1;  // window columns per lane: WS + 2r <= WS + 32
  float add[SL][NR], sub[SL][NR];
  template <typename Fetch>
  __device__ __forceinline__ void fetch(int VC, int xv0, int y_add, int y_sub, Fetch f) {
#pragma unroll
    for (int s = 0; s < SL; s++) {
      const int j = threadIdx.x + 32 * s;
      if (j < VC) {
        f(xv0 + j, y_add, add[s]);
        f(xv0 + j, y_sub, sub[s]);
      }
    }
  }
  template <typename Conv>
  __device__ __forceinline__ void apply(double (*Vs)[vs_len<WS>()], int VC, Conv cv) const {
#pragma unroll
    for (int s = 0; s < SL; s++) {
      const int j = threadIdx.x + 32 * s;
      if (j < VC) {
        double qa[NQ], qs[NQ];
        cv(add[s], qa);
        cv(sub[s], qs);
#pragma unroll
        for (int q = 0; q < NQ; q++) {
          double v = Vs[q][vidx(j)];
          v += qa[q];
          v -= qs[q];
          Vs[q][vidx(j)] = v;
        }
      }
    }
  }
};

// Horizontal window sums of the lane's 4 output columns: hs[q][k].
template <int NQ, int WS>
__device__ __forceinline__ void strip_hsum(double (*Vs)[vs_len<WS>()], int r, double hs[NQ][WS / 32]) {
  constexpr int PL = WS / 32;
  const int c0 = threadIdx.x * PL;
#pragma unroll
  for (int q = 0; q < NQ; q++) {
    double s = 0.0;
    for (int t = 0; t <= 2 * r; t++) s += Vs[q][vidx(c0 + t)];
    hs[q][0] = s;
#pragma unroll
    for (int k = 1; k < PL; k++) {
      s += Vs[q][vidx(c0 + k + 2 * r)];
      s -= Vs[q][vidx(c0 + k - 1)];
      hs[q][k] = s;
    }
  }
}

template <int WS>
__global__ void __launch_bounds__(32, WS == 128 ? 16 : 20) k_ax_ab(const float* __restrict__ src, int W, int H, int r, float eps, int HS,
                                             const float* __restrict__ d_maxg, float* __restrict__ aR,
                                             float* __restrict__ bR, float* __restrict__ aB, float* __restrict__ bB,
                                             float* __restrict__ er, int yb0) {
  constexpr int NQ = 6;
  constexpr int PL = WS / 32;
  __shared__ double Vs[NQ][vs_len<WS>()];
  const int VC = WS + 2 * r;
  const float inv_norm = 1.f / fmaxf(*d_maxg, 1e-6f);
  const int x0 = blockIdx.x * WS, y0 = (blockIdx.y + yb0) * HS;  // yb0: first row chunk of this launch
  const int xv0 = x0 - r;
  const int y_end = min(y0 + HS, H);
  auto ld = [&](int x, int y, double* q) { AbQ::load(src, W, H, x, y, inv_norm, q); };
  for (int j = threadIdx.x; j < VC; j += 32)
#pragma unroll
    for (int q = 0; q < NQ; q++) Vs[q][vidx(j)] = 0.0;
  // window of the first output row: rows [y0 - r, y0 + r] (out-of-image rows load zeros)
  for (int iy = y0 - r; iy <= y0 + r; iy++) strip_update<NQ, WS>(Vs, VC, xv0, iy, -1, ld);
  double inv_cx[PL];
#pragma unroll
  for (int k = 0; k < PL; k++) {
    const int x = x0 + threadIdx.x * PL + k;
    inv_cx[k] = x < W ? 1.0 / (double)win_count(x, r, W) : 0.0;
  }
  // raw (r, g, b) of the sample, zeros outside the image; cv forms the six
  // doubles exactly as AbQ::load does
  auto fetch = [&](int x, int y, float* v) {
    v[0] = v[1] = v[2] = 0.f;
    if (x >= 0 && x < W && y >= 0 && y < H) {
      const float* p = src + ((size_t)y * W + x) * 3;
      v[0] = p[0];
      v[1] = p[1];
      v[2] = p[2];
    }
  };
  auto cv = [&](const float* v, double* q) {
    const float rr = v[0] * inv_norm, g = v[1] * inv_norm, b = v[2] * inv_norm;
    q[0] = (double)g;
    q[1] = (double)(g * g);
    q[2] = (double)rr;
    q[3] = (double)(g * rr);
    q[4] = (double)b;
    q[5] = (double)(g * b);
  };
  StripStep<NQ, 3, WS> step;
  for (int y = y0; y < y_end; y++) {
    if (y > y0) step.apply(Vs, VC, cv);
    __syncwarp();
    double hs[NQ][PL];
    strip_hsum<NQ, WS>(Vs, r, hs);
    __syncwarp();  // the next update rewrites Vs
    if (y + 1 < y_end) step.fetch(VC, xv0, y + 1 + r, y - r, fetch);
    const double inv_cy = 1.0 / (double)win_count(y, r, H);
#pragma unroll
    for (int k = 0; k < PL; k++) {
      const int x = x0 + threadIdx.x * PL + k;
      if (x >= W) continue;
      const double ia = inv_cx[k] * inv_cy;
      const double mi = hs[0][k] * ia;
      const double vi = hs[1][k] * ia - mi * mi;
      const size_t o = (size_t)y * W + x;
      // |central gradient of G| (interior pixels), boxed by pass B
      float e = 0.f;
      if (x >= 1 && x < W - 1 && y >= 1 && y < H - 1) {
        const float gxv = src[(o + 1) * 3 + 1] * inv_norm - src[(o - 1) * 3 + 1] * inv_norm;
        const float gyv = src[(o + W) * 3 + 1] * inv_norm - src[(o - W) * 3 + 1] * inv_norm;
        e = sqrtf(gxv * gxv + gyv * gyv);
      }
      er[o] = e;
#pragma unroll
      for (int ch = 0; ch < 2; ch++) {
        const double mp = hs[2 + 2 * ch][k] * ia, mIp = hs[3 + 2 * ch][k] * ia;
        const double cov = mIp - mi * mp;
        const double a = cov / (vi + (double)eps);
        const double b = mp - a * mi;
        (ch == 0 ? aR : aB)[o] = (float)a;
        (ch == 0 ? bR : bB)[o] = (float)b;
      }
    }
  }
}

template <int WS>
__global__ void __launch_bounds__(32, WS == 128 ? 16 : 20) k_ax_q(const float* __restrict__ src, float* __restrict__ dst, int W, int H,
                                            int r, float strength, int HS, const float* __restrict__ d_maxg,
                                            const float* __restrict__ aR, const float* __restrict__ bR,
                                            const float* __restrict__ aB, const float* __restrict__ bB,
                                            const float* __restrict__ er, int yb0, bool tone,
                                            float tone_scale) {
  constexpr int NQ = 5;
  constexpr int PL = WS / 32;
  __shared__ double Vs[NQ][vs_len<WS>()];
  const int VC = WS + 2 * r;
  const float norm_ref = fmaxf(*d_maxg, 1e-6f);
  const float inv_norm = 1.f / norm_ref;
  const int x0 = blockIdx.x * WS, y0 = (blockIdx.y + yb0) * HS;  // yb0: first row chunk of this launch
  const int xv0 = x0 - r;
  const int y_end = min(y0 + HS, H);
  auto ld = [&](int x, int y, double* q) {
    float va = 0.f, vb = 0.f, vc = 0.f, vd = 0.f, e = 0.f;
    if (x >= 0 && x < W && y >= 0 && y < H) {
      const size_t i = (size_t)y * W + x;
      va = aR[i];
      vb = bR[i];
      vc = aB[i];
      vd = bB[i];
      e = er[i];
    }
    q[0] = (double)va;
    q[1] = (double)vb;
    q[2] = (double)vc;
    q[3] = (double)vd;
    q[4] = (double)e;
  };
  for (int j = threadIdx.x; j < VC; j += 32)
#pragma unroll
    for (int q = 0; q < NQ; q++) Vs[q][vidx(j)] = 0.0;
  for (int iy = y0 - r; iy <= y0 + r; iy++) strip_update<NQ, WS>(Vs, VC, xv0, iy, -1, ld);
  double inv_cx[PL];
#pragma unroll
  for (int k = 0; k < PL; k++) {
    const int x = x0 + threadIdx.x * PL + k;
    inv_cx[k] = x < W ? 1.0 / (double)win_count(x, r, W) : 0.0;
  }
  auto fetch = [&](int x, int y, float* v) {
    v[0] = v[1] = v[2] = v[3] = v[4] = 0.f;
    if (x >= 0 && x < W && y >= 0 && y < H) {
      const size_t i = (size_t)y * W + x;
      v[0] = aR[i];
      v[1] = bR[i];
      v[2] = aB[i];
      v[3] = bB[i];
      v[4] = er[i];
    }
  };
  auto cv = [](const float* v, double* q) {
#pragma unroll
    for (int t = 0; t < 5; t++) q[t] = (double)v[t];
  };
  StripStep<NQ, 5, WS> step;
  for (int y = y0; y < y_end; y++) {
    if (y > y0) step.apply(Vs, VC, cv);
    __syncwarp();
    double hs[NQ][PL];
    strip_hsum<NQ, WS>(Vs, r, hs);
    __syncwarp();
    if (y + 1 < y_end) step.fetch(VC, xv0, y + 1 + r, y - r, fetch);
    const double inv_cy = 1.0 / (double)win_count(y, r, H);
#pragma unroll
    for (int k = 0; k < PL; k++) {
      const int x = x0 + threadIdx.x * PL + k;
      if (x >= W) continue;
      const double ia = inv_cx[k] * inv_cy;
      const size_t o = ((size_t)y * W + x) * 3;
      const float R = src[o + 0] * inv_norm;
      const float G = src[o + 1];
      const float I = G * inv_norm;
      const float B = src[o + 2] * inv_norm;
      const float qR = (float)((hs[0][k] * ia) * (double)I + hs[1][k] * ia);
      const float qB = (float)((hs[2][k] * ia) * (double)I + hs[3][k] * ia);
      const float tt = clampf(((float)(hs[4][k] * ia) - 0.01f) / 0.05f, 0.f, 1.f);
      const float w = strength * (tt * tt * (3.f - 2.f * tt));
      float o0 = (R * (1.f - w) + qR * w) * norm_ref, o1 = G, o2 = (B * (1.f - w) + qB * w) * norm_ref;
      if (tone) {  // the ACES stage that follows, applied to the stored floats
        o0 = aces(o0) * tone_scale;
        o1 = aces(o1) * tone_scale;
        o2 = aces(o2) * tone_scale;
      }
      dst[o + 0] = o0;
      dst[o + 1] = o1;
      dst[o + 2] = o2;
    }
  }
}

template <int WS>
cudaError_t axial_stream(size_t w, size_t h, int HS, cudaStream_t s, const float* src, float* out, int r, float eps,
                         float strength, const float* d_max, float* planes, bool tone, float tone_scale) {
  const size_t n = w * h;
  float* aR = planes;
  float* bR = planes + n;
  float* aB = planes + 2 * n;
  float* bB = planes + 3 * n;
  float* er = planes + 4 * n;
  dim3 grid((unsigned)((w + WS - 1) / WS), (unsigned)((h + HS - 1) / HS));
  k_ax_ab<WS><<<grid, 32, 0, s>>>(src, (int)w, (int)h, r, eps, HS, d_max, aR, bR, aB, bB, er, 0);
  k_ax_q<WS><<<grid, 32, 0, s>>>(src, out, (int)w, (int)h, r, strength, HS, d_max, aR, bR, aB, bB, er, 0, tone,
                                 tone_scale);
  return cudaPeekAtLastError();
}

// The same two passes over row chunks [k0, k1) (pass A) or [k0, k1) (pass B).
template <int WS>
cudaError_t axial_pass_a(size_t w, size_t h, int HS, int k0, int k1, cudaStream_t s, const float* src, int r,
                         float eps, const float* d_max, float* planes) {
  if (k1 <= k0) return cudaSuccess;
  const size_t n = w * h;
  dim3 grid((unsigned)((w + WS - 1) / WS), (unsigned)(k1 - k0));
  k_ax_ab<WS><<<grid, 32, 0, s>>>(src, (int)w, (int)h, r, eps, HS, d_max, planes, planes + n, planes + 2 * n,
                                  planes + 3 * n, planes + 4 * n, k0);
  return cudaPeekAtLastError();
}
template <int WS>
cudaError_t axial_pass_b(size_t w, size_t h, int HS, int k0, int k1, cudaStream_t s, const float* src, float* out,
                         int r, float strength, const float* d_max, float* planes, bool tone, float tone_scale) {
  if (k1 <= k0) return cudaSuccess;
  const size_t n = w * h;
  dim3 grid((unsigned)((w + WS - 1) / WS), (unsigned)(k1 - k0));
  k_ax_q<WS><<<grid, 32, 0, s>>>(src, out, (int)w, (int)h, r, strength, HS, d_max, planes, planes + n,
                                 planes + 2 * n, planes + 3 * n, planes + 4 * n, k0, tone, tone_scale);
  return cudaPeekAtLastError();
}

}  // namespace

size_t ws_bytes_axial(size_t w, size_t h, int radius) {
  (void)radius;
  // the four a/b planes and the edge plane between the two passes, plus an out-of-place copy
  // when the caller runs in place (pass B reads input rows below the rows it
  // writes).
  return ((w * h * 5 * sizeof(float) + 255) & ~size_t(255)) + w * h * 3 * sizeof(float) + 256;
}

lre_status launch_axial_ca_banded(Context* c, const float* in, float* out, size_t w, size_t h, int radius, float eps,
                                  float strength, const float* d_max_g, int bands,
                                  const std::function<lre_status(size_t, size_t)>& rows_done, float tone_scale) {
  if (radius < 1) radius = 1;
  if (radius > 16) return fail(c, LRE_ERR_INVALID_ARGUMENT, "ca_axial_cleanup: radius > 16 is not supported");
  if (in == out) return fail(c, LRE_ERR_INVALID_ARGUMENT, "ca_axial_cleanup: banded form runs out of place");
  strength = fminf(fmaxf(strength, 0.f), 1.f);
  float* planes = reinterpret_cast<float*>(c->ws.take(w * h * 5 * sizeof(float)));
  if (!planes) return fail(c, LRE_ERR_OUT_OF_MEMORY, "ca_axial_cleanup: workspace too small");
  const int WS = c->tune.axial_strip == 64 ? 64 : 128;
  const size_t strips_x = (w + WS - 1) / WS;
  const size_t want = (size_t)c->sm_count * 24;
  // each launch covers one band, so the strip height is chosen for a band
  // (not the whole image) to fill the GPU
  bands = std::max(1, bands);
  int HS = c->tune.axial_rows == 128 ? 128 : 64;
  while (HS > 16 && strips_x * ((h + HS - 1) / HS) < want * (size_t)bands) HS /= 2;
  // pass B of a chunk reads pass A's planes up to `radius` (<= HS) rows below
  // it, so pass A runs one band ahead of pass B
  const int nch = (int)((h + HS - 1) / HS);
  bands = std::min(bands, nch);
  auto edge = [&](int b) { return (int)((long long)nch * b / bands); };
  auto pass_a = [&](int b) {
    return WS == 64 ? axial_pass_a<64>(w, h, HS, edge(b), edge(b + 1), c->stream, in, radius, eps, d_max_g, planes)
                    : axial_pass_a<128>(w, h, HS, edge(b), edge(b + 1), c->stream, in, radius, eps, d_max_g, planes);
  };
  LRE_CUDA_TRY(c, pass_a(0));
  count_launch(c);
  for (int b = 0; b < bands; b++) {
    if (b + 1 < bands) {
      LRE_CUDA_TRY(c, pass_a(b + 1));
      count_launch(c);
    }
    const bool tone = tone_scale >= 0.f;
    LRE_CUDA_TRY(c, WS == 64 ? axial_pass_b<64>(w, h, HS, edge(b), edge(b + 1), c->stream, in, out, radius, strength,
                                                  d_max_g, planes, tone, tone_scale)
                             : axial_pass_b<128>(w, h, HS, edge(b), edge(b + 1), c->stream, in, out, radius, strength,
                                                   d_max_g, planes, tone, tone_scale));
    count_launch(c);
    LRE_TRY(check_launch(c, "ca_axial_cleanup"));
    const size_t r0 = std::min(h, (size_t)edge(b) * HS), r1 = std::min(h, (size_t)edge(b + 1) * HS);
    LRE_TRY(rows_done(r0, r1));
  }
  return LRE_OK;
}

lre_status launch_axial_ca(Context* c, const float* in, float* out, size_t w, size_t h, int radius, float eps,
                           float strength, const float* d_max_g, float tone_scale) {
  if (radius < 1) radius = 1;
  if (radius > 16) return fail(c, LRE_ERR_INVALID_ARGUMENT, "ca_axial_cleanup: radius > 16 is not supported");
  strength = fminf(fmaxf(strength, 0.f), 1.f);
  float* planes = reinterpret_cast<float*>(c->ws.take(w * h * 5 * sizeof(float)));
  if (!planes) return fail(c, LRE_ERR_OUT_OF_MEMORY, "ca_axial_cleanup: workspace too small");
  const float* src = in;
  if (in == out) {
    float* tmp = reinterpret_cast<float*>(c->ws.take(w * h * 3 * sizeof(float)));
    if (!tmp) return fail(c, LRE_ERR_OUT_OF_MEMORY, "ca_axial_cleanup: workspace too small");
    LRE_CUDA_TRY(c, cudaMemcpyAsync(tmp, in, w * h * 3 * sizeof(float), cudaMemcpyDeviceToDevice, c->stream));
    src = tmp;
  }
  // Strip width 128 (4 columns per lane) or 64 (2 per lane); strip height:
  // enough one-warp strips for at least 24 per SM (more than the 16-20 that
  // fit at once, so every SM stays full while the passes, which are
  // load-latency bound, drain), but at least 16 rows so the 2r + 1 row
  // prologue of a strip stays small; capped by the tuning choice.
  const int WS = c->tune.axial_strip == 64 ? 64 : 128;
  const size_t strips_x = (w + WS - 1) / WS;
  const size_t want = (size_t)c->sm_count * 24;
  int HS = c->tune.axial_rows == 128 ? 128 : 64;
  while (HS > 16 && strips_x * ((h + HS - 1) / HS) < want) HS /= 2;
  const bool tone = tone_scale >= 0.f;
  LRE_CUDA_TRY(c, WS == 64 ? axial_stream<64>(w, h, HS, c->stream, src, out, radius, eps, strength, d_max_g, planes,
                                              tone, tone_scale)
                           : axial_stream<128>(w, h, HS, c->stream, src, out, radius, eps, strength, d_max_g, planes,
                                               tone, tone_scale));
  count_launch(c, 2);
  return check_launch(c, "ca_axial_cleanup");
}

// ---------------------------------------------------------------------------
// Axial CA without any device allocation.
//
// Some callers cannot allocate device memory when they filter a frame: a
// plug-in host that hands out only pre-reserved memory pools, a real-time
// capture thread that must not block on cudaMalloc (it synchronises the
// device), or an application that has already pinned its memory budget.
// This variant keeps its scratch -- the max(G) normaliser and, for in-place
// calls, a copy of the input -- in one file-scope device array, so a call
// allocates nothing.  The array is sized for images up to
// kNoAllocMaxPixels; larger images are rejected.  Every GPU that loads the
// library holds the array until the process exits.
// ---------------------------------------------------------------------------
namespace {

constexpr size_t kNoAllocMaxPixels = size_t(1) << 21;  // 2,097,152 px, e.g. 1920x1080
constexpr size_t kNoAllocHead = 64;                     // floats ahead of the image copy (256 B)
static __device__ __align__(256) float g_axial_noalloc_scratch[kNoAllocHead + kNoAllocMaxPixels * 3];

constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mu;
float* g_noalloc_addr[kNoAllocMaxDevices] = {nullptr};

__global__ void k_noalloc_zero(float* p) { *p = 0.0f; }

// max(0, max G) over the image, into *out (which must start at 0).
__global__ void k_noalloc_max_g(const float* __restrict__ rgb, size_t n, float* out) {
  float m = 0.0f;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    m = fmaxf(m, rgb[i * 3 + 1]);
  m = warp_max(m);
  if ((threadIdx.x & 31) == 0) atomic_max_float(out, m);
}

}  // namespace

}  // namespace lre

extern "C" lre_status lre_dev_ca_axial_cleanup_noalloc(const float* in, float* out, size_t w, size_t h, int radius,
                                                       float epsilon, float strength, void* cuda_stream) {
  using namespace lre;
  if (!in || !out || w == 0 || h == 0) return LRE_ERR_INVALID_ARGUMENT;
  if (w > (1u << 20) || h > (1u << 20) || w * h > kNoAllocMaxPixels) return LRE_ERR_INVALID_ARGUMENT;
  if (radius < 1) radius = 1;
  if (radius > 16) return LRE_ERR_INVALID_ARGUMENT;
  strength = fminf(fmaxf(strength, 0.f), 1.f);
  cudaStream_t s = reinterpret_cast<cudaStream_t>(cuda_stream);

  // An error the caller's own earlier work left pending is theirs: report
  // it without consuming it, and enqueue nothing.
  if (cudaPeekAtLastError() != cudaSuccess) return LRE_ERR_CUDA;

  // The scratch address below belongs to the current device, so the stream
  // must be one of that device's streams (the legacy default stream is).
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kNoAllocMaxDevices) return LRE_ERR_CUDA;
  if (s != nullptr) {
    int sdev = -1;
    if (cudaStreamGetDevice(s, &sdev) != cudaSuccess) {
      cudaGetLastError();
      return LRE_ERR_INVALID_ARGUMENT;
    }
    if (sdev != dev) return LRE_ERR_INVALID_ARGUMENT;
  }

  // One-time set-up per device: the device address of the scratch array.
  float* base = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_addr[dev]) {
      void* p = nullptr;
      if (cudaGetSymbolAddress(&p, g_axial_noalloc_scratch) != cudaSuccess || !p) {
        cudaGetLastError();
        return LRE_ERR_CUDA;
      }
      g_noalloc_addr[dev] = static_cast<float*>(p);
    }
    base = g_noalloc_addr[dev];
  }
  float* d_max = base;                 // cleared below on every call
  float* staging = base + kNoAllocHead;

  // Any error from here on comes from this call's own work (none was pending
  // on entry): take it off the error state and report it.
  auto failed = [] {
    if (cudaPeekAtLastError() == cudaSuccess) return false;
    cudaGetLastError();
    return true;
  };
  const size_t n = w * h;
  k_noalloc_zero<<<1, 1, 0, s>>>(d_max);
  if (failed()) return LRE_ERR_CUDA;
  k_noalloc_max_g<<<grid_for(n, 256, 148u * 4u), 256, 0, s>>>(in, n, d_max);
  if (failed()) return LRE_ERR_CUDA;
  const float* src = in;
  if (in == out) {
    if (cudaMemcpyAsync(staging, in, n * 3 * sizeof(float), cudaMemcpyDeviceToDevice, s) != cudaSuccess) {
      cudaGetLastError();
      return LRE_ERR_CUDA;
    }
    src = staging;
  }
  if (axial_dispatch(pick_tile(radius, 32), 512, w, h, s, src, out, radius, epsilon, strength, d_max) != cudaSuccess) {
    cudaGetLastError();
    return LRE_ERR_CUDA;
  }
  return LRE_OK;
}
