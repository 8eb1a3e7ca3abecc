// k_xtrans.cu -- X-Trans demosaic: fast 1-pass interpolation and the 3-pass
// Markesteijn interpolation (RawTherapee's algorithm as ported in
// libraw_enhanced, YPbPr derivative variant), plus the X-Trans border fill.
//
// Semantics: core/cpu_accelerator.cpp:1664-2762 (XTrans_Processor):
//   xtrans_border_interpolate (:1806-1861), run_3pass (:1870-2676),
//   run_1pass (:2679-2762).
//
// 3-pass device design: the reference's 114 x 114 tiles (step 98, origin 3)
// are kept -- its homogeneity maps read outside the rows a tile computes at
// the first/last tile rows and columns, so the tiling is part of the result.
// One CTA runs one tile at a time; positions a tile reads without computing
// read zeros (a freshly allocated reference buffer).  Two kernels:
// * k_xtrans_3pass_planes, for every pattern whose row scans a host replay
//   reduces to "every site of the class" (the X-Trans layouts and their
//   shifts): one direction plane at a time in shared memory, every step one
//   site per thread;
// * k_xtrans_3pass, for any other pattern: the reference's row scans, one
//   row per thread in its column order, with the whole tile (8 directions x
//   114^2 RGB, derivatives, homogeneity maps) in a per-CTA global slab.
#include <cfloat>
#include <cstdlib>
#include <cstring>

#include "common.cuh"
#include "lre_internal.h"

namespace lre {

namespace {

constexpr int XTS = 114;
constexpr int NDIR = 8;
constexpr int XT_THREADS = 512;
constexpr int kXtCtasPerSm = 2;
constexpr int kXtMaxCtas = 148 * kXtCtasPerSm;

struct XtParams {
  char xt[6][6];
  short allhex0[3][3][8];
  short allhex1[3][3][8];
  int sgrow, sgcol;
  int right_shift[3];
};

struct XtArgs {
  const float* raw;
  const float* norm;  // dense raw / maximum (plane-resident kernel)
  int cstride;
  float* rgb_out;
  int W, H;
  float maximum;
  int n_top, n_left;
  unsigned char* scratch;
  int* tile_counter;
  XtParams P;
};

struct XtSlab {
  float* rgb;           // [NDIR][XTS][XTS][3]
  float2* gmm;          // [XTS][XTS/2] (min, max)
  float* drv;           // [NDIR][XTS-10][XTS-10]
  unsigned char* homo;  // [NDIR][XTS][XTS]
  unsigned char* homosum;
  unsigned char* homosummax;  // [XTS][XTS]
};

constexpr size_t kRgbBytes = (size_t)NDIR * XTS * XTS * 3 * 4;
constexpr size_t kGmmBytes = (size_t)XTS * (XTS / 2) * 8;
constexpr size_t kDrvBytes = (size_t)NDIR * (XTS - 10) * (XTS - 10) * 4;
constexpr size_t kHomoBytes = (size_t)NDIR * XTS * XTS;
constexpr size_t kHmaxBytes = (size_t)XTS * XTS;
constexpr size_t kXtSlabBytes = ((kRgbBytes + kGmmBytes + kDrvBytes + 2 * kHomoBytes + kHmaxBytes + 255) / 256) * 256;

__device__ XtSlab make_xt_slab(unsigned char* base) {
  XtSlab s;
  s.rgb = reinterpret_cast<float*>(base);
  base += kRgbBytes;
  s.gmm = reinterpret_cast<float2*>(base);
  base += kGmmBytes;
  s.drv = reinterpret_cast<float*>(base);
  base += kDrvBytes;
  s.homo = base;
  base += kHomoBytes;
  s.homosum = base;
  base += kHomoBytes;
  s.homosummax = base;
  return s;
}

__device__ __forceinline__ int xfc(const XtParams& P, int row, int col) { return P.xt[(row + 6) % 6][(col + 6) % 6]; }
__device__ __forceinline__ int xisgreen(const XtParams& P, int row, int col) { return P.xt[row % 3][col % 3] & 1; }

__device__ __forceinline__ float xraw(const XtArgs& A, int row, int col) {
  const size_t i = (size_t)row * A.W + col;
  const float v = A.cstride == 1 ? A.raw[i] : A.raw[i * 3 + xfc(A.P, row, col)];
  return v / A.maximum;
}
// raw_buffer_hex (:1691-1695): linear offset from (row, col), colour of the
// landing site.
__device__ __forceinline__ float xraw_hex(const XtArgs& A, int row, int col, int hex) {
  const long long pos = (long long)row * A.W + col + hex;
  float v;
  if (A.cstride == 1) {
    v = A.raw[pos];
  } else {  // the landing site's colour needs its (row, col)
    const int r = (int)(pos / A.W), c = (int)(pos % A.W);
    v = A.raw[pos * 3 + xfc(A.P, r, c)];
  }
  return v / A.maximum;
}

// The same samples from the dense normalised mosaic (k_xt_normalize): the
// value at (row, col), and at a linear offset from it.
__device__ __forceinline__ float xn(const XtArgs& A, int row, int col) { return A.norm[(size_t)row * A.W + col]; }
__device__ __forceinline__ float xn_hex(const XtArgs& A, int row, int col, int hex) {
  return A.norm[(long long)row * A.W + col + hex];
}

// n / d by a multiply-high, exact while n * d < 2^32 (every loop here); the
// per-site loops map a flat index to (row, column) every iteration.
struct XDiv {
  unsigned m;
  int d;
  __device__ explicit XDiv(int d_) : m(d_ > 1 ? 0xFFFFFFFFu / (unsigned)d_ + 1u : 0u), d(d_) {}
  __device__ __forceinline__ int div(int n) const { return (int)__umulhi((unsigned)n, m) + (d == 1 ? n : 0); }
};

// std::max(low, std::min(val, high)) -- LIM of core/metal/shader_common.h.
__device__ __forceinline__ float LIMf(float val, float low, float high) {
  float m = (high < val) ? high : val;
  return (low < m) ? m : low;
}
__device__ __forceinline__ float SQRf(float x) { return x * x; }

// --------------------------------------------------------- border fill
__device__ void xtrans_border_px(const XtArgs& A, int row, int col) {
  const float weight[3][3] = {{0.25f, 0.5f, 0.25f}, {0.5f, 0.f, 0.5f}, {0.25f, 0.5f, 0.25f}};
  const int W = A.W, H = A.H;
  float sum[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  int v = (row == 0) ? 0 : -1;
  for (int y = (row > 0) ? row - 1 : 0; y < row + 2 && y < H; y++, v++) {
    int h = (col == 0) ? 0 : -1;
    for (int x = (col > 0) ? col - 1 : 0; x < col + 2 && x < W; x++, h++) {
      const int f = xfc(A.P, y, x);
      sum[f] += xraw(A, y, x) * weight[v + 1][h + 1];
      sum[f + 3] += weight[v + 1][h + 1];
    }
  }
  float* o = A.rgb_out + ((size_t)row * W + col) * 3;
  switch (xfc(A.P, row, col)) {
    case 0:
      o[0] = xraw(A, row, col);
      o[1] = (sum[1] / sum[4]);
      o[2] = (sum[2] / sum[5]);
      break;
    case 1:
      if (sum[3] == 0.f) {
        const float r = xraw(A, row, col);
        o[0] = o[1] = o[2] = r;
      } else {
        o[0] = (sum[0] / sum[3]);
        o[1] = xraw(A, row, col);
        o[2] = (sum[2] / sum[5]);
      }
      break;
    case 2:
      o[0] = (sum[0] / sum[3]);
      o[1] = (sum[1] / sum[4]);
      o[2] = xraw(A, row, col);
      break;
  }
}

__global__ void k_xtrans_border(XtArgs A, int border) {
  const int W = A.W, H = A.H;
  const long long n_tb = 2LL * border * W;
  const long long n_lr = 2LL * border * (H - 2 * border > 0 ? H - 2 * border : 0);
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n_tb + n_lr; k += (long long)gridDim.x * blockDim.x) {
    int row, col;
    if (k < n_tb) {
      const int b = (int)(k / W);
      col = (int)(k % W);
      row = b < border ? b : H - 2 * border + b;
    } else {
      const long long q = k - n_tb;
      const int b = (int)(q % (2 * border));
      row = border + (int)(q / (2 * border));
      col = b < border ? b : W - 2 * border + b;
    }
    if (row < 0 || row >= H || col < 0 || col >= W) continue;
    if (col >= border && col < W - border && row >= border && row < H - border) continue;
    xtrans_border_px(A, row, col);
  }
}

// --------------------------------------------------------- 1-pass (:2679-2762)
__global__ void k_xtrans_1pass(XtArgs A) {
  const float weight[3][3] = {{0.25f, 0.5f, 0.25f}, {0.5f, 0.0f, 0.5f}, {0.25f, 0.5f, 0.25f}};
  const int W = A.W, H = A.H;
  const long long n = (long long)(H - 2) * (W - 2);
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    const int row = 1 + (int)(k / (W - 2)), col = 1 + (int)(k % (W - 2));
    float sum[3] = {0.f, 0.f, 0.f};
    for (int v = -1; v <= 1; v++)
      for (int h = -1; h <= 1; h++) {
        const int sr = row + v, sc = col + h;
        const int c = xfc(A.P, sr, sc);
        const float raw_val = xraw(A, sr, sc);
        sum[c] += raw_val * weight[v + 1][h + 1];
      }
    float rgb[3];
    switch (xfc(A.P, row, col)) {
      case 0:
        rgb[0] = xraw(A, row, col);
        rgb[1] = sum[1] * 0.5f;
        rgb[2] = sum[2];
        break;
      case 1: {
        rgb[1] = xraw(A, row, col);
        if (xfc(A.P, row, col - 1) == xfc(A.P, row, col + 1)) {
          rgb[0] = sum[0];
          rgb[2] = sum[2];
        } else {
          rgb[0] = sum[0] * 1.3333333f;
          rgb[2] = sum[2] * 1.3333333f;
        }
      } break;
      default:
        rgb[0] = sum[0];
        rgb[1] = sum[1] * 0.5f;
        rgb[2] = xraw(A, row, col);
        break;
    }
    float* o = A.rgb_out + ((size_t)row * W + col) * 3;
    o[0] = rgb[0];
    o[1] = rgb[1];
    o[2] = rgb[2];
  }
}

// --------------------------------------------------------- 3-pass
__global__ void __launch_bounds__(XT_THREADS, kXtCtasPerSm) k_xtrans_3pass(XtArgs Ain) {
  const int ts = XTS;
  const int tid = threadIdx.x, nth = blockDim.x;
  // The pattern tables are indexed at run time; read from the kernel's
  // parameter block that would force a local-memory copy of it per thread,
  // so one copy goes to shared memory (constant-offset parameter loads).
  __shared__ XtArgs sA;
  {
    constexpr int NW = (int)(sizeof(XtArgs) / 4);
    const int* from = reinterpret_cast<const int*>(&Ain);
    int* to = reinterpret_cast<int*>(&sA);
#pragma unroll
    for (int k = 0; k < NW; k++)
      if (k % XT_THREADS == tid) to[k] = from[k];
  }
  __syncthreads();
  const XtArgs& A = sA;
  const XtParams& P = A.P;
  XtSlab S = make_xt_slab(A.scratch + (size_t)blockIdx.x * kXtSlabBytes);
  __shared__ int s_tile;
  const int W = A.W, H = A.H;
  bool zeroed_once = false;

  for (;;) {
    if (tid == 0) s_tile = atomicAdd(A.tile_counter, 1);
    __syncthreads();
    const int tile = s_tile;
    __syncthreads();
    if (tile >= A.n_top * A.n_left) break;
    const int top = 3 + (tile / A.n_left) * (ts - 16);
    const int left = 3 + (tile % A.n_left) * (ts - 16);
    const int mrow_g = min(top + ts, H - 3);  // global row bound of the computations
    const int mcol_g = min(left + ts, W - 3);

    // Fresh scratch (zeros) for tiles on the image border: only their
    // outputs read positions the tile never computes (the homogeneity maps
    // of the first/last tile rows and columns).  Interior tiles clear only
    // direction plane 0, as the reference does for every tile; they write
    // every other position before reading it.
    const bool border_tile = tile / A.n_left == 0 || tile / A.n_left == A.n_top - 1 || tile % A.n_left == 0 ||
                             tile % A.n_left == A.n_left - 1;
    if (border_tile || !zeroed_once) {
      float4* z = reinterpret_cast<float4*>(S.rgb);
      const size_t n4 = kXtSlabBytes / 16;
      for (size_t i = tid; i < n4; i += nth) z[i] = make_float4(0.f, 0.f, 0.f, 0.f);
      zeroed_once = true;
    } else {
      // direction plane 0 is cleared for every tile (:2058)
      float4* z = reinterpret_cast<float4*>(S.rgb);
      for (int i = tid; i < XTS * XTS * 3 / 4; i += nth) z[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    __syncthreads();
    float* rgb = S.rgb;
    auto RGB = [&](int d, int lr, int lc) -> float* { return rgb + (((size_t)d * ts + lr) * ts + lc) * 3; };

    // (a) green min / max per row (:1968-2053), one row per thread
    for (int row = top + tid; row < mrow_g; row += nth) {
      int leftstart = left;
      for (; leftstart < mcol_g; leftstart++)
        if (!xisgreen(P, row, leftstart)) break;
      int coloffset = (P.right_shift[row % 3] == 1 ? 3 : 1 + (xfc(P, row, leftstart + 1) & 1));
      float2* g = S.gmm + (size_t)(row - top) * (ts / 2);
      auto mm = [&](int col, const short* hex) {
        float minval = FLT_MAX, maxval = 0.f;
        for (int c = 0; c < 6; c++) {
          const float val = xraw_hex(A, row, col, hex[c]);
          minval = minval < val ? minval : val;
          maxval = maxval > val ? maxval : val;
        }
        return make_float2(minval, maxval);
      };
      if (coloffset == 3) {
        const short* hex = P.allhex0[row % 3][leftstart % 3];
        for (int col = leftstart; col < mcol_g; col += coloffset) g[(col - left) >> 1] = mm(col, hex);
      } else {
        int col = leftstart;
        if (coloffset == 2) {
          const short* hex = P.allhex0[row % 3][col % 3];
          g[(col - left) >> 1] = mm(col, hex);
          col += 2;
        }
        const short* hex = P.allhex0[row % 3][col % 3];
        for (; col < mcol_g - 1; col += 3) {
          const float2 v = mm(col, hex);
          g[(col - left) >> 1] = v;
          g[(col + 1 - left) >> 1] = v;
        }
        if (col < mcol_g) g[(col - left) >> 1] = mm(col, hex);
      }
    }
    // native samples into direction 0 (:2055-2061)
    const XDiv fdn(mcol_g - left);
    for (int i = tid; i < (mrow_g - top) * (mcol_g - left); i += nth) {
      const int lr = fdn.div(i), lc = i - lr * (mcol_g - left);
      const int row = top + lr, col = left + lc;
      RGB(0, lr, lc)[xfc(P, row, col)] = xraw(A, row, col);
    }
    __syncthreads();
    // copy direction 0 to 1..3, all but the last float (:2067-2069); the
    // planes are 16-byte aligned (ts*ts*3 floats apart), so 4 floats a step
    {
      constexpr int NF = XTS * XTS * 3 - 1;
      const float4* s4 = reinterpret_cast<const float4*>(rgb);
      for (int i = tid; i < NF / 4; i += nth) {
        const float4 v = s4[i];
        reinterpret_cast<float4*>(rgb + (size_t)1 * XTS * XTS * 3)[i] = v;
        reinterpret_cast<float4*>(rgb + (size_t)2 * XTS * XTS * 3)[i] = v;
        reinterpret_cast<float4*>(rgb + (size_t)3 * XTS * XTS * 3)[i] = v;
      }
      for (int i = (NF / 4) * 4 + tid; i < NF; i += nth) {
        const float v = rgb[i];
        rgb[(size_t)1 * XTS * XTS * 3 + i] = v;
        rgb[(size_t)2 * XTS * XTS * 3 + i] = v;
        rgb[(size_t)3 * XTS * XTS * 3 + i] = v;
      }
    }
    __syncthreads();
    // (b) green in 4 directions (:2071-2127), one row per thread
    for (int row = top + tid; row < mrow_g; row += nth) {
      int leftstart = left;
      for (; leftstart < mcol_g; leftstart++)
        if (!xisgreen(P, row, leftstart)) break;
      int coloffset = (P.right_shift[row % 3] == 1 ? 3 : 1 + (xfc(P, row, leftstart + 1) & 1));
      const float2* g = S.gmm + (size_t)(row - top) * (ts / 2);
      auto colors = [&](int col, const short* hex, float* color) {
        color[0] = 0.6796875f * (xraw_hex(A, row, col, hex[1]) + xraw_hex(A, row, col, hex[0])) -
                   0.1796875f * (xraw_hex(A, row, col, 2 * hex[1]) + xraw_hex(A, row, col, 2 * hex[0]));
        color[1] = 0.87109375f * xraw_hex(A, row, col, hex[3]) + xraw_hex(A, row, col, hex[2]) * 0.12890625f +
                   0.359375f * (xraw_hex(A, row, col, 0) - xraw_hex(A, row, col, -hex[2]));
        for (int c = 0; c < 2; c++)
          color[2 + c] = 0.640625f * xraw_hex(A, row, col, hex[4 + c]) + 0.359375f * xraw_hex(A, row, col, -2 * hex[4 + c]) +
                         0.12890625f * (2.f * xraw_hex(A, row, col, 0) - xraw_hex(A, row, col, 3 * hex[4 + c]) -
                                        xraw_hex(A, row, col, -3 * hex[4 + c]));
      };
      if (coloffset == 3) {
        const short* hex = P.allhex0[row % 3][leftstart % 3];
        for (int col = leftstart; col < mcol_g; col += coloffset) {
          float color[4];
          colors(col, hex, color);
          const float2 mmv = g[(col - left) >> 1];
          for (int c = 0; c < 4; c++) RGB(c, row - top, col - left)[1] = LIMf(color[c], mmv.x, mmv.y);
        }
      } else {
        const short* hexmod[2] = {P.allhex0[row % 3][leftstart % 3], P.allhex0[row % 3][(leftstart + coloffset) % 3]};
        for (int col = leftstart, hexindex = 0; col < mcol_g; col += coloffset, coloffset ^= 3, hexindex ^= 1) {
          const short* hex = hexmod[hexindex];
          float color[4];
          colors(col, hex, color);
          const float2 mmv = g[(col - left) >> 1];
          for (int c = 0; c < 4; c++) RGB(c ^ 1, row - top, col - left)[1] = LIMf(color[c], mmv.x, mmv.y);
        }
      }
    }
    __syncthreads();

    for (int pass = 0; pass < 3; pass++) {
      if (pass == 1) {
        // copy directions 0..3 into 4..7, all but the last float (:2131-2136)
        constexpr int NF = 4 * XTS * XTS * 3 - 1;
        const float4* s4 = reinterpret_cast<const float4*>(S.rgb);
        float4* d4 = reinterpret_cast<float4*>(S.rgb + (size_t)4 * XTS * XTS * 3);
        for (int i = tid; i < NF / 4; i += nth) d4[i] = s4[i];
        for (int i = (NF / 4) * 4 + tid; i < NF; i += nth) S.rgb[(size_t)4 * XTS * XTS * 3 + i] = S.rgb[i];
        __syncthreads();
        rgb = S.rgb + (size_t)4 * ts * ts * 3;
      }
      // (c) recalculate green from closer pixels (:2138-2183)
      if (pass) {
        for (int row = top + 2 + tid; row < mrow_g - 2; row += nth) {
          int leftstart = left + 2;
          for (; leftstart < mcol_g - 2; leftstart++)
            if (!xisgreen(P, row, leftstart)) break;
          int coloffset = (P.right_shift[row % 3] == 1 ? 3 : 1 + (xfc(P, row, leftstart + 1) & 1));
          const float2* g = S.gmm + (size_t)(row - top) * (ts / 2);
          // A site's three directions write three different planes and
          // read only their own plane, so all fifteen operands are loaded
          // before the three stores; sites stay in the reference's order.
          auto site = [&](int col, int f, const short* hex, int flip) {
            float v[3][5];
#pragma unroll
            for (int d = 3; d < 6; d++) {
              const float* rix = RGB((d - 2) ^ flip, row - top, col - left);
              const int o1 = hex[d] * 3, o2 = -2 * hex[d] * 3;
              v[d - 3][0] = rix[o2 + 1];
              v[d - 3][1] = rix[o1 + 1];
              v[d - 3][2] = rix[o1 + f];
              v[d - 3][3] = rix[o2 + f];
              v[d - 3][4] = rix[f];
            }
            const float2 mmv = g[(col - left) >> 1];
#pragma unroll
            for (int d = 3; d < 6; d++) {
              const float* q = v[d - 3];
              const float val = 0.33333333f * (q[0] + 2 * (q[1] - q[2]) - q[3]) + q[4];
              RGB((d - 2) ^ flip, row - top, col - left)[1] = LIMf(val, mmv.x, mmv.y);
            }
          };
          if (coloffset == 3) {
            int f = xfc(P, row, leftstart);
            const short* hex = P.allhex1[row % 3][leftstart % 3];
            for (int col = leftstart; col < mcol_g - 2; col += coloffset, f ^= 2) site(col, f, hex, 0);
          } else {
            int f = xfc(P, row, leftstart);
            const short* hexmod[2] = {P.allhex1[row % 3][leftstart % 3], P.allhex1[row % 3][(leftstart + coloffset) % 3]};
            for (int col = leftstart, hexindex = 0; col < mcol_g - 2;
                 col += coloffset, coloffset ^= 3, f = f ^ (coloffset & 2), hexindex ^= 1)
              site(col, f, hexmod[hexindex], 1);
          }
        }
        __syncthreads();
      }
      // (d) R/B at solitary green pixels (:2185-2222)
      {
        const int sgstartcol = (left - P.sgcol + 4) / 3 * 3 + P.sgcol;
        const int row0 = (top - P.sgrow + 4) / 3 * 3 + P.sgrow;
        // One solitary green per thread: along a row the scan toggles h once
        // per site (its inner loops toggle it an even number of times), so
        // the k-th site starts from h0 ^ 2 (k & 1); sites are independent.
        const int nrow = row0 < mrow_g - 2 ? (mrow_g - 2 - row0 + 2) / 3 : 0;
        const int ncol = sgstartcol < mcol_g - 2 ? (mcol_g - 2 - sgstartcol + 2) / 3 : 0;
        for (int item = tid; item < nrow * ncol; item += nth) {
          const int row = row0 + 3 * (item / ncol), k = item % ncol;
          const int col = sgstartcol + 3 * k;
          float color[3][6];
          {
            int h = xfc(P, row, sgstartcol + 1) ^ ((k & 1) << 1);
            float* rix = RGB(0, row - top, col - left);
            float diff[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
            for (int i = 1, d = 0; d < 6; d++, i ^= ts ^ 1, h ^= 2) {
              for (int c = 0; c < 2; c++, h ^= 2) {
                const int op = i * (1 << c) * 3, om = -i * (1 << c) * 3;
                const float g = rix[1] + rix[1] - rix[op + 1] - rix[om + 1];
                color[h][d] = g + rix[op + h] + rix[om + h];
                if (d > 1) diff[d] += SQRf(rix[op + 1] - rix[om + 1] - rix[op + h] + rix[om + h]) + SQRf(g);
              }
              if (d > 2 && (d & 1))
                if (diff[d - 1] < diff[d])
                  for (int c = 0; c < 2; c++) color[c * 2][d] = color[c * 2][d - 1];
              if ((d & 1) || d < 2) {
                for (int c = 0; c < 2; c++) rix[c * 2] = 0.5f * color[c * 2][d];
                rix += (size_t)ts * ts * 3;
              }
            }
          }
        }
      }
      __syncthreads();
      // (e) red for blue pixels and vice versa (:2224-2264), one row per
      // thread in the reference's column order
      for (int row = top + 3 + tid; row < mrow_g - 3; row += nth) {
        int leftstart = left + 3;
        for (; leftstart < mcol_g - 1; leftstart++)
          if (!xisgreen(P, row, leftstart)) break;
        int coloffset = (P.right_shift[row % 3] == 1 ? 3 : 1);
        const int c = ((row - P.sgrow) % 3) ? ts : 1;
        const int h = 3 * (c ^ ts ^ 1);
        auto body = [&](int col, int f) {
          float* rix = RGB(0, row - top, col - left);
          for (int d = 0; d < 4; d++, rix += (size_t)ts * ts * 3) {
            const int i = d > 1 || ((d ^ c) & 1) ||
                                  ((fabsf(rix[1] - rix[c * 3 + 1]) + fabsf(rix[1] - rix[-c * 3 + 1])) <
                                   2.f * (fabsf(rix[1] - rix[h * 3 + 1]) + fabsf(rix[1] - rix[-h * 3 + 1])))
                              ? c
                              : h;
            rix[f] = rix[1] + 0.5f * (rix[i * 3 + f] + rix[-i * 3 + f] - rix[i * 3 + 1] - rix[-i * 3 + 1]);
          }
        };
        if (coloffset == 3) {
          int f = 2 - xfc(P, row, leftstart);
          for (int col = leftstart; col < mcol_g - 3; col += coloffset, f ^= 2) body(col, f);
        } else {
          coloffset = xfc(P, row, leftstart + 1) == 1 ? 2 : 1;
          int f = 2 - xfc(P, row, leftstart);
          for (int col = leftstart; col < mcol_g - 3; col += coloffset, coloffset ^= 3, f = f ^ (coloffset & 2)) body(col, f);
        }
      }
      __syncthreads();
      // (f) R and B for 2x2 green blocks (:2266-2310), one row per thread in
      // the reference's column order
      int topstart = top + 2;
      for (; topstart < mrow_g - 2; topstart++)
        if ((topstart - P.sgrow) % 3) break;
      int leftstart = left + 2;
      for (; leftstart < mcol_g - 2; leftstart++)
        if ((leftstart - P.sgcol) % 3) break;
      const int coloffsetstart = 2 - (xfc(P, topstart, leftstart + 1) & 1);
      for (int row = topstart + tid; row < mrow_g - 2; row += nth) {
        if (!((row - P.sgrow) % 3)) continue;
        const short* hexmod[2] = {P.allhex1[row % 3][leftstart % 3], P.allhex1[row % 3][(leftstart + coloffsetstart) % 3]};
        for (int col = leftstart, coloffset = coloffsetstart, hexindex = 0; col < mcol_g - 2;
             col += coloffset, coloffset ^= 3, hexindex ^= 1) {
          float* rix = RGB(0, row - top, col - left);
          const short* hex = hexmod[hexindex];
          for (int d = 0; d < NDIR; d += 2, rix += (size_t)ts * ts * 3) {
            const int o0 = hex[d] * 3, o1 = hex[d + 1] * 3;
            if (hex[d] + hex[d + 1]) {
              const float g = 3 * rix[1] - 2 * rix[o0 + 1] - rix[o1 + 1];
              for (int c = 0; c < 4; c += 2) rix[c] = (g + 2 * rix[o0 + c] + rix[o1 + c]) * 0.33333333f;
            } else {
              const float g = 2 * rix[1] - rix[o0 + 1] - rix[o1 + 1];
              for (int c = 0; c < 4; c += 2) rix[c] = (g + rix[o0 + c] + rix[o1 + c]) * 0.5f;
            }
          }
        }
      }
      __syncthreads();
    }
    rgb = S.rgb;
    int mrow = mrow_g - top;
    int mcol = mcol_g - left;

    // (g) YPbPr derivatives (:2346-2405), yuv recomputed at the 3 taps
    {
      const int dn = XTS - 10;
      const int rows = mrow - 10, cols = mcol - 10;
      const XDiv fdrc(rows * cols), fdcl(cols);
      const int n = NDIR * rows * cols;
      // four items per thread and step: their 36 loads are issued before the
      // first store (a store to the derivative planes could otherwise alias
      // the next item's loads for the compiler)
      constexpr int U = 4;
      for (int i0 = tid; i0 < n; i0 += U * nth) {
        float res[U];
        int at[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
          const int i = i0 + u * nth;
          at[u] = -1;
          if (i < n) {
            const int d = fdrc.div(i);
            const int rem = i - d * (rows * cols);
            const int q_ = fdcl.div(rem);
            const int row = 5 + q_, col = 5 + rem - q_ * cols;
            const int dv = d & 3;
            // direction steps 1, ts, ts + 1, ts - 1 of directions 0..3 (and 4..7)
            int f = dv == 0 ? 1 : (dv == 1 ? ts : (dv == 2 ? ts + 1 : ts - 1));
            f = f == 1 ? 1 : f - 8;
            // yuv buffer offset f (width ts-8) -> tile offset
            const int fr = (f == 1) ? 0 : 1, fc = (f == 1) ? 1 : (f - (XTS - 8));
            auto yuv = [&](int r, int c, float& y, float& uu, float& v) {
              const float* p = RGB(d, r, c);
              y = 0.2627f * p[0] + 0.6780f * p[1] + 0.0593f * p[2];
              uu = (p[2] - y) * 0.56433f;
              v = (p[0] - y) * 0.67815f;
            };
            float y0, u0, v0, yp, up, vp, ym, um, vm;
            yuv(row, col, y0, u0, v0);
            yuv(row + fr, col + fc, yp, up, vp);
            yuv(row - fr, col - fc, ym, um, vm);
            res[u] = SQRf(2 * y0 - yp - ym) + SQRf(2 * u0 - up - um) + SQRf(2 * v0 - vp - vm);
            at[u] = (d * dn + (row - 5)) * dn + (col - 5);
          }
        }
#pragma unroll
        for (int u = 0; u < U; u++)
          if (at[u] >= 0) S.drv[at[u]] = res[u];
      }
    }
    __syncthreads();
    // (h) homogeneity maps (:2407-2496)
    {
      const int dn = XTS - 10;
      const int rows = mrow - 12, cols = mcol - 12;
      const XDiv fdh(cols);
      for (int i = tid; i < rows * cols; i += nth) {
        const int q_ = fdh.div(i), row = 6 + q_, col = 6 + i - q_ * cols;
        auto D = [&](int d, int r, int c) { return S.drv[((size_t)d * dn + (r - 5)) * dn + (c - 5)]; };
        float tr = D(0, row, col) < D(1, row, col) ? D(0, row, col) : D(1, row, col);
        for (int d = 2; d < NDIR; d++) tr = (D(d, row, col) < tr ? D(d, row, col) : tr);
        tr *= 8;
        // all eight counts first, then the stores: a byte store may alias
        // any load for the compiler, which would otherwise wait for each
        // direction's loads in turn
        unsigned char temp[NDIR];
#pragma unroll
        for (int d = 0; d < NDIR; d++) {
          temp[d] = 0;
          for (int v = -1; v <= 1; v++)
            for (int h = -1; h <= 1; h++) temp[d] += (D(d, row + v, col + h) <= tr ? 1 : 0);
        }
#pragma unroll
        for (int d = 0; d < NDIR; d++) S.homo[((size_t)d * ts + row) * ts + col] = temp[d];
      }
    }
    __syncthreads();
    if (H - top < ts + 4) mrow = H - top + 2;
    if (W - left < ts + 4) mcol = W - left + 2;
    // (j) 5x5 homogeneity sums and their max (:2504-2612).  Integer sums
    // (at most 25 * 9 = 225, no wrap), so they are formed separably: row
    // 5-sums first, into the derivative planes' memory (dead after (h)).
    const int r0 = min(top, 8), c0 = min(left, 8);
    unsigned char* hs5 = reinterpret_cast<unsigned char*>(S.drv);  // [NDIR][ts][ts]
    {
      const int rows = mrow - 8 - r0 + 4, cols = mcol - 8 - c0;
      const XDiv fdr(rows * cols), fdc(cols);
      for (int i = tid; i < NDIR * rows * cols; i += nth) {
        const int d = fdr.div(i), rem = i - d * (rows * cols);
        const int q_ = fdc.div(rem), row = r0 - 2 + q_, col = c0 + rem - q_ * cols;
        const unsigned char* hp = S.homo + ((size_t)d * ts + row) * ts + col;
        hs5[((size_t)d * ts + row) * ts + col] = (unsigned char)(hp[-2] + hp[-1] + hp[0] + hp[1] + hp[2]);
      }
    }
    __syncthreads();
    {
      const int rows = mrow - 8 - r0, cols = mcol - 8 - c0;
      const XDiv fdj(cols);
      for (int i = tid; i < rows * cols; i += nth) {
        const int q_ = fdj.div(i), row = r0 + q_, col = c0 + i - q_ * cols;
        unsigned char maxval = 0;
        for (int d = 0; d < NDIR; d++) {
          int s = 0;
          for (int v = -2; v <= 2; v++) s += hs5[((size_t)d * ts + row + v) * ts + col];
          const unsigned char hs = (unsigned char)s;
          S.homosum[((size_t)d * ts + row) * ts + col] = hs;
          if (d == 0 || maxval < hs) maxval = hs;
        }
        maxval -= maxval >> 3;
        S.homosummax[(size_t)row * ts + col] = maxval;
      }
    }
    __syncthreads();
    // (l) average the most homogeneous directions (:2614-2650)
    {
      const int rows = mrow - 8 - r0, cols = mcol - 8 - c0;
      const XDiv fdj(cols);
      for (int i = tid; i < rows * cols; i += nth) {
        const int q_ = fdj.div(i), row = r0 + q_, col = c0 + i - q_ * cols;
        unsigned char hm[8];
        for (int d = 0; d < 4; d++) hm[d] = S.homosum[((size_t)d * ts + row) * ts + col];
        for (int d = 4; d < NDIR; d++) {
          hm[d] = S.homosum[((size_t)d * ts + row) * ts + col];
          if (hm[d - 4] < hm[d]) hm[d - 4] = 0;
          else if (hm[d - 4] > hm[d]) hm[d] = 0;
        }
        float avg[4] = {0.f, 0.f, 0.f, 0.f};
        const unsigned char maxval = S.homosummax[(size_t)row * ts + col];
        for (int d = 0; d < NDIR; d++)
          if (hm[d] >= maxval) {
            const float* p = RGB(d, row, col);
            for (int c = 0; c < 3; c++) avg[c] += p[c];
            avg[3] += 1.f;
          }
        float* o = A.rgb_out + ((size_t)(row + top) * W + (col + left)) * 3;
        o[0] = fmaxf(0.f, avg[0] / avg[3]);
        o[1] = fmaxf(0.f, avg[1] / avg[3]);
        o[2] = fmaxf(0.f, avg[2] / avg[3]);
      }
    }
    __syncthreads();
  }
}

// --------------------------------------------------------- 3-pass, one plane on chip
// The interpolation steps (b) to (f) never mix direction planes: each
// direction's reads and writes stay in its own plane, and passes 1 and 2
// continue planes 4..7 from copies of planes 0..3 (:2131-2136).  So one CTA
// carries one plane at a time in shared memory through all of its passes:
// plane k through pass 0, whose derivatives (g) and RGB then go to the CTA's
// global scratch, and on in place as plane k + 4 through passes 1 and 2.  The
// green min/max table stays in shared memory for the whole tile.  The
// homogeneity steps read the eight derivative planes back from the scratch
// and keep their byte maps in shared memory, and the final average reads the
// RGB planes back.  Every step visits each site of its class once and reads
// no value that the same step writes (xt_sites_ok replays the reference's
// scans), so each step runs one site per thread; sites stay in fresh-buffer
// semantics (zeros where a tile computes nothing).
constexpr int XS_THREADS = 1024;
constexpr int kXsMaxCtas = 148;
constexpr int XDN = XTS - 10;  // derivative plane edge
constexpr size_t kPlaneFloats = (size_t)XTS * XTS * 3;
constexpr size_t kPlaneBytes = kPlaneFloats * 4;            // 155,952
// site lists: 4 of every 3x3 sites per class (the replay's bound), 38 x 38
// such blocks in a tile
constexpr int kXsListCap = (XTS / 3) * (XTS / 3) * 4;  // 5,776
constexpr size_t kXsSmemBytes = kPlaneBytes + kGmmBytes + 2 * kXsListCap * 2 + 2 * XTS;  // 231,268
constexpr size_t kXsSpillBytes = ((kRgbBytes + kDrvBytes + 255) / 256) * 256;
static_assert(2 * kHomoBytes <= kPlaneBytes + kGmmBytes, "the homogeneity maps reuse the plane and table memory");
static_assert(kPlaneBytes % 16 == 0 && kHomoBytes % 16 == 0, "float4 fills");

// raw / maximum for every mosaic site, in the reference's IEEE division
// (xraw), once per image: the plane-resident kernel reads each sample in
// several steps and for each of its four plane pairs.
__global__ void k_xt_normalize(XtArgs A, float* norm) {
  const long long n = (long long)A.W * A.H;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    norm[i] = A.cstride == 1 ? A.raw[i] / A.maximum : xraw(A, (int)(i / A.W), (int)(i % A.W));
}

// (g) YPbPr derivatives of one finished direction plane D (:2346-2405),
// yuv recomputed at the three taps, and the plane's RGB, into the CTA's
// scratch.  Reads the plane only.
__device__ __forceinline__ void xs_plane_out(const float* pl, float* srgb, float* sdrv, int D, int nr, int nc) {
  constexpr int ts = XTS;
  const int tid = threadIdx.x, nth = blockDim.x;
  const int rows = nr - 10, cols = nc - 10;
  if (rows > 0 && cols > 0) {
    const int dv = D & 3;
    // direction steps 1, ts, ts + 1, ts - 1 of directions 0..3 (and 4..7)
    int f = dv == 0 ? 1 : (dv == 1 ? ts : (dv == 2 ? ts + 1 : ts - 1));
    f = f == 1 ? 1 : f - 8;
    // yuv buffer offset f (width ts - 8) -> tile offset
    const int fr = (f == 1) ? 0 : 1, fc = (f == 1) ? 1 : (f - (XTS - 8));
    const int step = (fr * ts + fc) * 3;
    float* out = sdrv + (size_t)D * XDN * XDN;
    const XDiv fd(cols);
    for (int i = tid; i < rows * cols; i += nth) {
      const int q = fd.div(i), row = 5 + q, col = 5 + i - q * cols;
      const float* p = pl + (row * ts + col) * 3;
      auto yuv = [](const float* s, float& y, float& u, float& v) {
        y = 0.2627f * s[0] + 0.6780f * s[1] + 0.0593f * s[2];
        u = (s[2] - y) * 0.56433f;
        v = (s[0] - y) * 0.67815f;
      };
      float y0, u0, v0, yp, up, vp, ym, um, vm;
      yuv(p, y0, u0, v0);
      yuv(p + step, yp, up, vp);
      yuv(p - step, ym, um, vm);
      out[(row - 5) * XDN + (col - 5)] = SQRf(2 * y0 - yp - ym) + SQRf(2 * u0 - up - um) + SQRf(2 * v0 - vp - vm);
    }
  }
  const float4* s4 = reinterpret_cast<const float4*>(pl);
  float4* d4 = reinterpret_cast<float4*>(srgb + (size_t)D * kPlaneFloats);
  for (int i = tid; i < (int)(kPlaneBytes / 16); i += nth) d4[i] = s4[i];
}

__global__ void __launch_bounds__(XS_THREADS, 1) k_xtrans_3pass_planes(XtArgs Ain) {
  constexpr int ts = XTS;
  extern __shared__ __align__(16) unsigned char xs_smem[];
  float* pl = reinterpret_cast<float*>(xs_smem);                   // [XTS][XTS][3]
  float2* gmm = reinterpret_cast<float2*>(xs_smem + kPlaneBytes);  // [XTS][XTS/2] (min, max)
  // the tile's non-green sites and 2x2-block greens, as row * XTS + column
  unsigned short* lst_ng = reinterpret_cast<unsigned short*>(xs_smem + kPlaneBytes + kGmmBytes);
  unsigned short* lst_gg = lst_ng + kXsListCap;
  // per tile row / column: pattern phase (bits 0-2, mod 6), off the
  // solitary-green class (bit 3), phase mod 3 (bits 4-5)
  unsigned char* rinfo = reinterpret_cast<unsigned char*>(lst_gg + kXsListCap);
  unsigned char* cinfo = rinfo + XTS;
  __shared__ int s_n[2];
  const int tid = threadIdx.x, nth = blockDim.x;
  __shared__ XtArgs sA;
  {
    constexpr int NW = (int)(sizeof(XtArgs) / 4);
    const int* from = reinterpret_cast<const int*>(&Ain);
    int* to = reinterpret_cast<int*>(&sA);
#pragma unroll
    for (int k = 0; k < NW; k++)
      if (k % XS_THREADS == tid) to[k] = from[k];
  }
  __syncthreads();
  const XtArgs& A = sA;
  const XtParams& P = A.P;
  float* srgb = reinterpret_cast<float*>(A.scratch + (size_t)blockIdx.x * kXsSpillBytes);  // [NDIR][XTS][XTS][3]
  float* sdrv = srgb + NDIR * kPlaneFloats;                                                // [NDIR][XDN][XDN]
  __shared__ int s_tile;
  const int W = A.W, H = A.H;

  for (;;) {
    if (tid == 0) s_tile = atomicAdd(A.tile_counter, 1);
    __syncthreads();
    const int tile = s_tile;
    __syncthreads();
    if (tile >= A.n_top * A.n_left) break;
    const int top = 3 + (tile / A.n_left) * (ts - 16);
    const int left = 3 + (tile % A.n_left) * (ts - 16);
    const int mrow_g = min(top + ts, H - 3);  // global row bound of the computations
    const int mcol_g = min(left + ts, W - 3);
    const int nr = mrow_g - top, nc = mcol_g - left;
    const int warp = tid >> 5, lane = tid & 31, nwarps = nth >> 5;

    // site classes of the tile: line info, then the two site lists (their
    // order is free: every step's sites are independent)
    for (int i = tid; i < XTS; i += nth) {
      const int r6 = (top + i) % 6, c6 = (left + i) % 6;
      rinfo[i] = (unsigned char)(r6 | (((top + i - P.sgrow) % 3 != 0) << 3) | ((r6 % 3) << 4));
      cinfo[i] = (unsigned char)(c6 | (((left + i - P.sgcol) % 3 != 0) << 3) | ((c6 % 3) << 4));
    }
    if (tid == 0) s_n[0] = s_n[1] = 0;
    __syncthreads();
    for (int lr = warp; lr < nr; lr += nwarps) {
      const int ri = rinfo[lr];
      for (int c0 = 0; c0 < nc; c0 += 32) {
        const int lc = c0 + lane;
        const int ci = lc < nc ? cinfo[lc] : 0;
        const bool ng = lc < nc && !(P.xt[ri >> 4][ci >> 4] & 1);
        const bool gg = lc < nc && (ri & 8) && (ci & 8);
        const unsigned mng = __ballot_sync(0xffffffffu, ng), mgg = __ballot_sync(0xffffffffu, gg);
        int bng = 0, bgg = 0;
        if (lane == 0) {
          bng = atomicAdd(&s_n[0], __popc(mng));
          bgg = atomicAdd(&s_n[1], __popc(mgg));
        }
        bng = __shfl_sync(0xffffffffu, bng, 0);
        bgg = __shfl_sync(0xffffffffu, bgg, 0);
        const unsigned lt = (1u << lane) - 1u;
        if (ng) lst_ng[bng + __popc(mng & lt)] = (unsigned short)(lr * XTS + lc);
        if (gg) lst_gg[bgg + __popc(mgg & lt)] = (unsigned short)(lr * XTS + lc);
      }
    }
    __syncthreads();
    const int n_ng = s_n[0], n_gg = s_n[1];

    // (a) green min / max (:1968-2053).  The scan stores a site's hexagon
    // min/max at its half-column slot; on rows with adjacent non-green pairs
    // it stores the first site's values at both sites' slots and computes
    // none for the second.
    for (int j = tid; j < n_ng; j += nth) {
      const int e = lst_ng[j], lr = e / XTS, lc = e - lr * XTS;
      const int r3 = rinfo[lr] >> 4;
      if (lc > 0 && !(P.xt[r3][cinfo[lc - 1] >> 4] & 1)) continue;  // second of a pair
      const int row = top + lr, col = left + lc;
      const short* hex = P.allhex0[r3][cinfo[lc] >> 4];
      float minval = FLT_MAX, maxval = 0.f;
      for (int c = 0; c < 6; c++) {
        const float val = xn_hex(A, row, col, hex[c]);
        minval = minval < val ? minval : val;
        maxval = maxval > val ? maxval : val;
      }
      const float2 v = make_float2(minval, maxval);
      float2* g = gmm + (size_t)lr * (ts / 2);
      g[lc >> 1] = v;
      if (lc + 1 < nc && !(P.xt[r3][cinfo[lc + 1] >> 4] & 1)) g[(lc + 1) >> 1] = v;
    }

    for (int k = 0; k < 4; k++) {
      // fresh plane k: zeros, the native samples (:2055-2061; planes 1..3 are
      // copies of plane 0 without its last float, :2067-2069) and (b) the
      // green of direction k at every non-green site (:2071-2127)
      {
        float4* z = reinterpret_cast<float4*>(pl);
        for (int i = tid; i < (int)(kPlaneBytes / 16); i += nth) z[i] = make_float4(0.f, 0.f, 0.f, 0.f);
      }
      __syncthreads();
      for (int lr = warp; lr < nr; lr += nwarps) {
        const int r6 = rinfo[lr] & 7;
        const float* src = A.norm + (size_t)(top + lr) * W + left;
        float* prow = pl + lr * ts * 3;
        for (int lc = lane; lc < nc; lc += 32) {
          const int fcv = P.xt[r6][cinfo[lc] & 7];
          if (k == 0 || lr * ts + lc != ts * ts - 1 || fcv != 2) prow[lc * 3 + fcv] = src[lc];
        }
      }
      for (int j = tid; j < n_ng; j += nth) {
        const int e = lst_ng[j], lr = e / XTS, lc = e - lr * XTS;
        const int row = top + lr, col = left + lc;
        const int r3 = rinfo[lr] >> 4;
        const short* hex = P.allhex0[r3][cinfo[lc] >> 4];
        const int cdir = k ^ (P.right_shift[r3] == 1 ? 0 : 1);
        float color;
        if (cdir == 0) {
          color = 0.6796875f * (xn_hex(A, row, col, hex[1]) + xn_hex(A, row, col, hex[0])) -
                  0.1796875f * (xn_hex(A, row, col, 2 * hex[1]) + xn_hex(A, row, col, 2 * hex[0]));
        } else if (cdir == 1) {
          color = 0.87109375f * xn_hex(A, row, col, hex[3]) + xn_hex(A, row, col, hex[2]) * 0.12890625f +
                  0.359375f * (xn_hex(A, row, col, 0) - xn_hex(A, row, col, -hex[2]));
        } else {
          const int h4 = hex[cdir + 2];
          color = 0.640625f * xn_hex(A, row, col, h4) + 0.359375f * xn_hex(A, row, col, -2 * h4) +
                  0.12890625f * (2.f * xn_hex(A, row, col, 0) - xn_hex(A, row, col, 3 * h4) -
                                 xn_hex(A, row, col, -3 * h4));
        }
        const float2 mmv = gmm[(size_t)lr * (ts / 2) + (lc >> 1)];
        pl[e * 3 + 1] = LIMf(color, mmv.x, mmv.y);
      }
      __syncthreads();

      for (int pass = 0; pass < 3; pass++) {
        if (pass == 1) {
          // plane k is final: (g) its derivatives and its RGB go to the
          // scratch, and the plane continues in place as plane k + 4
          xs_plane_out(pl, srgb, sdrv, k, nr, nc);
          __syncthreads();
        }
        // (c) recalculate green from closer pixels (:2138-2183): direction
        // d = 3..5 updates plane (d - 2) ^ flip, reading green sites only
        if (pass) {
          for (int j = tid; j < n_ng; j += nth) {
            const int e = lst_ng[j], lr = e / XTS, lc = e - lr * XTS;
            if (lr < 2 || lr >= nr - 2 || lc < 2 || lc >= nc - 2) continue;
            const int ri = rinfo[lr], ci = cinfo[lc];
            const int dd = k ^ (P.right_shift[ri >> 4] == 1 ? 0 : 1);
            if (dd == 0) continue;
            const int f = P.xt[ri & 7][ci & 7];
            const int hx = P.allhex1[ri >> 4][ci >> 4][dd + 2];
            float* rix = pl + e * 3;
            const int o1 = hx * 3, o2 = -2 * hx * 3;
            const float val = 0.33333333f * (rix[o2 + 1] + 2 * (rix[o1 + 1] - rix[o1 + f]) - rix[o2 + f]) + rix[f];
            const float2 mmv = gmm[(size_t)lr * (ts / 2) + (lc >> 1)];
            rix[1] = LIMf(val, mmv.x, mmv.y);
          }
          __syncthreads();
        }
        // (d) R/B at solitary green pixels (:2185-2222): plane k carries
        // direction k (k < 2), directions 2 and 3 (k = 2) or 4 and 5 (k = 3),
        // the second of a pair falling back to the first where its
        // difference is larger
        {
          const int sgstartcol = (left - P.sgcol + 4) / 3 * 3 + P.sgcol;
          const int row0 = (top - P.sgrow + 4) / 3 * 3 + P.sgrow;
          const int nrow = row0 < mrow_g - 2 ? (mrow_g - 2 - row0 + 2) / 3 : 0;
          const int ncol = sgstartcol < mcol_g - 2 ? (mcol_g - 2 - sgstartcol + 2) / 3 : 0;
          const int d_lo = k < 2 ? k : 2 * k - 2, nd = k < 2 ? 1 : 2;
          for (int item = tid; item < nrow * ncol; item += nth) {
            const int row = row0 + 3 * (item / ncol), kk = item % ncol;
            const int col = sgstartcol + 3 * kk;
            float* rix = pl + ((row - top) * ts + (col - left)) * 3;
            const int h0 = xfc(P, row, sgstartcol + 1) ^ ((kk & 1) << 1);
            float cr0 = 0.f, cb0 = 0.f, df0 = 0.f, r = 0.f, b = 0.f, df1 = 0.f;
#pragma unroll
            for (int j = 0; j < 2; j++) {
              if (j >= nd) break;
              const int d = d_lo + j;
              const int i = (d & 1) ? ts : 1;
              int h = h0 ^ ((d & 1) << 1);
              float df = 0.f, cr = 0.f, cb = 0.f;
#pragma unroll
              for (int c = 0; c < 2; c++, h ^= 2) {
                const int op = i * (1 << c) * 3, om = -i * (1 << c) * 3;
                const float g = rix[1] + rix[1] - rix[op + 1] - rix[om + 1];
                const float v = g + rix[op + h] + rix[om + h];
                if (h == 0) cr = v;
                else cb = v;
                if (d > 1) df += SQRf(rix[op + 1] - rix[om + 1] - rix[op + h] + rix[om + h]) + SQRf(g);
              }
              if (j == 0) {
                cr0 = cr;
                cb0 = cb;
                df0 = df;
              }
              r = cr;
              b = cb;
              df1 = df;
            }
            if (nd == 2 && df0 < df1) {
              r = cr0;
              b = cb0;
            }
            rix[0] = 0.5f * r;
            rix[2] = 0.5f * b;
          }
        }
        __syncthreads();
        // (e) red for blue pixels and vice versa (:2224-2264): every non-green
        // site writes its other colour f = 2 - own
        {
          for (int j = tid; j < n_ng; j += nth) {
            const int e = lst_ng[j], lr = e / XTS, lc = e - lr * XTS;
            if (lr < 3 || lr >= nr - 3 || lc < 3 || lc >= nc - 3) continue;
            const int ri = rinfo[lr];
            const int c = (ri & 8) ? ts : 1;  // (row - sgrow) % 3 != 0
            const int h = 3 * (c ^ ts ^ 1);
            const int f = 2 - P.xt[ri & 7][cinfo[lc] & 7];
            float* rix = pl + e * 3;
            const float g0 = rix[1];
            const bool use_c = k > 1 || ((k ^ c) & 1) ||
                               ((fabsf(g0 - rix[c * 3 + 1]) + fabsf(g0 - rix[-c * 3 + 1])) <
                                2.f * (fabsf(g0 - rix[h * 3 + 1]) + fabsf(g0 - rix[-h * 3 + 1])));
            const int s = use_c ? c : h;
            rix[f] = g0 + 0.5f * (rix[s * 3 + f] + rix[-s * 3 + f] - rix[s * 3 + 1] - rix[-s * 3 + 1]);
          }
        }
        __syncthreads();
        // (f) R and B for 2x2 green blocks (:2266-2310): greens off the
        // solitary-green row and column classes, hexagon allhex1
        {
          for (int j = tid; j < n_gg; j += nth) {
            const int e = lst_gg[j], lr = e / XTS, lc = e - lr * XTS;
            if (lr < 2 || lr >= nr - 2 || lc < 2 || lc >= nc - 2) continue;
            float* rix = pl + e * 3;
            const short* hex = P.allhex1[rinfo[lr] >> 4][cinfo[lc] >> 4];
            const int o0 = hex[2 * k] * 3, o1 = hex[2 * k + 1] * 3;
            const float v1 = rix[1], a1 = rix[o0 + 1], b1 = rix[o1 + 1];
            const float a0 = rix[o0], b0 = rix[o1], a2 = rix[o0 + 2], b2 = rix[o1 + 2];
            if (hex[2 * k] + hex[2 * k + 1]) {
              const float g = 3 * v1 - 2 * a1 - b1;
              rix[0] = (g + 2 * a0 + b0) * 0.33333333f;
              rix[2] = (g + 2 * a2 + b2) * 0.33333333f;
            } else {
              const float g = 2 * v1 - a1 - b1;
              rix[0] = (g + a0 + b0) * 0.5f;
              rix[2] = (g + a2 + b2) * 0.5f;
            }
          }
        }
        __syncthreads();
      }
      xs_plane_out(pl, srgb, sdrv, k + 4, nr, nc);
      __syncthreads();
    }

    // (h) homogeneity maps (:2407-2496) from the derivative planes
    unsigned char* homo = xs_smem;             // [NDIR][XTS][XTS]
    unsigned char* hs5 = xs_smem + kHomoBytes;  // [NDIR][XTS][XTS]
    {
      float4* z = reinterpret_cast<float4*>(homo);
      for (int i = tid; i < (int)(kHomoBytes / 16); i += nth) z[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    __syncthreads();
    {
      const int rows = nr - 12, cols = nc - 12;
      if (rows > 0 && cols > 0) {
        const XDiv fd(cols);
        for (int i = tid; i < rows * cols; i += nth) {
          const int q = fd.div(i), row = 6 + q, col = 6 + i - q * cols;
          const float* dp = sdrv + (row - 5) * XDN + (col - 5);
          float tr = dp[0] < dp[XDN * XDN] ? dp[0] : dp[XDN * XDN];
          for (int d = 2; d < NDIR; d++) tr = (dp[d * XDN * XDN] < tr ? dp[d * XDN * XDN] : tr);
          tr *= 8;
          unsigned char temp[NDIR];
#pragma unroll
          for (int d = 0; d < NDIR; d++) {
            temp[d] = 0;
            for (int v = -1; v <= 1; v++)
              for (int h = -1; h <= 1; h++) temp[d] += (dp[d * XDN * XDN + v * XDN + h] <= tr ? 1 : 0);
          }
#pragma unroll
          for (int d = 0; d < NDIR; d++) homo[(d * ts + row) * ts + col] = temp[d];
        }
      }
    }
    __syncthreads();
    int mrow = nr, mcol = nc;
    if (H - top < ts + 4) mrow = H - top + 2;
    if (W - left < ts + 4) mcol = W - left + 2;
    // (j) 5x5 homogeneity sums (:2504-2612), separably: row 5-sums first
    const int r0 = min(top, 8), c0 = min(left, 8);
    {
      const int rows = mrow - 8 - r0 + 4, cols = mcol - 8 - c0;
      if (rows > 0 && cols > 0) {
        const XDiv fdr(rows * cols), fdc(cols);
        for (int i = tid; i < NDIR * rows * cols; i += nth) {
          const int d = fdr.div(i), rem = i - d * (rows * cols);
          const int q = fdc.div(rem), row = r0 - 2 + q, col = c0 + rem - q * cols;
          const unsigned char* hp = homo + (d * ts + row) * ts + col;
          hs5[(d * ts + row) * ts + col] = (unsigned char)(hp[-2] + hp[-1] + hp[0] + hp[1] + hp[2]);
        }
      }
    }
    __syncthreads();
    // (j) column sums and their max, then (l) the average of the most
    // homogeneous directions (:2614-2650), one output pixel per thread
    {
      const int rows = mrow - 8 - r0, cols = mcol - 8 - c0;
      if (rows > 0 && cols > 0) {
        const XDiv fd(cols);
        for (int i = tid; i < rows * cols; i += nth) {
          const int q = fd.div(i), row = r0 + q, col = c0 + i - q * cols;
          unsigned char hm[NDIR];
          unsigned char maxval = 0;
#pragma unroll
          for (int d = 0; d < NDIR; d++) {
            int s = 0;
            for (int v = -2; v <= 2; v++) s += hs5[(d * ts + row + v) * ts + col];
            hm[d] = (unsigned char)s;
            if (d == 0 || maxval < hm[d]) maxval = hm[d];
          }
          maxval -= maxval >> 3;
#pragma unroll
          for (int d = 4; d < NDIR; d++) {
            if (hm[d - 4] < hm[d]) hm[d - 4] = 0;
            else if (hm[d - 4] > hm[d]) hm[d] = 0;
          }
          float avg[4] = {0.f, 0.f, 0.f, 0.f};
          const float* px = srgb + (size_t)(row * ts + col) * 3;
#pragma unroll
          for (int d = 0; d < NDIR; d++)
            if (hm[d] >= maxval) {
              const float* p = px + d * kPlaneFloats;
              for (int c = 0; c < 3; c++) avg[c] += p[c];
              avg[3] += 1.f;
            }
          float* o = A.rgb_out + ((size_t)(row + top) * W + (col + left)) * 3;
          o[0] = fmaxf(0.f, avg[0] / avg[3]);
          o[1] = fmaxf(0.f, avg[1] / avg[3]);
          o[2] = fmaxf(0.f, avg[2] / avg[3]);
        }
      }
    }
    __syncthreads();
  }
}

// allhex / solitary green / RightShift tables (:1887-1940), host side.
XtParams make_xt_params(const char* xtrans, int width) {
  XtParams P;
  memcpy(P.xt, xtrans, 36);
  const short orth[12] = {1, 0, 0, 1, -1, 0, 0, -1, 1, 0, 0, 1};
  const short patt[2][16] = {{0, 1, 0, -1, 2, 0, -1, 0, 1, 1, 1, -1, 0, 0, 0, 0},
                             {0, 1, 0, -2, 1, 0, -2, 0, 1, 1, -2, -2, 1, -1, -1, 1}};
  auto isg = [&](int row, int col) { return P.xt[row % 3][col % 3] & 1; };
  memset(P.allhex0, 0, sizeof(P.allhex0));
  memset(P.allhex1, 0, sizeof(P.allhex1));
  unsigned short sgrow = 0, sgcol = 0;
  for (int row = 0; row < 3; row++)
    for (int col = 0; col < 3; col++) {
      const int gint = isg(row, col);
      for (int ng = 0, d = 0; d < 10; d += 2) {
        if (isg(row + orth[d] + 6, col + orth[d + 2] + 6)) ng = 0;
        else ng++;
        if (ng == 4) {
          sgrow = row;
          sgcol = col;
        }
        if (ng == gint + 1)
          for (int c = 0; c < 8; c++) {
            const int v = orth[d] * patt[gint][c * 2] + orth[d + 1] * patt[gint][c * 2 + 1];
            const int h = orth[d + 2] * patt[gint][c * 2] + orth[d + 3] * patt[gint][c * 2 + 1];
            P.allhex0[row][col][c ^ (gint * 2 & d)] = (short)(h + v * width);
            P.allhex1[row][col][c ^ (gint * 2 & d)] = (short)(h + v * XTS);
          }
      }
    }
  P.sgrow = sgrow;
  P.sgcol = sgcol;
  for (int row = 0; row < 3; row++) {
    int greencount = 0;
    for (int col = 0; col < 3; col++) greencount += isg(row, col);
    P.right_shift[row] = (greencount == 2);
  }
  return P;
}

// Whether the reference's row scans of phases (a), (b), (c), (e) and (f)
// reduce to "every site of the class" for this pattern (true for the X-Trans
// layouts and their shifts), so the site-parallel kernels apply.  Checked by
// replaying the scans over every tile-origin residue.
bool xt_sites_ok(const XtParams& P) {
  auto isg = [&](int r, int c) { return P.xt[((r % 3) + 3) % 3][((c % 3) + 3) % 3] & 1; };
  auto fc = [&](int r, int c) { return (int)P.xt[(r + 6) % 6][(c + 6) % 6]; };
  // the plane kernel's site lists hold at most 4 non-green sites per 3x3
  int greens = 0;
  for (int r = 0; r < 3; r++)
    for (int c = 0; c < 3; c++) greens += isg(r, c);
  if (9 - greens > 4) return false;
  for (int t0 = 0; t0 < 6; t0++)
    for (int l0 = 0; l0 < 6; l0++) {
      const int top = 6 + t0, left = 6 + l0, mrow = top + 30, mcol = left + 30;
      for (int row = top; row < mrow; row++) {
        // (b): visits from the first non-green site
        int ls = left;
        while (ls < mcol && isg(row, ls)) ls++;
        int co = P.right_shift[row % 3] == 1 ? 3 : 1 + (fc(row, ls + 1) & 1);
        int expect = ls;
        for (int col = ls; col < mcol; col += co, co = (co == 3) ? 3 : (co ^ 3)) {
          while (expect < mcol && isg(row, expect)) expect++;
          if (col != expect) return false;
          expect++;
        }
        while (expect < mcol && isg(row, expect)) expect++;
        if (expect < mcol) return false;
        // (e): the written colour is 2 - own colour at every visit
        ls = left;
        while (ls < mcol - 1 && isg(row, ls)) ls++;
        int f = 2 - fc(row, ls);
        if (P.right_shift[row % 3] == 1) {
          for (int col = ls; col < mcol; col += 3, f ^= 2)
            if (isg(row, col) || f != 2 - fc(row, col)) return false;
        } else {
          co = fc(row, ls + 1) == 1 ? 2 : 1;
          for (int col = ls; col < mcol; col += co, co ^= 3, f ^= (co & 2))
            if (isg(row, col) || f != 2 - fc(row, col)) return false;
        }
      }
      // (a): the slot a non-green site reads holds the min/max of the site
      // itself, or of its left neighbour when that is a non-green site of
      // the tile (the second site of a pair); replayed in the scan's write
      // order
      for (int row = top; row < mrow; row++) {
        int src[40];
        for (int j = 0; j < 40; j++) src[j] = -1;
        int ls = left;
        while (ls < mcol && isg(row, ls)) ls++;
        const int co = P.right_shift[row % 3] == 1 ? 3 : 1 + (fc(row, ls + 1) & 1);
        if (co == 3) {
          for (int col = ls; col < mcol; col += 3) src[(col - left) >> 1] = col;
        } else {
          int col = ls;
          if (co == 2) {
            src[(col - left) >> 1] = col;
            col += 2;
          }
          for (; col < mcol - 1; col += 3) src[(col - left) >> 1] = src[(col + 1 - left) >> 1] = col;
          if (col < mcol) src[(col - left) >> 1] = col;
        }
        for (int col = left; col < mcol; col++) {
          if (isg(row, col)) continue;
          const int expect_src = (col > left && !isg(row, col - 1)) ? col - 1 : col;
          if (src[(col - left) >> 1] != expect_src) return false;
        }
      }
      // (c): visits every non-green site from left + 2 with f = own colour
      // and hexagon allhex1[row % 3][col % 3], and reads green sites only
      // (which the step does not write)
      for (int row = top + 2; row < mrow - 2; row++) {
        int ls = left + 2;
        while (ls < mcol - 2 && isg(row, ls)) ls++;
        int co = P.right_shift[row % 3] == 1 ? 3 : 1 + (fc(row, ls + 1) & 1);
        int f = fc(row, ls);
        int expect = ls;
        for (int col = ls; col < mcol - 2;) {
          while (expect < mcol - 2 && isg(row, expect)) expect++;
          if (col != expect || f != fc(row, col)) return false;
          expect++;
          for (int d = 3; d < 6; d++)
            for (int m = -2; m <= 1; m += 3) {
              const int x = m * P.allhex1[row % 3][col % 3][d];
              int v = -7, h = 0;
              for (int vv = -6; vv <= 6; vv++)
                if (x - vv * XTS >= -6 && x - vv * XTS <= 6) v = vv, h = x - vv * XTS;
              if (v < -6 || !isg(row + v, col + h)) return false;
            }
          if (co == 3) {
            col += 3;
            f ^= 2;
          } else {
            col += co;
            co ^= 3;
            f ^= (co & 2);
          }
        }
        while (expect < mcol - 2 && isg(row, expect)) expect++;
        if (expect < mcol - 2) return false;
      }
      // (f): visited columns are those off the solitary-green column class
      int ts_ = top;
      while (ts_ < mrow && !((ts_ - P.sgrow + 6) % 3)) ts_++;
      int lsf = left;
      while (lsf < mcol && !((lsf - P.sgcol + 6) % 3)) lsf++;
      const int cos = 2 - (fc(ts_, lsf + 1) & 1);
      for (int col = lsf, co = cos; col < mcol; col += co, co ^= 3)
        if (!((col - P.sgcol + 6) % 3)) return false;
      int visits = 0, expect_n = 0;
      for (int col = lsf, co = cos; col < mcol; col += co, co ^= 3) visits++;
      for (int col = lsf; col < mcol; col++) expect_n += ((col - P.sgcol + 6) % 3) != 0;
      if (visits != expect_n) return false;
    }
  return true;
}

// The plane-resident kernel runs where the replay accepts the pattern,
// unless LRE_XTRANS_ROWSCAN=1 asks for the row-scan kernel (a test hook:
// it keeps the fallback path covered on the X-Trans layouts).
bool xt_use_planes(const XtParams& P) {
  const char* force = std::getenv("LRE_XTRANS_ROWSCAN");
  if (force && force[0] == '1') return false;
  return xt_sites_ok(P);
}

}  // namespace

size_t ws_bytes_xtrans(size_t w, size_t h, int passes, const char* xtrans) {
  if (passes == 1) return 0;
  const size_t planes = (size_t)kXsMaxCtas * kXsSpillBytes + ((w * h * sizeof(float) + 255) / 256) * 256;
  const size_t rowscan = (size_t)kXtMaxCtas * kXtSlabBytes;
  if (xtrans) return (xt_use_planes(make_xt_params(xtrans, (int)w)) ? planes : rowscan) + 4096;
  return std::max(rowscan, planes) + 4096;
}

lre_status launch_xtrans(Context* c, const float* raw, int cstride, float* rgb, size_t w, size_t h, const char* xtrans,
                         float maximum_value, int passes) {
  XtArgs A;
  A.raw = raw;
  A.norm = nullptr;
  A.cstride = cstride;
  A.rgb_out = rgb;
  A.W = (int)w;
  A.H = (int)h;
  A.maximum = maximum_value;
  // hexagon offsets are 16-bit (h + v * width, |v| <= 2), as in the reference
  if (2 * w + 2 > 32767 && passes != 1)
    return fail(c, LRE_ERR_INVALID_ARGUMENT, "demosaic_xtrans_3pass: width above 16382 overflows the hexagon offsets");
  A.P = make_xt_params(xtrans, (int)w);
  if (passes == 1) {
    // border (1 px) first, then the interior (:2681-2760)
    k_xtrans_border<<<grid_for(4 * (w + h), 256, c->sm_count * 2), 256, 0, c->stream>>>(A, 1);
    if (w > 2 && h > 2)
      k_xtrans_1pass<<<grid_for((w - 2) * (h - 2), 256, c->sm_count * 8), 256, 0, c->stream>>>(A);
    count_launch(c, 2);
    return check_launch(c, "demosaic_xtrans_1pass");
  }
  // tile grid of :1968-1969
  int n_top = 0, n_left = 0;
  for (int top = 3; top < (int)h - 19; top += XTS - 16) n_top++;
  for (int left = 3; left < (int)w - 19; left += XTS - 16) n_left++;
  A.n_top = n_top;
  A.n_left = n_left;
  const int tiles = n_top * n_left;
  if (tiles > 0) {
    // Patterns whose scans the replay confirms run the plane-resident kernel:
    // one 1024-thread CTA per SM.  Others run the row-scan kernel, two
    // 512-thread CTAs per SM, each with its whole tile in a global slab.
    const bool sites = xt_use_planes(A.P);
    if (sites) {
      float* norm = reinterpret_cast<float*>(c->ws.take(w * h * sizeof(float)));
      if (!norm) return fail(c, LRE_ERR_OUT_OF_MEMORY, "demosaic_xtrans_3pass: workspace too small");
      k_xt_normalize<<<grid_for(w * h, 256, c->sm_count * 8), 256, 0, c->stream>>>(A, norm);
      count_launch(c);
      A.norm = norm;
    }
    const int nblk = sites ? std::min(std::min(tiles, c->sm_count), kXsMaxCtas)
                           : std::min(std::min(tiles, c->sm_count * kXtCtasPerSm), kXtMaxCtas);
    A.scratch = reinterpret_cast<unsigned char*>(c->ws.take((size_t)nblk * (sites ? kXsSpillBytes : kXtSlabBytes)));
    A.tile_counter = reinterpret_cast<int*>(c->ws.take(256));
    if (!A.scratch || !A.tile_counter) return fail(c, LRE_ERR_OUT_OF_MEMORY, "demosaic_xtrans_3pass: workspace too small");
    LRE_CUDA_TRY(c, cudaMemsetAsync(A.tile_counter, 0, sizeof(int), c->stream));
    if (sites) {
      LRE_CUDA_TRY(c, cudaFuncSetAttribute(k_xtrans_3pass_planes, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)kXsSmemBytes));
      k_xtrans_3pass_planes<<<nblk, XS_THREADS, kXsSmemBytes, c->stream>>>(A);
    } else {
      k_xtrans_3pass<<<nblk, XT_THREADS, 0, c->stream>>>(A);
    }
    count_launch(c);
  }
  k_xtrans_border<<<grid_for(16 * (w + h), 256, c->sm_count * 2), 256, 0, c->stream>>>(A, 8);
  count_launch(c);
  return check_launch(c, "demosaic_xtrans_3pass");
}

}  // namespace lre
