// k_aahd.cu -- AAHD Bayer demosaic (CPUAccelerator::demosaic_bayer_aahd,
// core/cpu_accelerator.cpp:617-633, running AAHD_Processor, :177-601).
//
// Layout.  The reference works on two padded float[3] images (horizontal and
// vertical interpolations, a 4-px zero margin), two int[3] YUV images, and a
// byte direction map.  Here each channel of each direction is its own padded
// plane in HBM ((W+8) x (H+8) floats): X (the native samples), R/G/B for
// d = 0 (horizontal) and d = 1 (vertical), and the direction map held as
// floats for the in-order refinement sweep.  The YUV images are never stored:
// evaluate_ahd recomputes them from the gamma table where it needs them.
//
// Ordering.  make_ahd_greens, make_ahd_rb and evaluate_ahd read only values
// their own loop does not write, so they run one thread per pixel.  Two
// passes rewrite in place and read rewritten neighbours:
//   * hide_hots: a hot/dead site is replaced from same-colour sites two
//     apart, and later sites test against the replaced values (k_gs_sweep,
//     rows paired, skew 3, after a parallel pre-test: if no site is hot against the
//     original values, no site is hot in order either, and the sweep exits);
//   * refine_hv_dirs: each row updates its even columns, then its odd ones,
//     reading the row above as already refined (k_gs_sweep, skew 1).
// Both are OpenMP row loops in the reference, whose result with several
// threads depends on timing at chunk boundaries (and whose channel min/max
// scan is an unsynchronised OpenMP reduction); the sequential order is the
// defined result and the one computed here.
//
// Arithmetic follows the reference's float/int conversions (truncations
// included) operation for operation, with --fmad=false.  The gamma table is
// built on the host with the reference's expression and uploaded once per
// device.  Samples must lie in [0, 65536): the reference indexes its 64 Ki
// gamma table with the sample (out-of-range indices are undefined there;
// here they clamp to the table).
#include <cmath>
#include <mutex>

#include "common.cuh"
#include "lre_internal.h"
#include "stencil.cuh"
#include "sweep.cuh"

namespace lre {

namespace {

constexpr int kMargin = 4;  // nr_margin
constexpr int kHor = 2, kVer = 4;

__device__ float g_aahd_gamma[0x10000];

// yuv_coeff (Rec. 2020) times the identity rgb_cam: the reference's
// yuv_cam (:228-240) equals yuv_coeff exactly.
__constant__ float c_yuv[3][3] = {{+0.2627f, +0.6780f, +0.0593f},
                                  {-0.13963f, -0.36037f, +0.5f},
                                  {+0.5034f, -0.4629f, -0.0405f}};

struct Aahd {
  int W, H, NW;  // image size, padded width
  uint32_t filters;
  float maxv;
  float* X;        // native samples (after hide_hots: with hot sites replaced)
  float* P[2][3];  // [d][channel]
  float* ND;       // direction map
  float* stats;    // channel max [3], channel min [3]
  int* hot;        // count of sites hot against the original samples
  __device__ __forceinline__ unsigned fc(int i, int j) const { return fcol3((unsigned)i, (unsigned)j, filters); }
  __device__ __forceinline__ size_t pi(int i, int j) const { return (size_t)(i + kMargin) * NW + (j + kMargin); }
  // Plane of direction d, channel c, selected without indexing the
  // parameter array at run time (which would copy it to local memory).
  __device__ __forceinline__ float* pl(int d, int c) const {
    float* const* row = d ? P[1] : P[0];
    return c == 0 ? row[0] : (c == 1 ? row[1] : row[2]);
  }
};

// One pixel per (i, j), independent of order.  Along x a block covers 64
// columns and each thread takes two of them of the same parity in two
// half-passes, so a warp's lanes see one Bayer colour at a time (launch with
// (W + 63) / 64 blocks in x).
#define AAHD_FOR_PIXELS(A)                                                                    \
  for (int i = blockIdx.y * blockDim.y + threadIdx.y; i < (A).H; i += gridDim.y * blockDim.y) \
    for (int aahd_half = 0; aahd_half < 2; aahd_half++)                                        \
      for (int j = 2 * (blockIdx.x * blockDim.x + threadIdx.x) + aahd_half; j < (A).W;         \
           j += 2 * gridDim.x * blockDim.x)

__device__ __forceinline__ void atomic_max_f(float* a, float v) {
  int old = __float_as_int(*a);
  while (__int_as_float(old) < v) {
    const int seen = atomicCAS(reinterpret_cast<int*>(a), old, __float_as_int(v));
    if (seen == old) break;
    old = seen;
  }
}
__device__ __forceinline__ void atomic_min_f(float* a, float v) {
  int old = __float_as_int(*a);
  while (__int_as_float(old) > v) {
    const int seen = atomicCAS(reinterpret_cast<int*>(a), old, __float_as_int(v));
    if (seen == old) break;
    old = seen;
  }
}

// channel_minimum starts from pixel 0's three channels (:223-226): the
// sparse (H,W,3) input's first three floats, or for a dense mosaic its first
// sample in its own channel and zero in the others.
__global__ void k_aahd_stats_init(const float* __restrict__ raw, int cs, Aahd A) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const unsigned f0 = A.fc(0, 0);
  for (int c = 0; c < 3; c++) {
    A.stats[c] = 0.0f;
    A.stats[3 + c] = cs == 1 ? ((unsigned)c == f0 ? raw[0] : 0.0f) : raw[c];
  }
  *A.hot = 0;
}

// Constructor copy (:276-306): non-zero samples go to both direction images
// and to the per-colour max/min (min starts from pixel 0's three channels).
__global__ void k_aahd_init(const float* __restrict__ raw, int cs, Aahd A) {
  AAHD_FOR_PIXELS(A) {
    const unsigned c = A.fc(i, j);
    const size_t k = (size_t)i * A.W + j;
    const float d = cs == 1 ? raw[k] : raw[k * 3 + c];
    if (d != 0) {
      const size_t p = A.pi(i, j);
      A.X[p] = d;
      A.pl(0, c)[p] = d;
      A.pl(1, c)[p] = d;
      atomic_max_f(&A.stats[c], d);
      atomic_min_f(&A.stats[3 + c], d);
    }
  }
}

// hide_hots' test and replacement (:354-402) for the non-green site at
// padded index p, reading X through `x(dr, dc)`.  Returns true and sets
// *out when the site is hot or dead.
template <class F>
__device__ __forceinline__ bool hot_site(F x, float* out) {
  const float v = x(0, 0);
  const int c = (int)v;
  const float fcv = (float)c;
  const float e2 = x(0, 2), w2 = x(0, -2), n2 = x(-2, 0), s2 = x(2, 0);
  const float ge = x(0, 1), gw = x(0, -1), gn = x(-1, 0), gs = x(1, 0);
  const bool above = fcv > e2 && fcv > w2 && fcv > n2 && fcv > s2 && fcv > ge && fcv > gw && fcv > gn && fcv > gs;
  const bool below = fcv < e2 && fcv < w2 && fcv < n2 && fcv < s2 && fcv < ge && fcv < gw && fcv < gn && fcv < gs;
  if (!above && !below) return false;
  const int chot = c >> 4, cdead = c << 4;
  int avg = 0;
  for (int k = -2; k < 3; k += 2)
    for (int m = -2; m < 3; m += 2) {
      if (m == 0 && k == 0) continue;
      avg = (int)((float)avg + x(k, m));
    }
  avg /= 8;
  if (!(chot > avg || cdead < avg)) return false;
  const int dh = (int)(fabsf(w2 - e2) + fabsf(gw - ge) + fabsf(gw - ge + e2 - w2));
  const int dv = (int)(fabsf(n2 - s2) + fabsf(gn - gs) + fabsf(gn - gs + s2 - n2));
  *out = (dv > dh) ? (w2 + e2) / 2 : (n2 + s2) / 2;
  return true;
}

__global__ void k_aahd_hot_pretest(Aahd A) {
  int found = 0;
  AAHD_FOR_PIXELS(A) {
    if (A.fc(i, j) == 1) continue;
    const size_t p = A.pi(i, j);
    float o;
    if (hot_site([&](int dr, int dc) { return A.X[p + (ptrdiff_t)dr * A.NW + dc]; }, &o)) found = 1;
  }
  if (__syncthreads_or(found) && threadIdx.x == 0 && threadIdx.y == 0) atomicAdd(A.hot, 1);
}

// hide_hots in row-major order over the padded X plane.  A site reads the
// same-colour sites of rows r - 2 .. r + 2 up to two columns away (the
// 8-neighbour average includes the diagonals (r - 2, c + 2) and
// (r + 2, c - 2)) and greens of rows r +- 1, which never change.  So rows r
// and r + 1 advance together, each row pair three columns behind the pair
// above: (r - 2, c + 2) is then already rewritten and (r + 2, c - 2) not yet.
struct OpHideHots {
  static constexpr int NS = 1, NP = 1, HALO = 2, SKEW = 3, PAIR = 2, NCH = 1, LAG = 0, RING = kRing;
  template <class T>
  __device__ static void cell(const T& t, int r, int c, const Geo& g) {
    // padded coordinates; the 2x2 pattern makes the 4-px offset invisible
    if (g.fc(r, c) == 1) return;
    float o;
    if (hot_site([&](int dr, int dc) { return t(0, r + dr, c + dc); }, &o)) t(0, r, c) = o;
  }
};

// make_ahd_gline (:413-442) for both directions at non-green sites, plus the
// (possibly replaced) native samples copied into both direction images.
__global__ void k_aahd_greens(Aahd A) {
  AAHD_FOR_PIXELS(A) {
    const unsigned kc = A.fc(i, j);
    const size_t p = A.pi(i, j);
    const float k0 = A.X[p];
    if (kc == 1) continue;
    A.pl(0, kc)[p] = k0;
    A.pl(1, kc)[p] = k0;
    const float gmax = A.stats[1], gmin = A.stats[4];
#pragma unroll
    for (int d = 0; d < 2; d++) {
      const ptrdiff_t dir = d ? (ptrdiff_t)A.NW : 1;
      const float gm = A.X[p - dir], gp = A.X[p + dir];
      const int h1 = (int)(2 * gm - (float)(int)(A.X[p - 2 * dir] + k0));
      const int h2 = (int)(2 * gp - (float)(int)(A.X[p + 2 * dir] + k0));
      int eg = (int)(k0 + (float)((h1 + h2) / 4));
      int mn = (int)smin(gm, gp);
      int mx = (int)smax(gm, gp);
      mn -= mn / 8;
      mx += mx / 8;
      if (eg < mn)
        eg = (int)((float)mn - sqrtf((float)(mn - eg)));
      else if (eg > mx)
        eg = (int)((float)mx + sqrtf((float)(eg - mx)));
      if ((float)eg > gmax)
        eg = (int)gmax;
      else if ((float)eg < gmin)
        eg = (int)gmin;
      A.pl(d, 1)[p] = (float)eg;
    }
  }
}

__device__ __forceinline__ int clamp_channel(int eg, const float* stats, int c) {
  if ((float)eg > stats[c]) return (int)stats[c];
  if ((float)eg < stats[3 + c]) return (int)stats[3 + c];
  return eg;
}

// make_ahd_rb_hv (:464-486): at green sites, the colour of the direction's
// neighbours from their samples and interpolated greens.
__global__ void k_aahd_rb_hv(Aahd A) {
  AAHD_FOR_PIXELS(A) {
    if (A.fc(i, j) != 1) continue;
    const int js = (int)(A.fc(i, 0) & 1);
    const int kc = (int)A.fc(i, js);
    const size_t p = A.pi(i, j);
#pragma unroll
    for (int d = 0; d < 2; d++) {
      const ptrdiff_t dir = d ? (ptrdiff_t)A.NW : 1;
      const int c = kc ^ (d << 1);
      const float* G = A.pl(d, 1);
      const float* Cc = A.pl(d, c);
      int eg = (int)(G[p] + (Cc[p - dir] - G[p - dir] + Cc[p + dir] - G[p + dir]) / 2);
      A.pl(d, c)[p] = (float)clamp_channel(eg, A.stats, c);
    }
  }
}

// make_ahd_rb_last (:488-519): the remaining colour at every site from the
// best-matching pair of opposite neighbours.
__global__ void k_aahd_rb_last(Aahd A) {
  AAHD_FOR_PIXELS(A) {
    const int js = (int)(A.fc(i, 0) & 1);
    const int kc = (int)A.fc(i, js);
    const size_t p = A.pi(i, j);
    const ptrdiff_t nw = A.NW;
#pragma unroll
    for (int d = 0; d < 2; d++) {
      int c = kc ^ 2;
      if ((j & 1) != js) c ^= d << 1;
      const ptrdiff_t dirs[3] = {-1 - nw, d ? (ptrdiff_t)-1 : -nw, d ? nw - 1 : 1 - nw};
      const float* G = A.pl(d, 1);
      float* Cc = A.pl(d, c);
      const float g0 = G[p];
      int bh = 0, bk = 0, bgd = 0;
      for (int k = 0; k < 3; ++k)
        for (int h = 0; h < 3; ++h) {
          const size_t a = p + dirs[k], b = p - dirs[h];
          const int gd = (int)(fabsf(2 * g0 - (G[a] + G[b])) + fabsf(Cc[a] - Cc[b]) / 4 +
                               fabsf(Cc[a] - G[a] + G[b] - Cc[b]) / 4);
          if (bgd == 0 || gd < bgd) {
            bgd = gd;
            bh = h;
            bk = k;
          }
        }
      auto dir = [&](int k) { return k == 0 ? dirs[0] : (k == 1 ? dirs[1] : dirs[2]); };
      const size_t a = p + dir(bk), b = p - dir(bh);
      const int eg = (int)(g0 + (Cc[a] - G[a] + Cc[b] - G[b]) / 2);
      Cc[p] = (float)clamp_channel(eg, A.stats, c);
    }
  }
}

__device__ __forceinline__ void yuv_of(const Aahd& A, int d, size_t q, int* y) {
  float l[3];
#pragma unroll
  for (int c = 0; c < 3; c++) {
    const float v = A.pl(d, c)[q];
    const unsigned idx = v <= 0.0f ? 0u : (v >= 65535.0f ? 65535u : (unsigned)v);
    l[c] = g_aahd_gamma[idx];
  }
#pragma unroll
  for (int k = 0; k < 3; k++) y[k] = (int)(c_yuv[k][0] * l[0] + c_yuv[k][1] * l[1] + c_yuv[k][2] * l[2]);
}

__device__ __forceinline__ int wrap_sq(int x) { return (int)((unsigned)x * (unsigned)x); }
__device__ __forceinline__ int wrap_add(int a, int b) { return (int)((unsigned)a + (unsigned)b); }

// evaluate_ahd (:521-556): horizontal vs vertical homogeneity from the
// gamma-mapped YUV of the pixel and its W/E (horizontal image) or N/S
// (vertical image) neighbours.
__global__ void k_aahd_evaluate(Aahd A) {
  AAHD_FOR_PIXELS(A) {
    const size_t p = A.pi(i, j);
    const ptrdiff_t nw = A.NW;
    int y0[3], ya[3], yb[3];
    yuv_of(A, 0, p, y0);
    yuv_of(A, 0, p - 1, ya);
    yuv_of(A, 0, p + 1, yb);
    const float yd00 = (float)abs(y0[0] - ya[0]), yd01 = (float)abs(y0[0] - yb[0]);
    const int uv00 = wrap_add(wrap_sq(y0[1] - ya[1]), wrap_sq(y0[2] - ya[2]));
    const int uv01 = wrap_add(wrap_sq(y0[1] - yb[1]), wrap_sq(y0[2] - yb[2]));
    yuv_of(A, 1, p, y0);
    yuv_of(A, 1, p - nw, ya);
    yuv_of(A, 1, p + nw, yb);
    const float yd12 = (float)abs(y0[0] - ya[0]), yd13 = (float)abs(y0[0] - yb[0]);
    const int uv12 = wrap_add(wrap_sq(y0[1] - ya[1]), wrap_sq(y0[2] - ya[2]));
    const int uv13 = wrap_add(wrap_sq(y0[1] - yb[1]), wrap_sq(y0[2] - yb[2]));
    const float toth = yd00 + yd01 + (float)wrap_add(uv00, uv01) / 1000.0f;
    const float totv = yd12 + yd13 + (float)wrap_add(uv12, uv13) / 1000.0f;
    int nd = 0;
    if (totv < toth * 1.2f) nd |= kVer;
    if (toth < totv * 1.2f) nd |= kHor;
    if (nd == 0) nd = kHor | kVer;
    A.ND[p] = (float)nd;
  }
}

// refine_hv_dirs (:558-584) in order: per row, the even columns then the odd
// ones, each reading its N/S/W/E flags.  Position c of the walk refines the
// even column c and then the odd column c - 1 (whose E neighbour c is then
// already refined, as in the reference); the walk runs one column past the
// image so the last odd column is reached.  Every neighbour read precedes or
// follows the site exactly as in the row-major loops with skew 1.
struct OpRefineDirs {
  static constexpr int NS = 1, NP = 1, HALO = 1, SKEW = 1, PAIR = 1, NCH = 1, LAG = 1, RING = kRing;
  template <class T>
  __device__ static void upd(const T& t, int r, int c) {
    const int n = (int)t(0, r - 1, c), s = (int)t(0, r + 1, c), w = (int)t(0, r, c - 1), e = (int)t(0, r, c + 1);
    int m = (int)t(0, r, c);
    const int nv = ((n & kVer) + (s & kVer) + (w & kVer) + (e & kVer)) / kVer;
    const int nh = ((n & kHor) + (s & kHor) + (w & kHor) + (e & kHor)) / kHor;
    const bool codir = (m & kVer) ? ((n & kVer) || (s & kVer)) : ((w & kHor) || (e & kHor));
    if ((m & kVer) && (nh > 2 && !codir)) m = kHor;
    if ((m & kHor) && (nv > 2 && !codir)) m = kVer;
    t(0, r, c) = (float)m;
  }
  // g.W here is the padded width; image columns are [kMargin, g.W - kMargin).
  template <class T>
  __device__ static void cell(const T& t, int r, int c, const Geo& g) {
    const int j = c - kMargin;
    if (j & 1) return;
    if (c < g.W - kMargin) upd(t, r, c);
    if (j >= 1) upd(t, r, c - 1);
  }
};

__global__ void k_aahd_combine(Aahd A, float* __restrict__ rgb) {
  AAHD_FOR_PIXELS(A) {
    const size_t p = A.pi(i, j);
    const int d = ((int)A.ND[p] & kVer) ? 1 : 0;
    float* o = rgb + ((size_t)i * A.W + j) * 3;
    o[0] = A.pl(d, 0)[p] / A.maxv;
    o[1] = A.pl(d, 1)[p] / A.maxv;
    o[2] = A.pl(d, 2)[p] / A.maxv;
  }
}

// The reference's gamma table (:246-253), evaluated on the host with the
// same expression and uploaded once per device when a context is created
// (outside any stream capture).
std::mutex g_lut_mu;
bool g_lut_done[64];

}  // namespace

lre_status aahd_upload_gamma(Context* c) {
  std::lock_guard<std::mutex> lk(g_lut_mu);
  if (c->device >= 0 && c->device < 64 && g_lut_done[c->device]) return LRE_OK;
  static float lut[0x10000];
  static bool built = false;
  if (!built) {
    for (int i = 0; i < 0x10000; i++) {
      const float r = (float)i / 0x10000;
      lut[i] = 0x10000 * (r < 0.0181 ? 4.5f * r : 1.0993f * powf(r, 0.45f) - 0.0993f);
    }
    built = true;
  }
  LRE_CUDA_TRY(c, cudaMemcpyToSymbol(g_aahd_gamma, lut, sizeof(lut)));
  if (c->device >= 0 && c->device < 64) g_lut_done[c->device] = true;
  return LRE_OK;
}

namespace {

size_t padded_bytes(size_t w, size_t h) {
  return (((w + 2 * kMargin) * (h + 2 * kMargin) * sizeof(float)) + 255) & ~size_t(255);
}

}  // namespace

size_t ws_bytes_aahd(size_t w, size_t h) {
  const size_t nb = 2 * ((h + 2 * kMargin + 31) / 32 + 1);
  return 8 * padded_bytes(w, h) + 256 + (kSyncInts + nb) * sizeof(int) + 1024;
}

lre_status launch_aahd(Context* c, const float* raw, int raw_c_stride, float* rgb, size_t w, size_t h,
                       uint32_t filters, float maximum_value, int* d_err) {
  if (!bayer_2x2(filters))
    return fail(c, LRE_ERR_INVALID_ARGUMENT, "demosaic_bayer_aahd: needs a 2x2 Bayer layout (RGGB/BGGR/GRBG/GBRG)");
  const size_t pb = padded_bytes(w, h);
  Aahd A{};
  A.W = (int)w;
  A.H = (int)h;
  A.NW = (int)w + 2 * kMargin;
  A.filters = filters;
  A.maxv = maximum_value;
  char* base = reinterpret_cast<char*>(c->ws.take(8 * pb));
  float* stats = reinterpret_cast<float*>(c->ws.take(256));
  const int nb_max = 2 * (int)((h + 2 * kMargin + 31) / 32 + 1);
  int* sync = reinterpret_cast<int*>(c->ws.take((kSyncInts + nb_max) * sizeof(int)));
  if (!base || !stats || !sync) return fail(c, LRE_ERR_CUDA, "demosaic_bayer_aahd: workspace not reserved");
  auto plane = [&](int k) { return reinterpret_cast<float*>(base + (size_t)k * pb); };
  A.X = plane(0);
  for (int d = 0; d < 2; d++)
    for (int ch = 0; ch < 3; ch++) A.P[d][ch] = plane(1 + 3 * d + ch);
  A.ND = plane(7);
  A.stats = stats;
  A.hot = reinterpret_cast<int*>(stats + 8);
  cudaStream_t s = c->stream;
  LRE_CUDA_TRY(c, cudaMemsetAsync(base, 0, 8 * pb, s));
  int* err = d_err ? d_err : sync + 1;
  if (!d_err) LRE_CUDA_TRY(c, cudaMemsetAsync(err, 0, sizeof(int), s));
  k_aahd_stats_init<<<1, 32, 0, s>>>(raw, raw_c_stride, A);
  count_launch(c);
  LRE_TRY(check_launch(c, "demosaic_bayer_aahd"));

  const dim3 blk(32, 8);
  const dim3 grd((unsigned)std::min<size_t>((w + 63) / 64, 1024), (unsigned)std::min<size_t>((h + 7) / 8, 8192));
#define AAHD_LAUNCH(k, ...)                             \
  do {                                                  \
    k<<<grd, blk, 0, s>>>(__VA_ARGS__);                 \
    count_launch(c);                                    \
    LRE_TRY(check_launch(c, "demosaic_bayer_aahd"));    \
  } while (0)

  AAHD_LAUNCH(k_aahd_init, raw, raw_c_stride, A);
  AAHD_LAUNCH(k_aahd_hot_pretest, A);
  SweepArgs sa{};
  sa.g = Geo{A.NW, (int)h + 2 * kMargin, filters, maximum_value};
  sa.err = err;
  {
    SweepArgs hh = sa;
    hh.plane[0] = A.X;
    hh.r_lo = kMargin;
    hh.r_hi = (int)h + kMargin - 1;
    hh.c_lo = kMargin;
    hh.c_hi = (int)w + kMargin - 1;
    hh.skip_if_zero = A.hot;
    LRE_TRY(sweep<OpHideHots>(c, hh, sync, nb_max, "aahd_hide_hots"));
  }
  AAHD_LAUNCH(k_aahd_greens, A);
  AAHD_LAUNCH(k_aahd_rb_hv, A);
  AAHD_LAUNCH(k_aahd_rb_last, A);
  AAHD_LAUNCH(k_aahd_evaluate, A);
  {
    SweepArgs rd = sa;
    rd.plane[0] = A.ND;
    rd.r_lo = kMargin;
    rd.r_hi = (int)h + kMargin - 1;
    rd.c_lo = kMargin;
    rd.c_hi = (int)w + kMargin;  // one past the image: the last odd column
    LRE_TRY(sweep<OpRefineDirs>(c, rd, sync, nb_max, "aahd_refine_dirs"));
  }
  AAHD_LAUNCH(k_aahd_combine, A, rgb);
#undef AAHD_LAUNCH
  LRE_TRY(launch_border_interp(c, rgb, w, h, filters, 2));
  if (d_err) return LRE_OK;  // the caller reads the flag after its own synchronisation
  int e = 0;
  LRE_CUDA_TRY(c, cudaMemcpyAsync(&e, err, sizeof(int), cudaMemcpyDeviceToHost, s));
  LRE_CUDA_TRY(c, cudaStreamSynchronize(s));
  if (e) return fail(c, LRE_ERR_TIMEOUT, "demosaic_bayer_aahd: a sweep band timed out waiting for the band above");
  return LRE_OK;
}

}  // namespace lre
