// k_dcb.cu -- DCB Bayer demosaic (CPUAccelerator::demosaic_bayer_dcb,
// core/cpu_accelerator.cpp:1043-1137, running DCB_Processor::run_dcb,
// :998-1035; Accelerator::demosaic_bayer_dcb defaults iterations = 1 and
// dcb_enhance = true, core/accelerator.h:273-277).
//
// Layout.  The reference keeps one float[4] per pixel (R, G, B, direction
// map) plus two float[3] scratch images.  Here every channel is its own W*H
// plane in HBM: R, G, B and four scratch planes as float, the map as bytes.
// The scratch images of the reference are never materialised:
//   * dcb_hor/dcb_ver/dcb_color2/dcb_color3 only feed dcb_decide, which reads
//     the green estimates and the first-loop chroma estimates at non-green
//     sites -- four planes (k_dcb_hv, k_dcb_hvc), then k_dcb_decide;
//   * dcb_copy_to_buffer / dcb_restore_from_buffer put R and B back to their
//     seeded values, and dcb_color only reads the native samples of R and B,
//     so "restore + color" is one kernel that reads the mosaic (k_dcb_color).
//
// Ordering.  Most DCB passes read only channels the pass does not write, so
// they run one thread per pixel.  Four do not, and the reference's
// row-major loops define a Gauss-Seidel order for them:
//   * dcb_nyquist: a site reads the new green two rows up and two columns left;
//   * dcb_pp: the new R/B of its W, NW, N and NE neighbours;
//   * dcb_refinement: its final clamp reads the new green of the NW/NE sites;
//   * the last dcb_color_full loop: the new R/B of W, NW, N and NE.
// (Three of these are OpenMP row-parallel loops in the reference, so with
// more than one thread rows at chunk boundaries depend on timing; the
// sequential order is the defined result and the one computed here.)
// k_gs_sweep (sweep.cuh) evaluates them in exactly that order with one warp
// per 32-row band walking the columns on a skewed wavefront.
//
// Arithmetic is the reference's, operation for operation (--fmad=false); the
// result is bit-identical to the reference run single-threaded.
#include "common.cuh"
#include "lre_internal.h"
#include "stencil.cuh"
#include "sweep.cuh"

namespace lre {

namespace {

__device__ __forceinline__ float dclip(float v, float m) { return v > m ? m : (v < 0.0f ? 0.0f : v); }
// ulim_generic (core/metal/shader_common.h:37-42)
__device__ __forceinline__ float ulim(float v, float hi, float lo) { return v > hi ? hi : (v < lo ? lo : v); }

__device__ __forceinline__ float raw_at(const float* __restrict__ raw, int cs, const Geo& g, int r, int c) {
  const size_t i = g.at(r, c);
  return cs == 1 ? raw[i] : raw[i * 3 + g.fc(r, c)];
}

// Seed (cpu_accelerator.cpp:1061-1116): each site keeps its own sample; in
// the interior each missing colour is the mean of that colour's samples in
// the 8-neighbourhood (summed in row-major order).
__global__ void k_dcb_init(const float* __restrict__ raw, int cs, float* __restrict__ R, float* __restrict__ G,
                           float* __restrict__ B, Geo g) {
  GS_FOR_PIXELS(g) {
    const unsigned f = g.fc(r, c);
    float v[3] = {0.0f, 0.0f, 0.0f};
    v[f] = raw_at(raw, cs, g, r, c);
    if (r >= 1 && r < g.H - 1 && c >= 1 && c < g.W - 1) {
      for (unsigned ch = 0; ch < 3; ch++) {
        if (ch == f) continue;
        float sum = 0.0f;
        int count = 0;
        for (int dr = -1; dr <= 1; dr++)
          for (int dc = -1; dc <= 1; dc++) {
            if (dr == 0 && dc == 0) continue;
            if (g.fc(r + dr, c + dc) == ch) {
              sum += raw_at(raw, cs, g, r + dr, c + dc);
              count++;
            }
          }
        if (count > 0) v[ch] = sum / count;
      }
    }
    const size_t i = g.at(r, c);
    R[i] = v[0];
    G[i] = v[1];
    B[i] = v[2];
  }
}

// dcb_hor / dcb_ver (:677-697): green from the horizontal / vertical pair at
// non-green sites of rows/cols [2, n-3]; zero elsewhere (the scratch images
// start zeroed).
__global__ void k_dcb_hv(const float* __restrict__ G, float* __restrict__ H1, float* __restrict__ V1, Geo g) {
  GS_FOR_PIXELS(g) {
    const size_t i = g.at(r, c);
    float h = 0.0f, v = 0.0f;
    if (g.fc(r, c) != 1 && r >= 2 && r < g.H - 2 && c >= 2 && c < g.W - 2) {
      h = dclip((G[i + 1] + G[i - 1]) / 2.0f, g.maxv);
      v = dclip((G[i + g.W] + G[i - g.W]) / 2.0f, g.maxv);
    }
    H1[i] = h;
    V1[i] = v;
  }
}

// First loops of dcb_color2 / dcb_color3 (:724-760): the opposite colour at
// non-green sites of rows/cols [1, n-2] from each scratch green and the
// diagonal samples; zero elsewhere.  (Their second loops write green sites,
// which dcb_decide never reads.)
__global__ void k_dcb_hvc(const float* __restrict__ R, const float* __restrict__ B, const float* __restrict__ H1,
                          const float* __restrict__ V1, float* __restrict__ HC, float* __restrict__ VC, Geo g) {
  GS_FOR_PIXELS(g) {
    const size_t i = g.at(r, c);
    float hc = 0.0f, vc = 0.0f;
    const unsigned f = g.fc(r, c);
    if (f != 1 && r >= 1 && r < g.H - 1 && c >= 1 && c < g.W - 1) {
      const float* X = (2 - f) == 0 ? R : B;
      const size_t u = g.W;
      hc = dclip((4 * H1[i] - H1[i + u + 1] - H1[i + u - 1] - H1[i - u + 1] - H1[i - u - 1] + X[i + u + 1] +
                  X[i + u - 1] + X[i - u + 1] + X[i - u - 1]) /
                     4.0f,
                 g.maxv);
      vc = dclip((4 * V1[i] - V1[i + u + 1] - V1[i + u - 1] - V1[i - u + 1] - V1[i - u - 1] + X[i + u + 1] +
                  X[i + u - 1] + X[i - u + 1] + X[i - u - 1]) /
                     4.0f,
                 g.maxv);
    }
    HC[i] = hc;
    VC[i] = vc;
  }
}

__device__ __forceinline__ float max4(float a, float b, float c, float d) { return smax(smax(smax(a, b), c), d); }
__device__ __forceinline__ float min4(float a, float b, float c, float d) { return smin(smin(smin(a, b), c), d); }

// max - min + max - min of two 4-sample sets, left to right as written.
__device__ __forceinline__ float spread(const float* __restrict__ Pa, const float* __restrict__ Pb, size_t i,
                                        size_t u) {
  const size_t v = 2 * u;
  return max4(Pa[i + v], Pa[i - v], Pa[i - 2], Pa[i + 2]) - min4(Pa[i + v], Pa[i - v], Pa[i - 2], Pa[i + 2]) +
         max4(Pb[i + 1 + u], Pb[i + 1 - u], Pb[i - 1 + u], Pb[i - 1 - u]) -
         min4(Pb[i + 1 + u], Pb[i + 1 - u], Pb[i - 1 + u], Pb[i - 1 - u]);
}

// dcb_decide (:774-798): per non-green site of rows/cols [2, n-3], keep the
// horizontal or the vertical green, whichever scratch image's local colour
// ranges are closer to the seeded image's.
__global__ void k_dcb_decide(const float* __restrict__ R, const float* __restrict__ B, const float* __restrict__ H1,
                             const float* __restrict__ V1, const float* __restrict__ HC,
                             const float* __restrict__ VC, float* __restrict__ G, Geo g) {
  GS_FOR_PIXELS(g) {
    const unsigned f = g.fc(r, c);
    if (f == 1 || r < 2 || r >= g.H - 2 || c < 2 || c >= g.W - 2) continue;
    const size_t i = g.at(r, c), u = g.W;
    const float cur = f == 0 ? spread(R, B, i, u) : spread(B, R, i, u);
    const float cur2 = spread(HC, HC, i, u);
    const float cur3 = spread(VC, VC, i, u);
    G[i] = (fabsf(cur - cur2) < fabsf(cur - cur3)) ? H1[i] : V1[i];
  }
}

// dcb_map (:917-930): direction flag per pixel of rows/cols [1, n-2].
__global__ void k_dcb_map(const float* __restrict__ G, uint8_t* __restrict__ M, Geo g) {
  GS_FOR_PIXELS(g) {
    if (r < 1 || r >= g.H - 1 || c < 1 || c >= g.W - 1) continue;
    const size_t i = g.at(r, c), u = g.W;
    const float w = G[i - 1], e = G[i + 1], n = G[i - u], s = G[i + u];
    bool m;
    if (G[i] > (w + e + n + s) / 4.0f)
      m = (smin(w, e) + w + e) < (smin(n, s) + n + s);
    else
      m = (smax(w, e) + w + e) > (smax(n, s) + n + s);
    M[i] = m ? 1 : 0;
  }
}

__device__ __forceinline__ int map_weight(const uint8_t* __restrict__ M, size_t i, size_t u) {
  return 4 * M[i] + 2 * (M[i + u] + M[i - u] + M[i + 1] + M[i - 1]) + M[i + 2 * u] + M[i - 2 * u] + M[i + 2] +
         M[i - 2];
}

// dcb_correction (:932-941) and dcb_correction2 (:943-957): green at
// non-green sites re-blended from the map-weighted directions.  Both read
// green only at green sites, so they run in place.
__global__ void k_dcb_correction(float* __restrict__ G, const uint8_t* __restrict__ M, Geo g) {
  GS_FOR_PIXELS(g) {
    if (g.fc(r, c) == 1 || r < 2 || r >= g.H - 2 || c < 2 || c >= g.W - 2) continue;
    const size_t i = g.at(r, c), u = g.W;
    const int cur = map_weight(M, i, u);
    G[i] = ((16 - cur) * (G[i - 1] + G[i + 1]) / 2.0f + cur * (G[i - u] + G[i + u]) / 2.0f) / 16.0f;
  }
}

__global__ void k_dcb_correction2(float* __restrict__ G, const float* __restrict__ R, const float* __restrict__ B,
                                  const uint8_t* __restrict__ M, Geo g) {
  GS_FOR_PIXELS(g) {
    const unsigned f = g.fc(r, c);
    if (f == 1 || r < 4 || r >= g.H - 4 || c < 4 || c >= g.W - 4) continue;
    const size_t i = g.at(r, c), u = g.W, v = 2 * (size_t)g.W;
    const float* X = f == 0 ? R : B;
    const int cur = map_weight(M, i, u);
    G[i] = dclip(((16 - cur) * ((G[i - 1] + G[i + 1]) / 2.0f + X[i] - (X[i + 2] + X[i - 2]) / 2.0f) +
                  cur * ((G[i - u] + G[i + u]) / 2.0f + X[i] - (X[i + v] + X[i - v]) / 2.0f)) /
                     16.0f,
                 g.maxv);
  }
}

// dcb_restore_from_buffer + dcb_color (:699-722, :810-818): R and B back to
// their seeded values, then the missing colours of rows/cols [1, n-2] from
// green and the neighbouring samples.  The seeded R/B outside that frame is
// the site's own sample (or 0), and inside it every value the formulas read
// is a native sample, so the kernel reads the mosaic instead of R/B.
__global__ void k_dcb_color(const float* __restrict__ raw, int cs, const float* __restrict__ G,
                            float* __restrict__ R, float* __restrict__ B, Geo g) {
  GS_FOR_PIXELS(g) {
    const size_t i = g.at(r, c), u = g.W;
    const unsigned f = g.fc(r, c);
    float rv = 0.0f, bv = 0.0f;
    if (f == 0) rv = raw_at(raw, cs, g, r, c);
    if (f == 2) bv = raw_at(raw, cs, g, r, c);
    if (r >= 1 && r < g.H - 1 && c >= 1 && c < g.W - 1) {
      if (f != 1) {
        const float x = dclip((4 * G[i] - G[i + u + 1] - G[i + u - 1] - G[i - u + 1] - G[i - u - 1] +
                               raw_at(raw, cs, g, r + 1, c + 1) + raw_at(raw, cs, g, r + 1, c - 1) +
                               raw_at(raw, cs, g, r - 1, c + 1) + raw_at(raw, cs, g, r - 1, c - 1)) /
                                  4.0f,
                              g.maxv);
        if (f == 0) bv = x; else rv = x;
      } else {
        const unsigned cc = g.fc(r, c + 1);
        const float xc = dclip((2 * G[i] - G[i + 1] - G[i - 1] + raw_at(raw, cs, g, r, c + 1) +
                                raw_at(raw, cs, g, r, c - 1)) /
                                   2.0f,
                               g.maxv);
        const float xd = dclip((2 * G[i] - G[i + u] - G[i - u] + raw_at(raw, cs, g, r + 1, c) +
                                raw_at(raw, cs, g, r - 1, c)) /
                                   2.0f,
                               g.maxv);
        if (cc == 0) { rv = xc; bv = xd; } else { bv = xc; rv = xd; }
      }
    }
    R[i] = rv;
    B[i] = bv;
  }
}

// dcb_refinement (:959-996), everything but the final clamp: the green at
// non-green sites of rows/cols [4, n-5] from the ratio-weighted vertical and
// horizontal estimates.  It reads green only at green sites, so every site
// is independent; the clamp against the 8 neighbours is the sweep below.
__global__ void k_dcb_refine_pre(const float* __restrict__ G, const float* __restrict__ R,
                                 const float* __restrict__ B, const uint8_t* __restrict__ M,
                                 float* __restrict__ V, Geo g) {
  GS_FOR_PIXELS(g) {
    const unsigned f = g.fc(r, c);
    if (f == 1 || r < 4 || r >= g.H - 4 || c < 4 || c >= g.W - 4) continue;
    const size_t i = g.at(r, c), u = g.W, v = 2 * (size_t)g.W, w = 3 * (size_t)g.W;
    const float* X = f == 0 ? R : B;
    const int cur = map_weight(M, i, u);
    const float x = X[i];
    float out;
    if (x > 1) {
      float f0 = (G[i - u] + G[i + u]) / (2.0f * x);
      float f1 = (X[i - v] > 0) ? 2.0f * G[i - u] / (X[i - v] + x) : f0;
      float f2 = (X[i - v] > 0) ? (G[i - u] + G[i - w]) / (2.0f * X[i - v]) : f0;
      float f3 = (X[i + v] > 0) ? 2.0f * G[i + u] / (X[i + v] + x) : f0;
      float f4 = (X[i + v] > 0) ? (G[i + u] + G[i + w]) / (2.0f * X[i + v]) : f0;
      const float g1 = (5.0f * f0 + 3.0f * f1 + f2 + 3.0f * f3 + f4) / 13.0f;
      f0 = (G[i - 1] + G[i + 1]) / (2.0f * x);
      f1 = (X[i - 2] > 0) ? 2.0f * G[i - 1] / (X[i - 2] + x) : f0;
      f2 = (X[i - 2] > 0) ? (G[i - 1] + G[i - 3]) / (2.0f * X[i - 2]) : f0;
      f3 = (X[i + 2] > 0) ? 2.0f * G[i + 1] / (X[i + 2] + x) : f0;
      f4 = (X[i + 2] > 0) ? (G[i + 1] + G[i + 3]) / (2.0f * X[i + 2]) : f0;
      const float g2 = (5.0f * f0 + 3.0f * f1 + f2 + 3.0f * f3 + f4) / 13.0f;
      out = dclip(x * (cur * g1 + (16 - cur) * g2) / 16.0f, g.maxv);
    } else {
      out = x;
    }
    V[i] = out;
  }
}

// dcb_color_full (:850-915), first two loops: the native chroma (sample -
// green) at non-green sites of rows/cols [1, n-2], and the opposite chroma
// at non-green sites of rows/cols [3, n-4] from the eight surrounding
// opposite-colour sites; zero elsewhere.  Native chroma is recomputed on the
// fly where the second loop needs it.
__device__ __forceinline__ float chroma_native(const float* __restrict__ R, const float* __restrict__ B,
                                               const float* __restrict__ G, const Geo& g, int r, int c) {
  if (r < 1 || r >= g.H - 1 || c < 1 || c >= g.W - 1) return 0.0f;
  const size_t i = g.at(r, c);
  return (g.fc(r, c) == 0 ? R[i] : B[i]) - G[i];
}

// The native chroma of every non-green site (0 outside the first loop's
// frame), stored once for the second loop's eight-site reads.
__global__ void k_dcb_chroma_native(const float* __restrict__ R, const float* __restrict__ B,
                                    const float* __restrict__ G, float* __restrict__ N, Geo g) {
  GS_FOR_PIXELS(g) {
    if (g.fc(r, c) == 1) continue;
    N[g.at(r, c)] = chroma_native(R, B, G, g, r, c);
  }
}

__global__ void k_dcb_chroma(const float* __restrict__ N, float* __restrict__ C0, float* __restrict__ C1, Geo g) {
  GS_FOR_PIXELS(g) {
    const unsigned f = g.fc(r, c);
    if (f == 1) continue;
    const float nat = N[g.at(r, c)];
    float opp = 0.0f;
    if (r >= 3 && r < g.H - 3 && c >= 3 && c < g.W - 3) {
      auto ch = [&](int dr, int dc) { return N[g.at(r + dr, c + dc)]; };
      const float a = ch(-1, -1), b = ch(1, 1), d = ch(-1, 1), e = ch(1, -1);
      const float f0 = 1.0f / (1.0f + fabsf(a - b) + fabsf(a - ch(-3, -3)) + fabsf(b - ch(-3, -3)));
      const float f1 = 1.0f / (1.0f + fabsf(d - e) + fabsf(d - ch(-3, 3)) + fabsf(e - ch(-3, 3)));
      const float f2 = 1.0f / (1.0f + fabsf(e - d) + fabsf(e - ch(3, 3)) + fabsf(d - ch(3, -3)));
      const float f3 = 1.0f / (1.0f + fabsf(b - a) + fabsf(b - ch(3, -3)) + fabsf(a - ch(3, 3)));
      const float g0 = 1.325f * a - 0.175f * ch(-3, -3) - 0.075f * ch(-3, -1) - 0.075f * ch(-1, -3);
      const float g1 = 1.325f * d - 0.175f * ch(-3, 3) - 0.075f * ch(-3, 1) - 0.075f * ch(-1, 3);
      const float g2 = 1.325f * e - 0.175f * ch(3, -3) - 0.075f * ch(3, -1) - 0.075f * ch(1, -3);
      const float g3 = 1.325f * b - 0.175f * ch(3, 3) - 0.075f * ch(3, 1) - 0.075f * ch(1, 3);
      opp = (f0 * g0 + f1 * g1 + f2 * g2 + f3 * g3) / (f0 + f1 + f2 + f3);
    }
    const size_t i = g.at(r, c);
    (f == 0 ? C0 : C1)[i] = nat;
    (f == 0 ? C1 : C0)[i] = opp;
  }
}

// dcb_color_full, third loop (chroma at green sites from the four
// non-green neighbours at distance 1 and 3) fused with the value the last
// loop assigns before its clamp: V = CLIP(chroma + green) over rows/cols
// [6, n-7].
__global__ void k_dcb_chroma_g(const float* __restrict__ C0, const float* __restrict__ C1,
                               const float* __restrict__ G, float* __restrict__ V0, float* __restrict__ V2, Geo g) {
  GS_FOR_PIXELS(g) {
    if (r < 6 || r >= g.H - 6 || c < 6 || c >= g.W - 6) continue;
    const size_t i = g.at(r, c), u = g.W, w = 3 * (size_t)g.W;
    float cr[2];
    if (g.fc(r, c) != 1) {
      cr[0] = C0[i];
      cr[1] = C1[i];
    } else {
      int k = (int)g.fc(r, c + 1) / 2;
      for (int d = 0; d <= 1; k = 1 - k, d++) {
        const float* C = k == 0 ? C0 : C1;
        const float f0 = 1.0f / (1.0f + fabsf(C[i - u] - C[i + u]) + fabsf(C[i - u] - C[i - w]) + fabsf(C[i + u] - C[i - w]));
        const float f1 = 1.0f / (1.0f + fabsf(C[i + 1] - C[i - 1]) + fabsf(C[i + 1] - C[i + 3]) + fabsf(C[i - 1] - C[i + 3]));
        const float f2 = 1.0f / (1.0f + fabsf(C[i - 1] - C[i + 1]) + fabsf(C[i - 1] - C[i - 3]) + fabsf(C[i + 1] - C[i - 3]));
        const float f3 = 1.0f / (1.0f + fabsf(C[i + u] - C[i - u]) + fabsf(C[i + u] - C[i + w]) + fabsf(C[i - u] - C[i + w]));
        const float g0 = 0.875f * C[i - u] + 0.125f * C[i - w];
        const float g1 = 0.875f * C[i + 1] + 0.125f * C[i + 3];
        const float g2 = 0.875f * C[i - 1] + 0.125f * C[i - 3];
        const float g3 = 0.875f * C[i + u] + 0.125f * C[i + w];
        cr[k] = (f0 * g0 + f1 * g1 + f2 * g2 + f3 * g3) / (f0 + f1 + f2 + f3);
      }
    }
    V0[i] = dclip(cr[0] + G[i], g.maxv);
    V2[i] = dclip(cr[1] + G[i], g.maxv);
  }
}

__global__ void k_dcb_output(const float* __restrict__ R, const float* __restrict__ G, const float* __restrict__ B,
                             float* __restrict__ rgb, Geo g) {
  GS_FOR_PIXELS(g) {
    const size_t i = g.at(r, c);
    rgb[i * 3 + 0] = R[i] / g.maxv;
    rgb[i * 3 + 1] = G[i] / g.maxv;
    rgb[i * 3 + 2] = B[i] / g.maxv;
  }
}

// Terms of dcb_nyquist that do not change during the pass: the site's own
// sample and (S + N + W + E) / 4 of the same colour two sites away.
__global__ void k_dcb_nyq_terms(const float* __restrict__ R, const float* __restrict__ B, float* __restrict__ A,
                                float* __restrict__ Q, Geo g) {
  GS_FOR_PIXELS(g) {
    const unsigned f = g.fc(r, c);
    if (f == 1 || r < 2 || r >= g.H - 2 || c < 2 || c >= g.W - 2) continue;
    const size_t i = g.at(r, c), v = 2 * (size_t)g.W;
    const float* X = f == 0 ? R : B;
    A[i] = X[i];
    Q[i] = (X[i + v] + X[i - v] + X[i - 2] + X[i + 2]) / 4.0f;
  }
}

// dcb_pp's green term G - mean8(G), in the reference's summation order.
__global__ void k_dcb_pp_terms(const float* __restrict__ G, float* __restrict__ K, Geo g) {
  GS_FOR_PIXELS(g) {
    if (r < 2 || r >= g.H - 2 || c < 2 || c >= g.W - 2) continue;
    const size_t i = g.at(r, c), u = g.W;
    const float g1 = (G[i - 1] + G[i + 1] + G[i - u] + G[i + u] + G[i - u - 1] + G[i + u + 1] + G[i - u + 1] +
                      G[i + u - 1]) /
                     8.0f;
    K[i] = G[i] - g1;
  }
}

// ------------------------------------------------------------------ sweeps

// Each sweep op names its planes per warp: NS state planes first, then
// inputs.  NCH = 2 runs two independent channels (R and B) as separate
// warps; PAIR = 2 gives two adjacent rows the same column when a row only
// depends on rows two above it.

// dcb_nyquist (:836-848): state G; inputs the site's own sample A and the
// quarter-sum Q of the four same-colour samples two sites away (k_dcb_nyq_terms;
// R and B do not change across the nyquist passes).  A site reads rows r +- 2
// only, so rows r and r + 1 advance together.
struct OpNyquist {
  static constexpr int NS = 1, NP = 3, HALO = 2, SKEW = 1, PAIR = 2, NCH = 1, LAG = 0, RING = kRing;
  template <class T>
  __device__ static void cell(const T& t, int r, int c, const Geo& g) {
    if (g.fc(r, c) == 1) return;
    t(0, r, c) = dclip((t(0, r + 2, c) + t(0, r - 2, c) + t(0, r, c - 2) + t(0, r, c + 2)) / 4.0f + t(1, r, c) -
                           t(2, r, c),
                       g.maxv);
  }
};

// dcb_pp (:820-834), one channel (R or B) per warp: state the channel;
// input K = G - mean8(G) (k_dcb_pp_terms; green does not change in the pass).
struct OpPP {
  static constexpr int NS = 1, NP = 2, HALO = 1, SKEW = 2, PAIR = 1, NCH = 2, LAG = 0, RING = kRing;
  template <class T>
  __device__ static void cell(const T& t, int r, int c, const Geo& g) {
    const float x1 = (t(0, r, c - 1) + t(0, r, c + 1) + t(0, r - 1, c) + t(0, r + 1, c) + t(0, r - 1, c - 1) +
                      t(0, r + 1, c + 1) + t(0, r - 1, c + 1) + t(0, r + 1, c - 1)) /
                     8.0f;
    t(0, r, c) = dclip(x1 + t(1, r, c), g.maxv);
  }
};

template <class T>
__device__ __forceinline__ void clamp8(const T& t, int p, int r, int c, float v) {
  const float n0 = t(p, r + 1, c + 1), n1 = t(p, r - 1, c + 1), n2 = t(p, r + 1, c - 1), n3 = t(p, r - 1, c - 1),
              n4 = t(p, r, c - 1), n5 = t(p, r, c + 1), n6 = t(p, r - 1, c), n7 = t(p, r + 1, c);
  const float lo = smin(smin(smin(smin(smin(smin(smin(n0, n1), n2), n3), n4), n5), n6), n7);
  const float hi = smax(smax(smax(smax(smax(smax(smax(n0, n1), n2), n3), n4), n5), n6), n7);
  t(p, r, c) = ulim(v, hi, lo);
}

// dcb_refinement's closing clamp (:992-994): state G; input the pre-clamp value.
struct OpRefine {
  static constexpr int NS = 1, NP = 2, HALO = 1, SKEW = 2, PAIR = 1, NCH = 1, LAG = 0, RING = kRing;
  template <class T>
  __device__ static void cell(const T& t, int r, int c, const Geo& g) {
    if (g.fc(r, c) == 1) return;
    clamp8(t, 0, r, c, t(1, r, c));
  }
};

// dcb_color_full's last loop (:898-913), one channel per warp: state R or B;
// input that channel's CLIP(chroma + G).
struct OpColorFull {
  static constexpr int NS = 1, NP = 2, HALO = 1, SKEW = 2, PAIR = 1, NCH = 2, LAG = 0, RING = kRing;
  template <class T>
  __device__ static void cell(const T& t, int r, int c, const Geo&) {
    clamp8(t, 0, r, c, t(1, r, c));
  }
};

size_t plane_bytes(size_t w, size_t h) { return (w * h * sizeof(float) + 255) & ~size_t(255); }

}  // namespace

bool bayer_2x2_layout(uint32_t filters) { return bayer_2x2(filters); }

size_t ws_bytes_dcb(size_t w, size_t h) {
  const size_t nb = 2 * ((h + 31) / 32 + 1);
  return 7 * plane_bytes(w, h) + ((w * h + 255) & ~size_t(255)) + (kSyncInts + nb) * sizeof(int) + 1024;
}

lre_status launch_dcb(Context* c, const float* raw, int raw_c_stride, float* rgb, size_t w, size_t h,
                      uint32_t filters, float maximum_value, int iterations, bool enhance, int* d_err) {
  if (!bayer_2x2(filters))
    return fail(c, LRE_ERR_INVALID_ARGUMENT, "demosaic_bayer_dcb: needs a 2x2 Bayer layout (RGGB/BGGR/GRBG/GBRG)");
  if (iterations < 0) return fail(c, LRE_ERR_INVALID_ARGUMENT, "demosaic_bayer_dcb: negative iterations");
  const size_t pb = plane_bytes(w, h);
  auto take = [&](size_t b) { return c->ws.take(b); };
  float* R = reinterpret_cast<float*>(take(pb));
  float* G = reinterpret_cast<float*>(take(pb));
  float* B = reinterpret_cast<float*>(take(pb));
  float* P1 = reinterpret_cast<float*>(take(pb));
  float* P2 = reinterpret_cast<float*>(take(pb));
  float* P3 = reinterpret_cast<float*>(take(pb));
  float* P4 = reinterpret_cast<float*>(take(pb));
  uint8_t* M = reinterpret_cast<uint8_t*>(take((w * h + 255) & ~size_t(255)));
  const int nb_max = 2 * (int)((h + 31) / 32 + 1);
  int* sync = reinterpret_cast<int*>(take((kSyncInts + nb_max) * sizeof(int)));
  if (!R || !G || !B || !P1 || !P2 || !P3 || !P4 || !M || !sync)
    return fail(c, LRE_ERR_CUDA, "demosaic_bayer_dcb: workspace not reserved");

  Geo g{(int)w, (int)h, filters, maximum_value};
  const dim3 blk(32, 8);
  const dim3 grd((unsigned)std::min<size_t>((w + 63) / 64, 1024), (unsigned)std::min<size_t>((h + 7) / 8, 8192));
  cudaStream_t s = c->stream;
#define DCB_LAUNCH(k, ...)                              \
  do {                                                  \
    k<<<grd, blk, 0, s>>>(__VA_ARGS__);                 \
    count_launch(c);                                    \
    LRE_TRY(check_launch(c, "demosaic_bayer_dcb"));     \
  } while (0)

  LRE_CUDA_TRY(c, cudaMemsetAsync(M, 0, w * h, s));
  int* err = d_err ? d_err : sync + 1;
  if (!d_err) LRE_CUDA_TRY(c, cudaMemsetAsync(err, 0, sizeof(int), s));
  DCB_LAUNCH(k_dcb_init, raw, raw_c_stride, R, G, B, g);
  DCB_LAUNCH(k_dcb_hv, G, P1, P2, g);
  DCB_LAUNCH(k_dcb_hvc, R, B, P1, P2, P3, P4, g);
  DCB_LAUNCH(k_dcb_decide, R, B, P1, P2, P3, P4, G, g);

  SweepArgs sa{};
  sa.g = g;
  sa.err = err;
  const int W = (int)w, H = (int)h;
  auto rect = [&](SweepArgs x, int m) {
    x.r_lo = m;
    x.r_hi = H - 1 - m;
    x.c_lo = m;
    x.c_hi = W - 1 - m;
    return x;
  };
  if (iterations > 0) DCB_LAUNCH(k_dcb_nyq_terms, R, B, P1, P2, g);
  for (int it = 1; it <= iterations; it++) {
    SweepArgs ny = rect(sa, 2);
    ny.plane[0] = G;
    ny.plane[1] = P1;
    ny.plane[2] = P2;
    for (int k = 0; k < 3; k++) LRE_TRY(sweep<OpNyquist>(c, ny, sync, nb_max, "dcb_nyquist"));
    DCB_LAUNCH(k_dcb_map, G, M, g);
    DCB_LAUNCH(k_dcb_correction, G, M, g);
  }
  DCB_LAUNCH(k_dcb_color, raw, raw_c_stride, G, R, B, g);
  {
    DCB_LAUNCH(k_dcb_pp_terms, G, P1, g);
    SweepArgs pp = rect(sa, 2);
    pp.plane[0] = R;
    pp.plane[1] = B;
    pp.plane[2] = P1;
    pp.plane[3] = P1;
    LRE_TRY(sweep<OpPP>(c, pp, sync, nb_max, "dcb_pp"));
  }
  DCB_LAUNCH(k_dcb_map, G, M, g);
  DCB_LAUNCH(k_dcb_correction2, G, R, B, M, g);
  for (int k = 0; k < 3; k++) {
    DCB_LAUNCH(k_dcb_map, G, M, g);
    DCB_LAUNCH(k_dcb_correction, G, M, g);
  }
  DCB_LAUNCH(k_dcb_map, G, M, g);
  DCB_LAUNCH(k_dcb_color, raw, raw_c_stride, G, R, B, g);
  if (enhance) {
    DCB_LAUNCH(k_dcb_refine_pre, G, R, B, M, P1, g);
    SweepArgs rf = rect(sa, 4);
    rf.plane[0] = G;
    rf.plane[1] = P1;
    LRE_TRY(sweep<OpRefine>(c, rf, sync, nb_max, "dcb_refinement"));
    DCB_LAUNCH(k_dcb_chroma_native, R, B, G, P4, g);
    DCB_LAUNCH(k_dcb_chroma, P4, P2, P3, g);
    DCB_LAUNCH(k_dcb_chroma_g, P2, P3, G, P1, P4, g);
    SweepArgs cf = rect(sa, 6);
    cf.plane[0] = R;
    cf.plane[1] = B;
    cf.plane[2] = P1;
    cf.plane[3] = P4;
    LRE_TRY(sweep<OpColorFull>(c, cf, sync, nb_max, "dcb_color_full"));
  }
  DCB_LAUNCH(k_dcb_output, R, G, B, rgb, g);
#undef DCB_LAUNCH
  LRE_TRY(launch_border_interp(c, rgb, w, h, filters, 3));
  if (d_err) return LRE_OK;  // the caller reads the flag after its own synchronisation
  int e = 0;
  LRE_CUDA_TRY(c, cudaMemcpyAsync(&e, err, sizeof(int), cudaMemcpyDeviceToHost, s));
  LRE_CUDA_TRY(c, cudaStreamSynchronize(s));
  if (e) return fail(c, LRE_ERR_TIMEOUT, "demosaic_bayer_dcb: a sweep band timed out waiting for the band above");
  return LRE_OK;
}

}  // namespace lre
