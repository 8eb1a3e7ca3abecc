/*
 * lre_oracle.c -- TEST INFRASTRUCTURE (oracle), never part of the product.
 *
 * A plain-C restatement of the pieces of libraw_enhanced's develop path that
 * live in LibRaw-dependent files and therefore cannot be compiled from the
 * reference here (LibRaw is not vendored).  Each function states the reference
 * lines it follows.  Integer pieces are bit-exact restatements; the float
 * pieces keep the reference's operation order (build with -ffp-contract=off).
 *
 * The rest of the hot path (AMaZE, X-Trans, defringe, axial/lateral CA, ACES,
 * micro-contrast, white balance) is checked against the reference itself,
 * compiled from its sources into oracle/_ref/liblre_ref.so.  A few of those
 * are also restated here (ACES, white balance, border interpolation, CFA
 * indexing) so the restatement can be pinned against the compiled reference.
 */
#include <math.h>
#include <stddef.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* core/metal/shader_common.h:63-75 */
unsigned port_fcol_bayer_native(unsigned row, unsigned col, uint32_t filters) {
  return filters >> ((((row << 1) & 14) | (col & 1)) << 1) & 3;
}
unsigned port_fcol_bayer(unsigned row, unsigned col, uint32_t filters) {
  static const unsigned to3[4] = {0, 1, 2, 1};
  return to3[port_fcol_bayer_native(row, col, filters)];
}
unsigned port_fcol_xtrans(unsigned row, unsigned col, const char xtrans[36]) {
  return (unsigned)xtrans[((row + 6) % 6) * 6 + (col + 6) % 6];
}

/*
 * core/libraw_wrapper.cpp:401-491 (apply_black_level_correction).
 * mode 2: positional cblack[6+...] plus per-channel cblack[c];
 * mode 1: per-channel cblack[c]; mode 0: global `black`.
 * Every result is clamped to [0, maximum] and stored back as uint16.
 * The mode is chosen exactly as the reference chooses it.
 */
void port_black_level(uint16_t* img4, size_t w, size_t h, const unsigned* cblack /* >= 6 + 4096 */,
                      unsigned black, unsigned maximum) {
  size_t total = w * h;
  if (cblack[4] && cblack[5]) {
    for (size_t q = 0; q < total; q++) {
      int row = (int)(q / w), col = (int)(q % w);
      int pos_black = (int)cblack[6 + (row % cblack[4]) * cblack[5] + (col % cblack[5])];
      for (int c = 0; c < 4; c++) {
        int v = img4[q * 4 + c];
        v -= pos_black;
        v -= (int)cblack[c];
        if (v < 0) v = 0;
        if (v > (int)maximum) v = (int)maximum;
        img4[q * 4 + c] = (uint16_t)v;
      }
    }
  } else if (cblack[0] || cblack[1] || cblack[2] || cblack[3]) {
    for (size_t q = 0; q < total; q++)
      for (int c = 0; c < 4; c++) {
        int v = img4[q * 4 + c] - (int)cblack[c];
        if (v < 0) v = 0;
        if (v > (int)maximum) v = (int)maximum;
        img4[q * 4 + c] = (uint16_t)v;
      }
  } else {
    for (size_t q = 0; q < total; q++)
      for (int c = 0; c < 4; c++) {
        int v = img4[q * 4 + c] - (int)black;
        if (v < 0) v = 0;
        if (v > (int)maximum) v = (int)maximum;
        img4[q * 4 + c] = (uint16_t)v;
      }
  }
}

/* core/cpu_accelerator.cpp:2808-2869 (apply_wb_bayer / apply_wb_xtrans) */
void port_white_balance(const uint16_t* raw4, float* rgb, size_t w, size_t h, const float wb[4],
                        uint32_t filters, const char xtrans[36]) {
  for (size_t row = 0; row < h; row++)
    for (size_t col = 0; col < w; col++) {
      size_t i = row * w + col;
      unsigned c = filters == 9 ? port_fcol_xtrans((unsigned)row, (unsigned)col, xtrans)
                                : port_fcol_bayer_native((unsigned)row, (unsigned)col, filters);
      float v = (float)raw4[i * 4 + c] * wb[c];
      if (c == 3) c = 1;
      rgb[i * 3 + c] = v;
    }
}

/*
 * core/libraw_wrapper.cpp:1010-1087 (adjust_maximum).  Returns the (possibly
 * adjusted) maximum; *data_maximum is updated when it was 0 and had to be
 * scanned from the CFA samples.
 */
float port_adjust_maximum(const float* rgb, size_t w, size_t h, uint32_t filters, float threshold,
                          float* data_maximum, float maximum) {
  if (threshold < 0.00001f) return maximum;
  float thr = threshold > 0.99999f ? 0.75f : threshold;
  float real_max = *data_maximum;
  if (real_max == 0.f && rgb) {
    float m = 0.f;
    for (size_t row = 0; row < h; row++)
      for (size_t col = 0; col < w; col++) {
        float v = rgb[(row * w + col) * 3 + port_fcol_bayer((unsigned)row, (unsigned)col, filters)];
        if (v > m) m = v;
      }
    real_max = m;
    *data_maximum = m;
  }
  if (real_max > 0 && real_max < maximum && real_max > maximum * thr) return real_max;
  return maximum;
}

/* core/cpu_accelerator.cpp:3034-3068 (ACES tone map, no clamp) */
static float port_aces(float x) {
  const float a = 2.51f, b = 0.03f, c = 2.43f, d = 0.59f, e = 0.14f;
  return (x * (a * x + b)) / (x * (c * x + d) + e);
}
void port_tone_mapping(const float* in, float* out, size_t n_px, float after_scale) {
  for (size_t i = 0; i < n_px * 3; i++) out[i] = port_aces(in[i]) * after_scale;
}

/*
 * core/libraw_wrapper.cpp:45-116 (box_filter_normalized): a separable
 * sliding-window box mean with an edge-truncated window.  The running sum is
 * updated add-after-emit exactly as the reference does; the order matters.
 */
static void port_box_filter(const float* src, float* dst, float* tmp, size_t w, size_t h, int r) {
  size_t R = (size_t)r;
  for (size_t y = 0; y < h; y++) {
    const float* s = src + y * w;
    float* t = tmp + y * w;
    float sum = 0.f;
    size_t first = w - 1 < R ? w - 1 : R;
    for (size_t x = 0; x <= first; x++) sum += s[x];
    for (size_t x = 0; x < w; x++) {
      size_t left = x > R ? x - R : 0;
      size_t right = w - 1 < x + R ? w - 1 : x + R;
      t[x] = sum / (float)(right - left + 1);
      size_t rm = x >= R ? x - R : w;
      size_t add = x + R + 1;
      if (rm < w) sum -= s[rm];
      if (add < w) sum += s[add];
    }
  }
  for (size_t x = 0; x < w; x++) {
    float sum = 0.f;
    size_t first = h - 1 < R ? h - 1 : R;
    for (size_t y = 0; y <= first; y++) sum += tmp[y * w + x];
    for (size_t y = 0; y < h; y++) {
      size_t top = y > R ? y - R : 0;
      size_t bot = h - 1 < y + R ? h - 1 : y + R;
      dst[y * w + x] = sum / (float)(bot - top + 1);
      size_t rm = y >= R ? y - R : h;
      size_t add = y + R + 1;
      if (rm < h) sum -= tmp[rm * w + x];
      if (add < h) sum += tmp[add * w + x];
    }
  }
}

/*
 * core/libraw_wrapper.cpp:1389-1471 (apply_detail_preserving_tonemap),
 * in place on an interleaved (H,W,3) float image.  Returns the count of
 * pixels whose gain was applied (the reference's `mapped_pixels`).
 */
long long port_detail_tonemap(float* rgb, size_t w, size_t h) {
  size_t n = w * h;
  if (n == 0) return 0;
  const int radius = 12;
  const float eps = 0.0025f, edge0 = 0.55f, edge1 = 0.90f;
  float* guide = (float*)malloc(n * sizeof(float));
  float* mean = (float*)malloc(n * sizeof(float));
  float* work = (float*)malloc(n * sizeof(float));
  float* b = (float*)malloc(n * sizeof(float));
  float* tmp = (float*)malloc(n * sizeof(float));
  for (size_t i = 0; i < n; i++) {
    const float* p = rgb + i * 3;
    float m = p[1] > p[2] ? p[1] : p[2];
    m = p[0] > m ? p[0] : m;
    guide[i] = m > 0.0f ? m : 0.0f;
    work[i] = guide[i] * guide[i];
  }
  port_box_filter(guide, mean, tmp, w, h, radius);
  port_box_filter(work, work, tmp, w, h, radius);
  for (size_t i = 0; i < n; i++) {
    float var = work[i] - mean[i] * mean[i];
    var = var > 0.0f ? var : 0.0f;
    float a = var / (var + eps);
    work[i] = a;
    b[i] = mean[i] * (1.0f - a);
  }
  port_box_filter(work, work, tmp, w, h, radius);
  port_box_filter(b, b, tmp, w, h, radius);
  long long mapped = 0;
  for (size_t i = 0; i < n; i++) {
    float base = work[i] * guide[i] + b[i];
    base = base > 1e-6f ? base : 1e-6f;
    float gain = port_aces(base) / base;
    gain = gain < 0.0f ? 0.0f : (gain > 1.0f ? 1.0f : gain);
    float t = (base - edge0) / (edge1 - edge0);
    t = t < 0.0f ? 0.0f : (t > 1.0f ? 1.0f : t);
    t = t * t * (3.0f - 2.0f * t);
    if (t <= 0.0f) continue;
    gain = 1.0f + (gain - 1.0f) * t;
    rgb[i * 3 + 0] *= gain;
    rgb[i * 3 + 1] *= gain;
    rgb[i * 3 + 2] *= gain;
    mapped++;
  }
  free(guide);
  free(mean);
  free(work);
  free(b);
  free(tmp);
  return mapped;
}

/* core/python_bindings.cpp:235-257 (ProcessedImageData.to_numpy) */
void port_quantize_u16(const float* in, uint16_t* out, size_t n) {
  for (size_t i = 0; i < n; i++) {
    float v = in[i];
    v = v < 0.f ? 0.f : (v > 1.f ? 1.f : v);
    out[i] = (uint16_t)(v * 65535.0f + 0.5f);
  }
}
void port_quantize_u8(const float* in, uint8_t* out, size_t n) {
  for (size_t i = 0; i < n; i++) {
    float v = in[i];
    v = v < 0.f ? 0.f : (v > 1.f ? 1.f : v);
    out[i] = (uint8_t)(v * 255.0f + 0.5f);
  }
}

/*
 * core/libraw_wrapper.cpp:746-845 (scale_colors, camera-WB branch without a
 * white-point sample): scale_mul[c] = pre_mul[c] / min(pre_mul), after the
 * reference's pre_mul[1]/pre_mul[3] defaults; all ones when the minimum is
 * not positive or maximum <= 0.
 */
void port_scale_mul(const float pre_mul_in[4], int colors, float maximum, float scale_mul[4]) {
  float pre[4] = {pre_mul_in[0], pre_mul_in[1], pre_mul_in[2], pre_mul_in[3]};
  if (pre[1] == 0) pre[1] = 1;
  if (pre[3] == 0) pre[3] = colors < 4 ? pre[1] : 1;
  double dmin = 1.7976931348623157e308;
  for (int c = 0; c < 4; c++)
    if (dmin > pre[c]) dmin = pre[c];
  for (int c = 0; c < 4; c++) scale_mul[c] = (dmin > 0.00001 && maximum > 0) ? (float)(pre[c] / dmin) : 1.0f;
}

/*
 * core/libraw_wrapper.cpp:602-845 (scale_colors), the whole multiplier
 * derivation, in the reference's statement order and types:
 *   :612-618  user_mul replaces pre_mul when user_mul[0] != 0;
 *   :623-632  should_use_auto_wb;
 *   :633-664  auto-WB from the raw image (double sums of the samples,
 *             pow(., 1.0) identities, G2 folded into G);
 *   :740-772  camera WB from the 8x8 white block (unsigned sums; the
 *             white - cblack difference wraps as unsigned into an int);
 *   :774-784  Nikon sRAW daylight division;
 *   :786-792  pre_mul[1] / pre_mul[3] defaults;
 *   :800      maximum -= black (unsigned);
 *   :802-826  scale_mul = pre_mul / min(pre_mul) unless auto-WB ran;
 * plus the pipeline's no_auto_scale override (:1545-1553).
 * `raw4` (w*h uint16[4]) is read only when the auto-WB branch runs.
 * flags: bit0 use_auto_wb, bit1 use_camera_wb, bit2 camera-WB fallback to
 * daylight, bit3 as_shot_wb_applied, bit4 no_auto_scale.
 * out: scale_mul[4], pre_mul[4]; *maximum_io is updated; returns 1 when the
 * bad-camera-WB warning would be raised.
 */
int port_scale_colors(const uint16_t* raw4, size_t w, size_t h, uint32_t filters, const char xtrans[36],
                      const float user_mul[4], const float pre_mul_in[4], const float cam_mul[4],
                      const unsigned short white[64], const unsigned cblack[4], int colors, int flags,
                      unsigned* maximum_io, unsigned black, float scale_mul[4], float pre_mul_out[4]) {
  const int use_auto_wb = flags & 1, use_camera_wb = (flags >> 1) & 1, fallback = (flags >> 2) & 1;
  const int as_shot = (flags >> 3) & 1, no_auto_scale = (flags >> 4) & 1;
  float pre_mul[4];
  int warn = 0;
  memcpy(pre_mul, pre_mul_in, sizeof(pre_mul));
  if (user_mul[0]) memcpy(pre_mul, user_mul, sizeof(pre_mul));
  const int auto_wb = use_auto_wb || (use_camera_wb && (cam_mul[0] < -0.5 || (cam_mul[0] <= 0.00001f && !fallback)));
  if (auto_wb) {
    double p = 1.0;
    double norm[4] = {0.0, 0.0, 0.0, 0.0};
    double count[4] = {0.0, 0.0, 0.0, 0.0};
    for (size_t row = 0; row < h; ++row)
      for (size_t col = 0; col < w; ++col) {
        unsigned cc = filters == 9 ? port_fcol_xtrans((unsigned)row, (unsigned)col, xtrans)
                                   : port_fcol_bayer_native((unsigned)row, (unsigned)col, filters);
        norm[cc] += pow(raw4[(row * w + col) * 4 + cc], p);
        count[cc] += 1;
      }
    norm[1] += norm[3];
    count[1] += count[3];
    for (unsigned cc = 0; cc < 3; ++cc) norm[cc] = pow(norm[cc] / count[cc], 1.0 / p);
    pre_mul[0] = norm[1] / norm[0];
    pre_mul[1] = 1.0;
    pre_mul[2] = norm[1] / norm[2];
    pre_mul[3] = 1.0;
  }
  if (use_camera_wb && cam_mul[0] > 0.00001f) {
    unsigned sum[8];
    int val;
    memset(sum, 0, sizeof(sum));
    for (unsigned row = 0; row < 8; row++)
      for (unsigned col = 0; col < 8; col++) {
        unsigned c = port_fcol_bayer_native(row, col, filters);
        if ((val = white[row * 8 + col] - cblack[c]) > 0) sum[c] += val;
        sum[c + 4]++;
      }
    if (as_shot) {
      pre_mul[0] = pre_mul[1] = pre_mul[2] = pre_mul[3] = 1.0;
    } else if (sum[0] && sum[1] && sum[2] && sum[3]) {
      for (unsigned c = 0; c < 4; c++) pre_mul[c] = (float)sum[c + 4] / sum[c];
    } else if (cam_mul[0] > 0.00001f && cam_mul[2] > 0.00001f) {
      memcpy(pre_mul, cam_mul, sizeof(pre_mul));
    } else {
      warn = 1;
    }
  }
  if (as_shot && !use_camera_wb && !use_auto_wb && cam_mul[0] > 0.00001f && cam_mul[1] > 0.00001f &&
      cam_mul[2] > 0.00001f)
    for (unsigned c = 0; c < 3; c++) pre_mul[c] /= cam_mul[c];
  if (pre_mul[1] == 0) pre_mul[1] = 1;
  if (pre_mul[3] == 0) pre_mul[3] = colors < 4 ? pre_mul[1] : 1;
  *maximum_io -= black;
  if (!auto_wb) {
    double dmin = 1.7976931348623157e308;
    for (unsigned c = 0; c < 4; c++)
      if (dmin > pre_mul[c]) dmin = pre_mul[c];
    if (dmin > 0.00001 && *maximum_io > 0) {
      for (unsigned c = 0; c < 4; c++) scale_mul[c] = pre_mul[c] / dmin;
    } else {
      for (unsigned c = 0; c < 4; c++) scale_mul[c] = 1.0;
    }
  } else {
    for (unsigned c = 0; c < 4; c++) scale_mul[c] = pre_mul[c];
  }
  if (no_auto_scale)
    for (unsigned c = 0; c < 4; c++) scale_mul[c] = 1.0;
  memcpy(pre_mul_out, pre_mul, sizeof(pre_mul));
  return warn;
}

/*
 * core/libraw_wrapper.cpp:632-661 (scale_colors, auto-WB branch, p = 1):
 * per-CFA-channel means of the uint16[4] samples, G2 folded into G,
 * pre_mul = (G/R, 1, G/B, 1).  Double accumulation as in the reference.
 */
void port_auto_wb(const uint16_t* raw4, size_t w, size_t h, uint32_t filters, const char xtrans[36],
                  float pre_mul[4]) {
  double norm[4] = {0, 0, 0, 0}, count[4] = {0, 0, 0, 0};
  for (size_t row = 0; row < h; row++)
    for (size_t col = 0; col < w; col++) {
      unsigned c = filters == 9 ? port_fcol_xtrans((unsigned)row, (unsigned)col, xtrans)
                                : port_fcol_bayer_native((unsigned)row, (unsigned)col, filters);
      norm[c] += pow((double)raw4[(row * w + col) * 4 + c], 1.0);
      count[c] += 1;
    }
  norm[1] += norm[3];
  count[1] += count[3];
  for (int c = 0; c < 3; c++) norm[c] = pow(norm[c] / count[c], 1.0);
  pre_mul[0] = (float)(norm[1] / norm[0]);
  pre_mul[1] = 1.0f;
  pre_mul[2] = (float)(norm[1] / norm[2]);
  pre_mul[3] = 1.0f;
}

/*
 * core/cpu_accelerator.cpp:2984-3028 (border_interpolate): for pixels within
 * `border` of the frame, each non-native channel becomes the mean of that
 * colour's samples in the clipped 3x3 neighbourhood (G2 folded into G).
 */
void port_border_interpolate(float* rgb, size_t w, size_t h, uint32_t filters, size_t border) {
  for (size_t row = 0; row < h; row++)
    for (size_t col = 0; col < w; col++) {
      if (col >= border && col < w - border && row >= border && row < h - border) continue;
      float sum[8] = {0, 0, 0, 0, 0, 0, 0, 0};
      for (size_t y = row > 0 ? row - 1 : 0; y < row + 2 && y < h; y++)
        for (size_t x = col > 0 ? col - 1 : 0; x < col + 2 && x < w; x++) {
          unsigned f = port_fcol_bayer((unsigned)y, (unsigned)x, filters);
          sum[f] += rgb[(y * w + x) * 3 + f];
          sum[f + 4]++;
        }
      unsigned f = port_fcol_bayer((unsigned)row, (unsigned)col, filters);
      for (unsigned c = 0; c < 3; c++)
        if (c != f && sum[c + 4] > 0) rgb[(row * w + col) * 3 + c] = sum[c] / sum[c + 4];
    }
}

/*
 * core/libraw_wrapper.cpp:2299-2438 (copy_bayer_image standard path and
 * copy_xtrans_image): raw_image (uint16, raw_width x raw_height, Bayer rows
 * raw_pitch bytes apart, X-Trans rows raw_width pixels apart) into the
 * zero-initialised image4 (iwidth x iheight x 4), each sample into its CFA
 * channel; a Bayer colour-3 sample is also copied into channel 1.  With
 * shrink = 1 (half size) the four samples of a 2x2 cell land in one pixel in
 * row-major order, later samples overwriting earlier ones.
 */
void port_raw2image(const uint16_t* raw, size_t raw_width, size_t raw_height, size_t raw_pitch,
                    size_t top_margin, size_t left_margin, size_t width, size_t height, int shrink,
                    uint32_t filters, const char xtrans[36], uint16_t* image4) {
  size_t iwidth = (width + shrink) >> shrink, iheight = (height + shrink) >> shrink;
  memset(image4, 0, iwidth * iheight * 4 * sizeof(uint16_t));
  int is_xtrans = filters == 9;
  for (size_t row = 0; row < height && row < raw_height - top_margin; row++)
    for (size_t col = 0; col < width && col < raw_width - left_margin; col++) {
      size_t src_row = row + top_margin, src_col = col + left_margin;
      size_t src_idx = is_xtrans ? src_row * raw_width + src_col : src_row * (raw_pitch / 2) + src_col;
      size_t dst_row = row >> shrink, dst_col = col >> shrink;
      if (dst_row >= iheight || dst_col >= iwidth) continue;
      size_t dst = dst_row * iwidth + dst_col;
      uint16_t val = raw[src_idx];
      if (is_xtrans) {
        image4[dst * 4 + port_fcol_xtrans((unsigned)row, (unsigned)col, xtrans)] = val;
      } else {
        unsigned c = port_fcol_bayer_native((unsigned)row, (unsigned)col, filters);
        image4[dst * 4 + c] = val;
        if (c == 3) image4[dst * 4 + 1] = val;
      }
    }
}

/*
 * core/libraw_wrapper.cpp:2342-2392 (copy_bayer_image, Fuji SuperCCD
 * honeycomb branch): raw rows [0, raw_height - 2 top_margin) and columns
 * [0, fuji_width << !fuji_layout) land on the 45-degree frame at
 *   fuji_layout:  r = fuji_width - 1 - col + row / 2, c = col + (row + 1) / 2
 *   otherwise:    r = fuji_width - 1 + row - col / 2, c = row + (col + 1) / 2
 * (halves rounded down), in the sample's fcol_bayer_native(r, c) channel (a
 * colour-3 sample also in channel 1), halved by `shrink`; later samples of
 * the row-major scan overwrite earlier ones.
 */
void port_raw2image_fuji(const uint16_t* raw, size_t raw_width, size_t raw_height, size_t raw_pitch,
                         size_t top_margin, size_t left_margin, size_t width, size_t height, int shrink,
                         uint32_t filters, int fuji_width, int fuji_layout, uint16_t* image4) {
  int iwidth = (int)((width + shrink) >> shrink), iheight = (int)((height + shrink) >> shrink);
  memset(image4, 0, (size_t)iwidth * iheight * 4 * sizeof(uint16_t));
  int copy_rows = (int)raw_height - (int)top_margin * 2;
  if (copy_rows < 0) copy_rows = 0;
  const int copy_cols = fuji_width << (fuji_layout ? 0 : 1);
  for (int row = 0; row < copy_rows; row++)
    for (int col = 0; col < copy_cols; col++) {
      int r, c;
      if (fuji_layout) {
        r = fuji_width - 1 - col + (row >> 1);
        c = col + ((row + 1) >> 1);
      } else {
        r = fuji_width - 1 + row - (col >> 1);
        c = row + ((col + 1) >> 1);
      }
      const int src_row = row + (int)top_margin, src_col = col + (int)left_margin;
      if (src_row < 0 || src_row >= (int)raw_height || src_col < 0 || src_col >= (int)raw_width) continue;
      if (r < 0 || c < 0 || r >= (int)height || c >= (int)width) continue;
      const int dst_row = r >> shrink, dst_col = c >> shrink;
      if (dst_row >= iheight || dst_col >= iwidth) continue;
      const uint16_t val = raw[(size_t)src_row * (raw_pitch / 2) + src_col];
      const unsigned ch = port_fcol_bayer_native((unsigned)r, (unsigned)c, filters);
      const size_t dst = (size_t)dst_row * iwidth + dst_col;
      image4[dst * 4 + ch] = val;
      if (ch == 3) image4[dst * 4 + 1] = val;
    }
}

/*
 * core/libraw_wrapper.cpp:1709-1750 (process_raw_to_rgb, Fuji rotate):
 * fuji_width' = (fuji_width - 1 + shrink) >> shrink, step = sqrt(0.5),
 * output wide = (int)(fuji_width' / step) by high = (int)((h - fuji_width') / step)
 * (returned through *out_w / *out_h; 0 when either is <= 1, no rotation);
 * each output pixel bilinearly samples the demosaiced image at
 *   r = (float)(fuji_width' + (row - col) step), c = (float)((row + col) step)
 * and stays 0 where (int)r >= h - 1 or (int)c >= w - 1.  `out` holds
 * wide * high * 3 floats (call once with out == NULL for the size).
 */
void port_fuji_rotate(const float* rgb, size_t w, size_t h, int fuji_width_io, int shrink, float* out,
                      size_t* out_w, size_t* out_h) {
  *out_w = *out_h = 0;
  const int fuji_width = (fuji_width_io - 1 + shrink) >> shrink;
  if (fuji_width <= 0) return;
  const double step = sqrt(0.5);
  const int wide_i = (int)(fuji_width / step);
  const int high_i = (int)(((int)h - fuji_width) / step);
  if (wide_i <= 1 || high_i <= 1) return;
  *out_w = (size_t)wide_i;
  *out_h = (size_t)high_i;
  if (!out) return;
  const size_t wide = (size_t)wide_i, high = (size_t)high_i;
  memset(out, 0, wide * high * 3 * sizeof(float));
  for (size_t row = 0; row < high; ++row)
    for (size_t col = 0; col < wide; ++col) {
      const float r = (float)(fuji_width + ((double)row - (double)col) * step);
      const float c = (float)(((double)row + (double)col) * step);
      const size_t ur = (size_t)r, uc = (size_t)c;
      if (ur >= h - 1 || uc >= w - 1) continue;
      const float fr = r - (float)ur, fc = c - (float)uc;
      const float* p00 = rgb + (ur * w + uc) * 3;
      const float* p01 = rgb + (ur * w + uc + 1) * 3;
      const float* p10 = rgb + ((ur + 1) * w + uc) * 3;
      const float* p11 = rgb + ((ur + 1) * w + uc + 1) * 3;
      float* dst = out + (row * wide + col) * 3;
      for (int ch = 0; ch < 3; ++ch) {
        const float top = p00[ch] * (1.0f - fc) + p01[ch] * fc;
        const float bottom = p10[ch] * (1.0f - fc) + p11[ch] * fc;
        dst[ch] = top * (1.0f - fr) + bottom * fr;
      }
    }
}

/*
 * core/libraw_wrapper.cpp:496-585 (apply_green_matching): at the G2
 * positions of an RGGB layout (rows 3, 5, ..., columns 2, 4, ...), in flat,
 * unsaturated areas, scale channel 3 by the ratio of the surrounding G1 and
 * G2 means.  Reads a copy of the image, writes the image.  No-op for X-Trans.
 */
void port_green_matching(uint16_t* img4, size_t w, size_t h, uint32_t filters, int maximum) {
  if (filters == 9) return;
  const int margin = 3;
  const float thr = 0.01f;
  const int width = (int)w, height = (int)h;
  uint16_t* img = (uint16_t*)malloc(w * h * 4 * sizeof(uint16_t));
  if (!img) return;
  memcpy(img, img4, w * h * 4 * sizeof(uint16_t));
  for (int j = 1 + 2; j < height - margin; j += 2)
    for (int i = 0 + 2; i < width - margin; i += 2) {
      if (j - 1 < 0 || j + 1 >= height || i - 1 < 0 || i + 1 >= width || j - 2 < 0 || j + 2 >= height || i - 2 < 0 ||
          i + 2 >= width)
        continue;
      int o1_1 = img[((j - 1) * width + i - 1) * 4 + 1];
      int o1_2 = img[((j - 1) * width + i + 1) * 4 + 1];
      int o1_3 = img[((j + 1) * width + i - 1) * 4 + 1];
      int o1_4 = img[((j + 1) * width + i + 1) * 4 + 1];
      int o2_1 = img[((j - 2) * width + i) * 4 + 3];
      int o2_2 = img[((j + 2) * width + i) * 4 + 3];
      int o2_3 = img[(j * width + i - 2) * 4 + 3];
      int o2_4 = img[(j * width + i + 2) * 4 + 3];
      double m1 = (o1_1 + o1_2 + o1_3 + o1_4) / 4.0;
      double m2 = (o2_1 + o2_2 + o2_3 + o2_4) / 4.0;
      double c1 = (abs(o1_1 - o1_2) + abs(o1_1 - o1_3) + abs(o1_1 - o1_4) + abs(o1_2 - o1_3) + abs(o1_3 - o1_4) +
                   abs(o1_2 - o1_4)) / 6.0;
      double c2 = (abs(o2_1 - o2_2) + abs(o2_1 - o2_3) + abs(o2_1 - o2_4) + abs(o2_2 - o2_3) + abs(o2_3 - o2_4) +
                   abs(o2_2 - o2_4)) / 6.0;
      if ((img[(j * width + i) * 4 + 3] < maximum * 0.95) && (c1 < maximum * thr) && (c2 < maximum * thr) &&
          (m2 > 0.1)) {
        float correction = img4[(j * width + i) * 4 + 3] * m1 / m2;
        img4[(j * width + i) * 4 + 3] = correction > maximum ? (uint16_t)maximum : (uint16_t)correction;
      }
    }
  free(img);
}
