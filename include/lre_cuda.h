/*
 * lre_cuda.h -- C ABI of the B200 (sm_100a) develop backend for libraw_enhanced.
 *
 * This is the drop-in boundary for the reference's GPU accelerator: every
 * stage entry point below replaces one method of `GPUAccelerator`
 * (core/gpu_accelerator.h:18-118 in uniuyuni/libraw_enhanced), which
 * `Accelerator` (core/accelerator.cpp) dispatches to when
 * `use_gpu_acceleration` is set.  Argument meaning and defaults follow the
 * reference method each one cites; the C++ adapter `CudaAccelerator`
 * (libraw_enhanced_b200/csrc/cuda_accelerator.h) restores the exact C++
 * signatures on top of this ABI.
 *
 * Conventions
 *   - Images use the reference layouts (core/accelerator.h:59-80):
 *       float RGB : interleaved float[H][W][3], row stride = W pixels
 *                   (ImageBufferFloat);
 *       raw uint16: uint16_t[H][W][4] (ImageBuffer);
 *       dense CFA : float[H][W] holding each site's own sample (the packed
 *                   form of the reference's sparse raw buffer).
 *   - `lre_<stage>` functions take HOST pointers and are synchronous: the
 *     result is in the host buffer on return, exactly like the reference's
 *     blocking Metal path.  Input and output may alias for every
 *     post-demosaic stage (the pipeline calls them in place).
 *   - `lre_dev_<stage>` functions take DEVICE pointers, enqueue on the
 *     context's stream and return without synchronising.
 *   - Every function returns an lre_status; on failure `lre_last_error(ctx)`
 *     holds a message.  There is no CPU fallback: a missing device or a
 *     failed launch is reported, never silently computed on the host.
 */
#ifndef LRE_CUDA_H
#define LRE_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LRE_ABI_VERSION 1

typedef enum lre_status {
  LRE_OK = 0,
  LRE_ERR_INVALID_ARGUMENT = 1, /* shape / pointer / parameter rejected     */
  LRE_ERR_CUDA = 2,             /* a CUDA runtime call or launch failed      */
  LRE_ERR_OUT_OF_MEMORY = 3,    /* device or pinned allocation failed        */
  LRE_ERR_NO_DEVICE = 4,        /* no usable sm_100 device                   */
  LRE_ERR_TIMEOUT = 5,          /* a bounded device-side wait expired        */
  LRE_ERR_INJECTED = 6,         /* host-side fault injection fired           */
  LRE_ERR_BUSY = 7              /* admission refused (device budget)         */
} lre_status;

/* X-Trans `filters` sentinel (core/accelerator.h:179). */
#define LRE_FILTERS_XTRANS 9u

typedef struct lre_ctx lre_ctx;

/* ---------------------------------------------------------------- context */
/* Create a context on `device` (GPUAccelerator::initialize,
 * core/gpu_accelerator.mm:47-105).  One context owns a stream, a growable
 * device workspace and pinned staging buffers. */
lre_status lre_create(int device, lre_ctx** out);
void lre_destroy(lre_ctx* ctx);
/* Message of the last failure on this context (never NULL). */
const char* lre_last_error(const lre_ctx* ctx);
/* GPUAccelerator::get_device_info (core/gpu_accelerator.h:25). */
lre_status lre_device_info(lre_ctx* ctx, char* buf, size_t buflen);
/* GPUAccelerator::is_available (core/gpu_accelerator.h:24). */
int lre_is_available(void);
int lre_abi_version(void);
/* Use a caller-owned cudaStream_t for all later work (NULL: own stream). */
lre_status lre_set_stream(lre_ctx* ctx, void* cuda_stream);
void* lre_get_stream(lre_ctx* ctx);
lre_status lre_synchronize(lre_ctx* ctx);
/* Pre-size the device workspace (bytes); later calls reuse it. */
lre_status lre_reserve_workspace(lre_ctx* ctx, size_t bytes);
size_t lre_workspace_bytes(const lre_ctx* ctx);
/* Number of kernels this context has launched so far. */
uint64_t lre_launch_count(const lre_ctx* ctx);
/* Page-locked host memory for fast transfers (PageAlignedAllocator,
 * core/accelerator.h:24-53, is the reference's analogue). */
lre_status lre_host_alloc(lre_ctx* ctx, size_t bytes, void** out);
lre_status lre_host_free(lre_ctx* ctx, void* p);
/* Host-side fault injection for failure-path tests: the next `countdown`-th
 * device operation on this context fails with LRE_ERR_INJECTED before any
 * work is enqueued (0 disables).  Never touches the GPU. */
void lre_inject_fault(lre_ctx* ctx, int countdown);
/* Bound of every device-side wait of the in-order sweeps (DCB, AAHD,
 * highlight recovery: a band waits for the band above to publish its
 * columns), in SM clock cycles; cycles <= 0 restores the default (~2 s).
 * A wait that runs out sets an error flag, stops waiting and lets the kernel
 * finish; the call then returns LRE_ERR_TIMEOUT and the context stays
 * usable.  No counterpart in the reference (its loops run on the CPU). */
lre_status lre_set_wait_limit(lre_ctx* ctx, long long cycles);
/* Host-side fault injection for the bounded waits: in the next in-order
 * sweep, band `band` (32 rows each, from the top) never publishes its
 * progress -- a message that is dropped -- so the band below it waits until
 * its bound runs out.  One-shot; band < 0 clears it.  No device fault. */
void lre_inject_sweep_stall(lre_ctx* ctx, int band);

/* ------------------------------------------------ stages, host buffers */
/* GPUAccelerator::demosaic_bayer_amaze (core/gpu_accelerator.h:35-39;
 * CPU semantics core/cpu_accelerator.cpp:1635-1653, AMaZE then a 4-px
 * border interpolation).  `raw_rgb` is the reference's sparse (H,W,3) raw
 * buffer: only each site's own channel is read. */
lre_status lre_demosaic_bayer_amaze(lre_ctx* ctx, const float* raw_rgb, float* rgb, size_t width,
                                    size_t height, uint32_t filters, const float cam_mul[4],
                                    float maximum_value);
/* GPUAccelerator::demosaic_xtrans_1pass / _3pass (core/gpu_accelerator.h:42-53;
 * core/cpu_accelerator.cpp:2767-2784).  `color_matrix` is accepted for
 * signature parity; the reference's YPbPr 3-pass does not use it. */
lre_status lre_demosaic_xtrans_1pass(lre_ctx* ctx, const float* raw_rgb, float* rgb, size_t width,
                                     size_t height, const char xtrans[36],
                                     const float color_matrix[12], float maximum_value);
lre_status lre_demosaic_xtrans_3pass(lre_ctx* ctx, const float* raw_rgb, float* rgb, size_t width,
                                     size_t height, const char xtrans[36],
                                     const float color_matrix[12], float maximum_value);
/* GPUAccelerator::apply_white_balance (core/gpu_accelerator.h:62-66;
 * core/cpu_accelerator.cpp:2789-2869).  Writes only each site's own
 * channel of `rgb` (G2 into channel 1); other channels are left as they are. */
lre_status lre_apply_white_balance(lre_ctx* ctx, const uint16_t* raw4, float* rgb, size_t width,
                                   size_t height, const float wb[4], uint32_t filters,
                                   const char xtrans[36]);
/* GPUAccelerator::tone_mapping (core/gpu_accelerator.h:78-80;
 * core/cpu_accelerator.cpp:3034-3068): ACES per channel times after_scale. */
lre_status lre_tone_mapping(lre_ctx* ctx, const float* in, float* out, size_t width, size_t height,
                            float after_scale);
/* GPUAccelerator::apply_detail_preserving_tonemap (core/gpu_accelerator.h:94-95;
 * CPU semantics core/libraw_wrapper.cpp:1389-1471). */
lre_status lre_detail_tonemap(lre_ctx* ctx, const float* in, float* out, size_t width,
                              size_t height);
/* GPUAccelerator::enhance_micro_contrast (core/gpu_accelerator.h:85-90;
 * core/cpu_accelerator.cpp:3130-3319).  `mask` (W*H floats) may be NULL. */
lre_status lre_enhance_micro_contrast(lre_ctx* ctx, const float* in, float* out, size_t width,
                                      size_t height, float threshold, float strength,
                                      float target_contrast, const float* mask);
/* GPUAccelerator::ca_register_lateral (core/gpu_accelerator.h:98-104;
 * core/cpu_accelerator.cpp:3496-3673). */
lre_status lre_ca_register_lateral(lre_ctx* ctx, const float* in, float* out, size_t width,
                                   size_t height, int cell_size, int max_iterations,
                                   float max_shift, float min_confidence, int pyramid_levels);
/* GPUAccelerator::ca_axial_cleanup (core/gpu_accelerator.h:107-111;
 * core/cpu_accelerator.cpp:3799-3928). */
lre_status lre_ca_axial_cleanup(lre_ctx* ctx, const float* in, float* out, size_t width,
                                size_t height, int radius, float epsilon, float strength);
/* GPUAccelerator::defringe (core/gpu_accelerator.h:114-121;
 * core/cpu_accelerator.cpp:3939-5064). */
lre_status lre_defringe(lre_ctx* ctx, const float* in, float* out, size_t width, size_t height,
                        float radius, float edge_threshold, float chroma_threshold, float strength,
                        int defringe_green, float green_strength_scale);

/* Integer pieces around the path (core/libraw_wrapper.cpp, bit-exact). */
/* apply_black_level_correction (core/libraw_wrapper.cpp:401-491), in place.
 * `cblack` has LibRaw's layout: [0..3] per channel, [4],[5] the positional
 * pattern size, [6..] the pattern; `cblack_len` entries are read. */
lre_status lre_black_level(lre_ctx* ctx, uint16_t* raw4, size_t width, size_t height,
                           const unsigned* cblack, size_t cblack_len, unsigned black,
                           unsigned maximum);
/* adjust_maximum (core/libraw_wrapper.cpp:1010-1087): scans the CFA samples
 * of a sparse raw buffer when *data_maximum == 0 and returns the adopted
 * maximum in *maximum. */
lre_status lre_adjust_maximum(lre_ctx* ctx, const float* raw_rgb, size_t width, size_t height,
                              uint32_t filters, float threshold, float* data_maximum,
                              float* maximum);
/* ProcessedImageData.to_numpy quantisation (core/python_bindings.cpp:235-257):
 * out = (uint16)(clamp(x,0,1)*65535 + 0.5) over n floats. */
lre_status lre_quantize_u16(lre_ctx* ctx, const float* in, uint16_t* out, size_t n);
lre_status lre_quantize_u8(lre_ctx* ctx, const float* in, uint8_t* out, size_t n);

/* ------------------------------------------------ stages, device buffers */
/* Same arithmetic as the host versions, on device pointers, asynchronous on
 * the context stream.  `raw` is a DENSE float CFA mosaic (H*W floats). */
lre_status lre_dev_demosaic_bayer_amaze(lre_ctx* ctx, const float* raw, float* rgb, size_t width,
                                        size_t height, uint32_t filters, const float cam_mul[4],
                                        float maximum_value);
lre_status lre_dev_demosaic_xtrans(lre_ctx* ctx, const float* raw, float* rgb, size_t width,
                                   size_t height, const char xtrans[36], float maximum_value,
                                   int passes);
lre_status lre_dev_tone_mapping(lre_ctx* ctx, const float* in, float* out, size_t width,
                                size_t height, float after_scale);
lre_status lre_dev_detail_tonemap(lre_ctx* ctx, const float* in, float* out, size_t width,
                                  size_t height);
lre_status lre_dev_enhance_micro_contrast(lre_ctx* ctx, const float* in, float* out, size_t width,
                                          size_t height, float threshold, float strength,
                                          float target_contrast, const float* mask);
lre_status lre_dev_ca_register_lateral(lre_ctx* ctx, const float* in, float* out, size_t width,
                                       size_t height, int cell_size, int max_iterations,
                                       float max_shift, float min_confidence, int pyramid_levels);
lre_status lre_dev_ca_axial_cleanup(lre_ctx* ctx, const float* in, float* out, size_t width,
                                    size_t height, int radius, float epsilon, float strength);
lre_status lre_dev_defringe(lre_ctx* ctx, const float* in, float* out, size_t width, size_t height,
                            float radius, float edge_threshold, float chroma_threshold,
                            float strength, int defringe_green, float green_strength_scale);
lre_status lre_dev_quantize_u16(lre_ctx* ctx, const float* in, uint16_t* out, size_t n);

/* Axial CA guided filter that allocates nothing.  This entry point has no
 * counterpart in the reference.  It serves callers that cannot allocate device
 * memory while they process a frame: a plug-in host that only lends
 * pre-reserved pools, a capture thread that must not block in cudaMalloc
 * (which synchronises the device), an application whose memory budget is
 * already committed.  It needs no lre_ctx.
 *
 * Arguments are those of lre_dev_ca_axial_cleanup (device pointers; `in ==
 * out` allowed), enqueued on `cuda_stream` (NULL = legacy default stream),
 * which must belong to the current device (else LRE_ERR_INVALID_ARGUMENT).
 * It runs a different kernel (one fused tile pass instead of the two-pass
 * stream), so its output matches lre_dev_ca_axial_cleanup's within the
 * float-stage tolerance (max-abs 1e-4), not bit for bit.  Its scratch (the
 * max-G normaliser and, for in-place calls, a copy of the input) is one
 * file-scope device array sized for images of at most 2,097,152 pixels
 * (1920x1080 and 2048x1024 fit); larger images, radius > 16 or null pointers
 * return LRE_ERR_INVALID_ARGUMENT before any work.  Every GPU that loads the
 * library keeps the array (about 24 MiB) until the process exits.  The first
 * call on a device looks up the array's device address; make that first call
 * before any stream capture.  All calls share the one array: the scratch is
 * re-initialised by every call, but calls that overlap on the GPU (different
 * streams, or several host threads) race on it, so serialise them.  A CUDA
 * error already pending when it is called is left in place and reported as
 * LRE_ERR_CUDA, with nothing enqueued. */
lre_status lre_dev_ca_axial_cleanup_noalloc(const float* in, float* out, size_t width, size_t height,
                                            int radius, float epsilon, float strength,
                                            void* cuda_stream);

/* ------------------------------------------------ develop pipeline */
/* Stage switches and parameters of one develop request.  Field names and
 * defaults follow ProcessingParams (core/accelerator.h:83-177); `cfa` is a
 * LibRaw filters word or LRE_FILTERS_XTRANS (then `xtrans` is read). */
typedef struct lre_develop_params {
  uint32_t filters;
  char xtrans[36];
  float cam_mul[4];
  float maximum_value;
  int xtrans_passes; /* 1 or 3 */
  int lateral_ca_correction;
  int lateral_ca_cell_size;
  int lateral_ca_max_iterations;
  float lateral_ca_max_shift;
  float lateral_ca_min_confidence;
  int lateral_ca_pyramid_levels;
  int axial_ca_correction;
  int axial_ca_radius;
  float axial_ca_epsilon;
  float axial_ca_strength;
  int defringe;
  float defringe_radius;
  float defringe_edge_threshold;
  float defringe_chroma_threshold;
  float defringe_strength;
  int defringe_green;
  float defringe_green_strength;
  int tone_mapping; /* 0 off, 1 ACES(after_scale), 2 detail-preserving */
  float tone_after_scale;
  int output_bits; /* 32: float RGB out; 16: uint16 RGB out */
  int stage_order; /* 0: reference order (lateral, axial, defringe, tone);
                      1: demosaic, defringe, axial, tone */
  int demosaic_algorithm; /* ProcessingParams::demosaic_algorithm routed as
                             Accelerator::demosaic_compute does
                             (core/accelerator.cpp:90-129): Bayer 0 bilinear,
                             4 DCB (1 iteration, enhanced), 12 AAHD, anything
                             else AMaZE; X-Trans 0 one-pass, else
                             xtrans_passes.  Default 1. */
  int highlight_recovery;    /* recover_highlights right after the demosaic, as
                                the pipeline runs it for highlight_mode > 2
                                (core/libraw_wrapper.cpp:1677-1683); default 0 */
  float highlight_threshold; /* its saturation threshold (the pipeline passes
                                maximum / data_maximum); default 1 */
} lre_develop_params;

/* Fill `p` with the reference defaults (ProcessingParams()). */
void lre_develop_params_default(lre_develop_params* p);

/* Plain per-image develop: dense float CFA mosaic (host) -> RGB (host, float
 * or uint16 per output_bits).  One upload, device-resident intermediates,
 * one download. */
lre_status lre_develop(lre_ctx* ctx, const float* mosaic, void* out, size_t width, size_t height,
                       const lre_develop_params* params);
/* Same on device buffers, asynchronous on the context stream. */
lre_status lre_dev_develop(lre_ctx* ctx, const float* mosaic, void* out, size_t width,
                           size_t height, const lre_develop_params* params);

/* GPUAccelerator::demosaic_bayer_linear (core/gpu_accelerator.h:29-32;
 * core/cpu_accelerator.cpp:74-156): bilinear interpolation of the missing
 * colours, then the 1-px border interpolation.  Sparse (H,W,3) raw in. */
lre_status lre_demosaic_bayer_linear(lre_ctx* ctx, const float* raw_rgb, float* rgb, size_t width,
                                     size_t height, uint32_t filters, float maximum_value);
/* Same on a dense device mosaic. */
lre_status lre_dev_demosaic_bayer_linear(lre_ctx* ctx, const float* raw, float* rgb, size_t width,
                                         size_t height, uint32_t filters, float maximum_value);

/* Accelerator::demosaic_bayer_dcb (core/accelerator.h:273-277, defaults
 * iterations = 1, dcb_enhance = true; the reference GPU path has no DCB and
 * falls back to the CPU, core/accelerator.cpp:180-199) and its CPU body
 * CPUAccelerator::demosaic_bayer_dcb (core/cpu_accelerator.cpp:1043-1137):
 * 8-neighbour seed, DCB_Processor::run_dcb(iterations, dcb_enhance), /max,
 * 3-px border interpolation.  Results equal the reference run with one
 * OpenMP thread (its row-parallel in-place passes are order-dependent).
 * Needs a 2x2 Bayer layout (RGGB, BGGR, GRBG, GBRG); returns
 * LRE_ERR_INVALID_ARGUMENT for other filters words.  Sparse (H,W,3) raw in. */
lre_status lre_demosaic_bayer_dcb(lre_ctx* ctx, const float* raw_rgb, float* rgb, size_t width,
                                  size_t height, uint32_t filters, float maximum_value, int iterations,
                                  int dcb_enhance);
/* Same on a dense device mosaic; returns after the stream has drained (the
 * sweeps' completion flag is read back). */
lre_status lre_dev_demosaic_bayer_dcb(lre_ctx* ctx, const float* raw, float* rgb, size_t width,
                                      size_t height, uint32_t filters, float maximum_value, int iterations,
                                      int dcb_enhance);

/* Accelerator::demosaic_bayer_aahd (core/accelerator.h:269-271; the
 * reference GPU path falls back to the CPU, core/accelerator.cpp:159-178) and
 * CPUAccelerator::demosaic_bayer_aahd (core/cpu_accelerator.cpp:617-633):
 * hot-pixel hiding, directional greens and colours, YUV homogeneity choice
 * and refinement, /max, 2-px border interpolation.  Results equal the
 * reference run with one OpenMP thread.  Needs a 2x2 Bayer layout and
 * samples in [0, 65536) (the reference indexes a 64 Ki gamma table with
 * them).  Sparse (H,W,3) raw in. */
lre_status lre_demosaic_bayer_aahd(lre_ctx* ctx, const float* raw_rgb, float* rgb, size_t width,
                                   size_t height, uint32_t filters, float maximum_value);
/* Same on a dense device mosaic; returns after the stream has drained. */
lre_status lre_dev_demosaic_bayer_aahd(lre_ctx* ctx, const float* raw, float* rgb, size_t width,
                                       size_t height, uint32_t filters, float maximum_value);

/* ------------------------------------------------ highlight recovery */
/* The develop pipeline's recover_highlights (core/libraw_wrapper.cpp:
 * 1095-1383, run for highlight_mode > 2 at :1677-1683; standalone as
 * LibRawWrapper::recover_highlights_numpy, :3066-3096): highlight R/G and
 * B/G ratios, G rebuilt in highlights, white pixels blended with their 8
 * neighbours, then the in-order LoCA green lift.  `rgb_in` and `rgb_out` are
 * (H,W,3) float and may be the same buffer.  `mask_out` (W*H floats) receives
 * the soft highlight mask when non-null; `wb_rgb` (3 floats) selects the
 * WB-undone chroma edges as the reference does; `max_val_out` (nullable)
 * receives the highlight maximum.  Bit-exact with the reference. */
lre_status lre_recover_highlights(lre_ctx* ctx, const float* rgb_in, float* rgb_out, size_t width,
                                  size_t height, float saturation_threshold, float* mask_out,
                                  const float* wb_rgb, float* max_val_out);
/* Same on device buffers (mask_out and max_val_out device pointers, wb_rgb
 * host); returns after the stream has drained. */
lre_status lre_dev_recover_highlights(lre_ctx* ctx, const float* rgb_in, float* rgb_out, size_t width,
                                      size_t height, float saturation_threshold, float* mask_out,
                                      const float* wb_rgb, float* max_val_out);

/* ------------------------------------------------------ output end */
/* GPUAccelerator::convert_color_space (core/gpu_accelerator.h:66-69;
 * core/cpu_accelerator.cpp:2874-2897): out = M[:, :3] * in + M[:, 3] with
 * the row-major 3x4 matrix `transform`. */
lre_status lre_convert_color_space(lre_ctx* ctx, const float* in, float* out, size_t width,
                                   size_t height, const float transform[12]);
/* GPUAccelerator::gamma_correct (core/gpu_accelerator.h:70-72;
 * core/cpu_accelerator.cpp:2903-2978): the output colour space's encoding
 * (1/7 sRGB, 2/3 power 2.222, 4 power 1.8, 8 Rec.2020, otherwise power
 * `gamma_power` with linear slope `gamma_slope`). */
lre_status lre_gamma_correct(lre_ctx* ctx, const float* in, float* out, size_t width, size_t height,
                             float gamma_power, float gamma_slope, int output_color_space);
lre_status lre_dev_convert_color_space(lre_ctx* ctx, const float* in, float* out, size_t width,
                                       size_t height, const float transform[12]);
lre_status lre_dev_gamma_correct(lre_ctx* ctx, const float* in, float* out, size_t width,
                                 size_t height, float gamma_power, float gamma_slope,
                                 int output_color_space);
/* The two above fused with ProcessedImageData.to_numpy's quantisation
 * (core/python_bindings.cpp:235-257): one pass from linear camera RGB to
 * 8-bit, 16-bit (or float, bits = 32) output RGB. */
lre_status lre_output_epilogue(lre_ctx* ctx, const float* in, void* out, size_t width, size_t height,
                               const float transform[12], float gamma_power, float gamma_slope,
                               int output_color_space, int bits);
lre_status lre_dev_output_epilogue(lre_ctx* ctx, const float* in, void* out, size_t width,
                                   size_t height, const float transform[12], float gamma_power,
                                   float gamma_slope, int output_color_space, int bits);

/* ------------------------------------------------------ white balance */
/* The inputs of LibRaw's white-balance multiplier derivation, as the
 * reference's scale_colors reads them (core/libraw_wrapper.cpp:602-845):
 * imgdata.params, imgdata.color and imgdata.idata fields. */
typedef struct lre_wb_inputs {
  float user_mul[4];               /* params.user_mul; user_mul[0] != 0 replaces pre_mul */
  float pre_mul[4];                /* color.pre_mul (daylight multipliers)              */
  float cam_mul[4];                /* color.cam_mul (as-shot multipliers)               */
  unsigned short white[8][8];      /* color.white                                       */
  unsigned cblack[4];              /* color.cblack[0..3]                                */
  int use_auto_wb;                 /* params.use_auto_wb                                */
  int use_camera_wb;               /* params.use_camera_wb                              */
  int camerawb_fallback_to_daylight; /* rawparams.options has
                                      LIBRAW_RAWOPTIONS_CAMERAWB_FALLBACK_TO_DAYLIGHT   */
  int as_shot_wb_applied;          /* color.as_shot_wb_applied                          */
  int colors;                      /* idata.colors                                      */
  int no_auto_scale;               /* params.no_auto_scale: multipliers all 1           */
} lre_wb_inputs;

/* What the derivation produces. */
typedef struct lre_wb_result {
  float scale_mul[4];  /* the multipliers apply_white_balance uses (effective_wb)   */
  float pre_mul[4];    /* color.pre_mul after the derivation                       */
  unsigned maximum;    /* color.maximum - color.black (scale_colors' unsigned update) */
  int auto_wb;         /* 1: the grey-world (auto-WB) branch ran                    */
  int bad_camera_wb;   /* 1: LibRaw would raise LIBRAW_WARN_BAD_CAMERA_WB           */
} lre_wb_result;

/* 1 when `in` selects the grey-world (auto-WB) branch, which needs the
 * per-channel sums of the black-subtracted image; 0 otherwise.  Replaces
 * should_use_auto_wb in core/libraw_wrapper.cpp:623-632. */
int lre_wb_needs_channel_sums(const lre_wb_inputs* in);

/* scale_colors' multiplier logic (core/libraw_wrapper.cpp:612-845: user
 * multipliers, auto-WB, camera WB from color.white, the Nikon sRAW daylight
 * case, pre_mul[1]/[3] defaults, maximum -= black, normalisation by the
 * smallest multiplier) on the host, bit-exact.  `channel_sums` /
 * `channel_counts` are the per-native-colour (0..3) sums and counts of the
 * uint16[4] image (lre_channel_sums); they are read only when
 * lre_wb_needs_channel_sums(in) is 1 and may be NULL otherwise
 * (LRE_ERR_INVALID_ARGUMENT if needed and NULL).  No device work. */
lre_status lre_wb_multipliers(const lre_wb_inputs* in, uint32_t filters, unsigned maximum, unsigned black,
                              const uint64_t channel_sums[4], const uint64_t channel_counts[4],
                              lre_wb_result* out);
/* The grey-world statistics of the auto-WB branch (core/libraw_wrapper.cpp:
 * 632-661): for each native colour c (fcol_xtrans, or fcol_bayer_native
 * 0..3), the sum of image[i][c] over the sites of colour c and their count,
 * as exact 64-bit integers (the reference's double sums of 16-bit values
 * are exact below 2^53).  `raw4` is width*height uint16[4] pixels in host
 * memory (lre_channel_sums) or device memory (lre_dev_channel_sums); both
 * return after the sums are in host memory. */
lre_status lre_channel_sums(lre_ctx* ctx, const uint16_t* raw4, size_t width, size_t height, uint32_t filters,
                            const char xtrans[36], uint64_t sums[4], uint64_t counts[4]);
lre_status lre_dev_channel_sums(lre_ctx* ctx, const uint16_t* raw4, size_t width, size_t height,
                                uint32_t filters, const char xtrans[36], uint64_t sums[4], uint64_t counts[4]);

/* ------------------------------------------------------ on-device ingest */
/* The LibRaw-side frame description the raw ingest reads (imgdata.sizes and
 * imgdata.color fields, plus the pipeline's WB and adjust_maximum inputs). */
typedef struct lre_raw_frame {
  size_t raw_width, raw_height;   /* raw_image geometry (sizes.raw_width/height)      */
  size_t raw_pitch;               /* bytes per Bayer raw_image row (sizes.raw_pitch)  */
  size_t top_margin, left_margin; /* sizes.top_margin / left_margin                   */
  size_t width, height;           /* visible frame (sizes.width / height)             */
  int shrink;                     /* 1: half-size frame (iwidth = (width + 1) / 2)     */
  uint32_t filters;               /* Bayer filters word or LRE_FILTERS_XTRANS         */
  char xtrans[36];                /* 6x6 X-Trans pattern (filters == X-Trans)          */
  unsigned cblack[6 + 36];        /* color.cblack: [0..3], [4],[5] pattern size, [6..] */
  unsigned black;                 /* color.black                                       */
  unsigned maximum;               /* color.maximum                                     */
  int green_matching;             /* 1: apply_green_matching (Bayer only)              */
  float wb[4];                    /* effective WB multipliers (scale_colors)           */
  float adjust_maximum_thr;       /* params.adjust_maximum_thr; 0: keep `maximum`       */
  float data_maximum;             /* color.data_maximum; 0: scanned on the device       */
  int derive_wb;                  /* 1: derive the WB multipliers from wb_in as the
                                     pipeline's scale_colors does (after black level and
                                     green matching; wb[] is then ignored, and adjust_maximum
                                     compares against maximum - black); 0: use wb[]       */
  lre_wb_inputs wb_in;            /* scale_colors inputs when derive_wb == 1              */
  int fuji_width;                 /* rawdata.ioparams.fuji_width; > 0 with a Bayer word:
                                     Fuji SuperCCD honeycomb raw2image                    */
  int fuji_layout;                /* unpacker_data.fuji_layout                           */
} lre_raw_frame;

/* raw2image (core/libraw_wrapper.cpp:2299-2438, copy_bayer_image standard
 * and Fuji honeycomb paths, copy_xtrans_image): the uint16 raw_image into
 * zero-initialised uint16[4] pixels (ImageBuffer), each sample in its CFA
 * channel, a Bayer colour-3 sample also in channel 1; half-size frames keep
 * the last sample of each 2x2 cell per channel, as the reference's scan
 * order does.  With frame->fuji_width > 0 and a Bayer filters word the raw
 * rows and columns are mapped onto the 45-degree SuperCCD frame
 * (:2342-2392). */
lre_status lre_raw2image(lre_ctx* ctx, const uint16_t* raw_image, const lre_raw_frame* frame,
                         uint16_t* image4);
/* apply_green_matching (core/libraw_wrapper.cpp:496-585), in place on
 * uint16[4] pixels; no-op for X-Trans. */
lre_status lre_green_matching(lre_ctx* ctx, uint16_t* raw4, size_t width, size_t height,
                              uint32_t filters, unsigned maximum);
/* process_raw_to_rgb from the decoded raw_image to the developed image
 * (core/libraw_wrapper.cpp:1477-1853 order): raw2image, black level, green
 * matching, the WB multipliers (frame->derive_wb: derived on the device and
 * host as scale_colors does; else frame->wb), white balance,
 * adjust_maximum, then the develop chain of
 * `params` (its filters/xtrans/maximum_value are taken from the frame and
 * the adopted maximum).  The frame crosses PCIe as 16-bit samples.
 * *maximum_used (may be NULL) receives the maximum handed to the demosaic. */
lre_status lre_develop_raw(lre_ctx* ctx, const uint16_t* raw_image, const lre_raw_frame* frame,
                           void* out, const lre_develop_params* params, float* maximum_used);
/* The Fuji SuperCCD rotate after demosaic (core/libraw_wrapper.cpp:1709-1750,
 * use_fuji_rotate): the demosaiced width x height image, sampled bilinearly
 * along the 45-degree grid, becomes *out_w x *out_h (wide = fuji_width' /
 * sqrt(0.5), high = (height - fuji_width') / sqrt(0.5), fuji_width' =
 * (fuji_width - 1 + shrink) >> shrink); pixels whose sample falls outside
 * stay 0.  lre_fuji_rotate_size gives the output size (0 x 0 when the
 * reference leaves the image unrotated).  `out` holds out_w * out_h * 3
 * floats; host buffers for lre_fuji_rotate, device for lre_dev_fuji_rotate. */
lre_status lre_fuji_rotate_size(int fuji_width, int shrink, size_t width, size_t height, size_t* out_w,
                                size_t* out_h);
lre_status lre_fuji_rotate(lre_ctx* ctx, const float* in, size_t width, size_t height, int fuji_width, int shrink,
                           float* out);
lre_status lre_dev_fuji_rotate(lre_ctx* ctx, const float* in, size_t width, size_t height, int fuji_width,
                               int shrink, float* out);
/* Same on device buffers; synchronises the context stream once when the
 * maximum has to be scanned. */
lre_status lre_dev_develop_raw(lre_ctx* ctx, const uint16_t* raw_image, const lre_raw_frame* frame,
                               void* out, const lre_develop_params* params, float* maximum_used);

/* ---------------------------------------------------------------- tuning */
/* Kernel-shape choices that never change results, only speed. */
typedef struct lre_tuning {
  int lanes;         /* batch/server: concurrent per-image pipelines (streams) */
  int axial_strip;   /* guided-filter strip width (columns per CTA): 128 or 64 */
  int axial_rows;    /* guided-filter output rows per CTA: 128 or 64          */
  int blur_tile;     /* defringe blur output tile edge: 32 or 64              */
} lre_tuning;
lre_status lre_set_tuning(lre_ctx* ctx, const lre_tuning* t);
lre_status lre_get_tuning(const lre_ctx* ctx, lre_tuning* t);

/* ------------------------------------------------------- batched develop */
/* Not in the reference (which develops one image per call): many images of
 * uneven sizes, CFA layouts and option sets in one call.  Images are spread
 * over `lanes` pipelines, each with its own stream and device buffers, so
 * the upload of one image and the download of another overlap the kernels
 * of a third; with use_graph the whole batch is captured once as one CUDA
 * graph and replayed while later calls repeat the same batch signature
 * (same pointers, sizes and parameters). */
typedef struct lre_image {
  const float* mosaic;        /* dense float32 CFA mosaic, width*height        */
  void* out;                  /* RGB out: float32 or uint16 per params.output_bits */
  size_t width, height;
  lre_develop_params params;  /* per image: CFA, WB, stages, output format     */
} lre_image;

typedef struct lre_batch_config {
  int device;
  int lanes;     /* 0: 3, or the autotuned value                              */
  int use_graph; /* 1: capture / replay the batch as one CUDA graph            */
  int autotune;  /* 1: time the kernel-shape choices on the first batch       */
} lre_batch_config;

typedef struct lre_batch_stats {
  double ms;             /* host wall time of the call                        */
  int graph;             /* 0 eager, 1 captured and launched, 2 replayed       */
  int lanes;
  uint64_t launches;     /* kernels enqueued by this call (a replay counts the graph's) */
  double tune_ms;        /* time spent autotuning in this call (0 after the first) */
} lre_batch_stats;

typedef struct lre_batch lre_batch;
lre_status lre_batch_create(const lre_batch_config* cfg, lre_batch** out);
void lre_batch_destroy(lre_batch* b);
const char* lre_batch_last_error(const lre_batch* b);
/* Host buffers in and out; synchronous.  Pageable buffers are page-locked
 * for the duration of the call (pass lre_host_alloc memory to avoid that);
 * a call with any pageable buffer runs without a graph. */
lre_status lre_batch_run(lre_batch* b, const lre_image* images, size_t n, lre_batch_stats* stats);
/* Device buffers in and out; synchronous. */
lre_status lre_dev_batch_run(lre_batch* b, const lre_image* images, size_t n, lre_batch_stats* stats);
lre_status lre_batch_get_tuning(const lre_batch* b, lre_tuning* t);
lre_status lre_batch_set_tuning(lre_batch* b, const lre_tuning* t);

/* ------------------------------------------------------- request server */
/* Not in the reference: a develop service with continuous batching.
 * Requests (host buffers, any size and option set) are queued on submit and
 * admitted onto a free lane as soon as one is idle and the device-memory
 * budget covers the request's buffers; mosaic, intermediates and result
 * stay on the device until the result is copied back.  Requests on
 * different lanes run concurrently on the GPU.  A request's result does not
 * depend on what else is in flight. */
typedef struct lre_server_config {
  int device;
  int lanes;                  /* concurrent requests on the device (0: 4)     */
  size_t device_budget_bytes; /* admission limit on resident buffers (0: 150 GB) */
  int decode_threads;         /* host threads running decode callbacks (0: 2) */
} lre_server_config;

typedef struct lre_request_stats {
  lre_status status;
  int lane;
  double queue_ms;  /* ready (submitted, or decoded) -> admitted              */
  double run_ms;    /* admitted -> result in host memory                      */
  double total_ms;  /* submit -> result in host memory                        */
  size_t device_bytes;
  double decode_ms; /* submit -> decode callback returned (0 without one)     */
} lre_request_stats;

typedef struct lre_server lre_server;
lre_status lre_server_create(const lre_server_config* cfg, lre_server** out);
/* Stops admitting, finishes every queued request, frees the device. */
void lre_server_destroy(lre_server* s);
const char* lre_server_last_error(const lre_server* s);
/* Queue a request; the image's buffers must stay valid until it completes.
 * Returns LRE_ERR_BUSY when the request alone exceeds the budget. */
lre_status lre_server_submit(lre_server* s, const lre_image* img, uint64_t* ticket);
/* Host-side decode overlapped with device work.  The reference decodes a
 * file with LibRaw on the CPU (load_file and unpack,
 * core/libraw_wrapper.cpp:2489-2503) before any develop stage runs; it has no
 * server, so nothing overlaps that decode.  This queues a request whose
 * mosaic is not decoded yet: one of the server's decode threads calls
 * decode(user, mosaic, width, height) to fill img->mosaic (caller-owned,
 * width * height floats, written through the callback), and the request
 * then joins the device queue.  While a decode thread works on one file,
 * the lanes develop earlier ones.  A non-LRE_OK return from decode
 * completes the request with that status.  The callback may run on any
 * decode thread, concurrently with itself for other requests. */
typedef lre_status (*lre_decode_fn)(void* user, float* mosaic, size_t width, size_t height);
lre_status lre_server_submit_decode(lre_server* s, const lre_image* img, lre_decode_fn decode, void* user,
                                    uint64_t* ticket);
/* Block until the request completes (timeout_ms < 0: no limit); LRE_ERR_TIMEOUT
 * if it has not completed in time.  The ticket is released on completion. */
lre_status lre_server_wait(lre_server* s, uint64_t ticket, double timeout_ms, lre_request_stats* stats);
/* Device bytes currently held by admitted requests, and the peak so far. */
lre_status lre_server_memory(const lre_server* s, size_t* in_use, size_t* peak);

#ifdef __cplusplus
}
#endif

#endif /* LRE_CUDA_H */
