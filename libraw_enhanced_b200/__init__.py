"""B200 (sm_100a) CUDA develop backend for libraw_enhanced.

The product is ``liblre_cuda.so`` (C ABI: ``include/lre_cuda.h``).  This
package is its Python face, mirroring the reference's operator surface for the
develop hot path:

* :class:`CudaAccelerator` -- the ``GPUAccelerator`` method set
  (core/gpu_accelerator.h:18-118 of uniuyuni/libraw_enhanced) on numpy arrays
  in the reference layouts (float32 ``(H, W, 3)``, uint16 ``(H, W, 4)``), and
  ``dev_*`` variants on CUDA tensors (device pointers, asynchronous on the
  accelerator's stream).
* :func:`tone_mapping`, :func:`enhance_micro_contrast`, :func:`defringe` --
  the standalone ``RawImage`` / ``LibRawWrapper`` numpy methods
  (libraw_enhanced/high_level_api.py:465-546, core/libraw_wrapper.cpp:3098-3214)
  with their argument names, defaults and shape errors.
* :func:`develop` -- the plain per-image develop of a CFA mosaic
  (core/libraw_wrapper.cpp:1477-1853 stage order) through ``lre_develop``.
* :class:`Batch` -- many images of uneven sizes and option sets per call,
  pipelined over several streams (optionally one CUDA graph per batch) with
  autotuned kernel shapes.
* :class:`Server` -- a develop request server with continuous batching under
  a device-memory budget, reporting per-request latency.

Everything runs on the GPU; there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np

from . import _lib
from ._lib import FILTERS_XTRANS, DevelopParams, LibRawError

__all__ = [
    "CudaAccelerator",
    "LibRawError",
    "FILTERS_XTRANS",
    "FILTERS",
    "DevelopParams",
    "develop",
    "defringe",
    "tone_mapping",
    "enhance_micro_contrast",
    "default_accelerator",
    "Batch",
    "Server",
    "develop_params",
    "raw_frame",
    "wb_inputs",
    "wb_multipliers",
    "wb_needs_channel_sums",
    "fuji_rotate_size",
]

# LibRaw `filters` words of the four Bayer layouts.
FILTERS = {"RGGB": 0x94949494, "BGGR": 0x16161616, "GRBG": 0x61616161, "GBRG": 0x49494949}


def _ptr(a: np.ndarray) -> C.c_void_p:
    return C.c_void_p(a.ctypes.data)


def _rgb(image, name: str) -> np.ndarray:
    a = np.asarray(image)
    if a.ndim != 3 or a.shape[2] != 3:
        raise ValueError(f"{name}: image must be shape (H, W, 3) float32")
    return np.ascontiguousarray(a, dtype=np.float32)


def _xtrans_bytes(xtrans) -> C.Array:
    buf = (C.c_char * 36)()
    if xtrans is not None:
        x = np.asarray(xtrans, dtype=np.int8).reshape(36)
        C.memmove(buf, x.ctypes.data, 36)
    return buf


def _dptr(t) -> C.c_void_p:
    """Device pointer of a CUDA tensor (torch) or an integer address."""
    if isinstance(t, int):
        return C.c_void_p(t)
    if hasattr(t, "data_ptr"):
        if not t.is_cuda or not t.is_contiguous():
            raise ValueError("device buffers must be contiguous CUDA tensors")
        return C.c_void_p(t.data_ptr())
    raise TypeError("expected a CUDA tensor or a device address")


class CudaAccelerator:
    """The GPUAccelerator method set on one CUDA device.

    Host methods take numpy arrays and are synchronous (result on return);
    ``dev_*`` methods take CUDA tensors and enqueue on :attr:`stream`.
    """

    def __init__(self, device: int = 0):
        self._lib = _lib.load()
        h = C.c_void_p()
        st = self._lib.lre_create(int(device), C.byref(h))
        if st != _lib.LRE_OK:
            raise LibRawError(st, f"lre_create(device={device}) failed (no usable sm_100 device?)")
        self._h = h
        self.device = int(device)

    # ------------------------------------------------------------ plumbing
    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.lre_destroy(self._h)
            self._h = None

    def __del__(self):  # pragma: no cover - interpreter shutdown order
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, st: int) -> None:
        if st != _lib.LRE_OK:
            msg = self._lib.lre_last_error(self._h)
            raise LibRawError(st, msg.decode() if msg else "")

    def is_available(self) -> bool:
        return bool(self._lib.lre_is_available())

    def get_device_info(self) -> str:
        buf = C.create_string_buffer(256)
        self._check(self._lib.lre_device_info(self._h, buf, 256))
        return buf.value.decode()

    @property
    def stream(self) -> int:
        return int(self._lib.lre_get_stream(self._h) or 0)

    def set_stream(self, cuda_stream: Optional[int]) -> None:
        """Run later work on a caller-owned cudaStream_t (None: own stream)."""
        self._check(self._lib.lre_set_stream(self._h, C.c_void_p(cuda_stream or 0)))

    def synchronize(self) -> None:
        self._check(self._lib.lre_synchronize(self._h))

    def reserve_workspace(self, nbytes: int) -> None:
        self._check(self._lib.lre_reserve_workspace(self._h, int(nbytes)))

    @property
    def launch_count(self) -> int:
        return int(self._lib.lre_launch_count(self._h))

    def inject_fault(self, countdown: int) -> None:
        """Host-side fault injection: the countdown-th next call fails."""
        self._lib.lre_inject_fault(self._h, int(countdown))

    def set_wait_limit(self, cycles: int = 0) -> None:
        """Bound of the in-order sweeps' device-side waits in SM cycles (0: default ~2 s)."""
        self._check(self._lib.lre_set_wait_limit(self._h, int(cycles)))

    def inject_sweep_stall(self, band: int) -> None:
        """Fault injection: in the next in-order sweep, `band` never reports progress."""
        self._lib.lre_inject_sweep_stall(self._h, int(band))

    # ------------------------------------------------------------ stages (host)
    def demosaic_bayer_amaze(self, raw_rgb, filters: int, cam_mul=(1.0, 1.0, 1.0, 1.0), maximum_value: float = 1.0):
        """AMaZE + 4-px border fill of the reference's sparse (H, W, 3) raw buffer."""
        raw = _rgb(raw_rgb, "demosaic_bayer_amaze")
        out = np.empty_like(raw)
        cm = np.asarray(cam_mul, dtype=np.float32)
        self._check(
            self._lib.lre_demosaic_bayer_amaze(
                self._h, _ptr(raw), _ptr(out), raw.shape[1], raw.shape[0], int(filters), _ptr(cm), float(maximum_value)
            )
        )
        return out

    def demosaic_bayer_linear(self, raw_rgb, filters: int, maximum_value: float = 1.0):
        raw = _rgb(raw_rgb, "demosaic_bayer_linear")
        out = np.empty_like(raw)
        self._check(self._lib.lre_demosaic_bayer_linear(self._h, _ptr(raw), _ptr(out), raw.shape[1], raw.shape[0],
                                                        int(filters), float(maximum_value)))
        return out

    def demosaic_bayer_dcb(self, raw_rgb, filters: int, maximum_value: float = 1.0, iterations: int = 1,
                           dcb_enhance: bool = True):
        """DCB demosaic (Accelerator::demosaic_bayer_dcb, core/accelerator.h:273-277)."""
        raw = _rgb(raw_rgb, "demosaic_bayer_dcb")
        out = np.empty_like(raw)
        self._check(self._lib.lre_demosaic_bayer_dcb(self._h, _ptr(raw), _ptr(out), raw.shape[1], raw.shape[0],
                                                     int(filters), float(maximum_value), int(iterations),
                                                     int(bool(dcb_enhance))))
        return out

    def demosaic_bayer_aahd(self, raw_rgb, filters: int, maximum_value: float = 1.0):
        """AAHD demosaic (Accelerator::demosaic_bayer_aahd, core/accelerator.h:269-271)."""
        raw = _rgb(raw_rgb, "demosaic_bayer_aahd")
        out = np.empty_like(raw)
        self._check(self._lib.lre_demosaic_bayer_aahd(self._h, _ptr(raw), _ptr(out), raw.shape[1], raw.shape[0],
                                                      int(filters), float(maximum_value)))
        return out

    def recover_highlights(self, rgb, saturation_threshold: float, want_mask: bool = False, wb_rgb=None):
        """The pipeline's highlight recovery (core/libraw_wrapper.cpp:1095-1383).

        Returns (recovered copy, mask or None, highlight max)."""
        img = _rgb(rgb, "recover_highlights")
        out = np.empty_like(img)
        h, w = img.shape[:2]
        mask = np.empty((h, w), np.float32) if want_mask else None
        wb = None if wb_rgb is None else np.ascontiguousarray(wb_rgb, dtype=np.float32)
        mx = C.c_float(0.0)
        self._check(self._lib.lre_recover_highlights(self._h, _ptr(img), _ptr(out), w, h, float(saturation_threshold),
                                                     None if mask is None else _ptr(mask),
                                                     None if wb is None else _ptr(wb), C.byref(mx)))
        return out, mask, mx.value

    def demosaic_xtrans_1pass(self, raw_rgb, xtrans, color_matrix=None, maximum_value: float = 1.0):
        return self._xtrans(raw_rgb, xtrans, color_matrix, maximum_value, 1)

    def demosaic_xtrans_3pass(self, raw_rgb, xtrans, color_matrix=None, maximum_value: float = 1.0):
        return self._xtrans(raw_rgb, xtrans, color_matrix, maximum_value, 3)

    def _xtrans(self, raw_rgb, xtrans, color_matrix, maximum_value, passes):
        raw = _rgb(raw_rgb, "demosaic_xtrans")
        out = np.empty_like(raw)
        cm = np.zeros(12, np.float32) if color_matrix is None else np.asarray(color_matrix, np.float32).reshape(12)
        xt = _xtrans_bytes(xtrans)
        fn = self._lib.lre_demosaic_xtrans_1pass if passes == 1 else self._lib.lre_demosaic_xtrans_3pass
        self._check(fn(self._h, _ptr(raw), _ptr(out), raw.shape[1], raw.shape[0], xt, _ptr(cm), float(maximum_value)))
        return out

    def apply_white_balance(self, raw4, wb, filters: int, xtrans=None, out=None):
        r = np.asarray(raw4)
        if r.ndim != 3 or r.shape[2] != 4:
            raise ValueError("apply_white_balance: raw buffer must be shape (H, W, 4) uint16")
        r = np.ascontiguousarray(r, dtype=np.uint16)
        h, w, _ = r.shape
        o = np.zeros((h, w, 3), np.float32) if out is None else np.ascontiguousarray(out, np.float32)
        wbv = np.asarray(wb, dtype=np.float32)
        xt = _xtrans_bytes(xtrans)
        self._check(self._lib.lre_apply_white_balance(self._h, _ptr(r), _ptr(o), w, h, _ptr(wbv), int(filters), xt))
        return o

    def tone_mapping(self, image, after_scale: float = 1.0):
        a = _rgb(image, "tone_mapping")
        out = np.empty_like(a)
        self._check(self._lib.lre_tone_mapping(self._h, _ptr(a), _ptr(out), a.shape[1], a.shape[0], float(after_scale)))
        return out

    def apply_detail_preserving_tonemap(self, image):
        a = _rgb(image, "apply_detail_preserving_tonemap")
        out = np.empty_like(a)
        self._check(self._lib.lre_detail_tonemap(self._h, _ptr(a), _ptr(out), a.shape[1], a.shape[0]))
        return out

    def enhance_micro_contrast(self, image, threshold: float, strength: float = 8.0, target_contrast: float = 0.06, mask=None):
        a = _rgb(image, "enhance_micro_contrast")
        out = np.empty_like(a)
        mp = None
        if mask is not None:
            mask = np.ascontiguousarray(mask, dtype=np.float32)
            if mask.size != a.shape[0] * a.shape[1]:
                raise ValueError("enhance_micro_contrast: mask must hold H*W floats")
            mp = _ptr(mask)
        self._check(
            self._lib.lre_enhance_micro_contrast(
                self._h, _ptr(a), _ptr(out), a.shape[1], a.shape[0], float(threshold), float(strength), float(target_contrast), mp
            )
        )
        return out

    def ca_register_lateral(self, image, cell_size=96, max_iterations=3, max_shift=6.0, min_confidence=0.02, pyramid_levels=3):
        a = _rgb(image, "ca_register_lateral")
        out = np.empty_like(a)
        self._check(
            self._lib.lre_ca_register_lateral(
                self._h, _ptr(a), _ptr(out), a.shape[1], a.shape[0], int(cell_size), int(max_iterations),
                float(max_shift), float(min_confidence), int(pyramid_levels),
            )
        )
        return out

    def ca_axial_cleanup(self, image, radius=6, epsilon=1e-4, strength=0.3):
        a = _rgb(image, "ca_axial_cleanup")
        out = np.empty_like(a)
        self._check(
            self._lib.lre_ca_axial_cleanup(self._h, _ptr(a), _ptr(out), a.shape[1], a.shape[0], int(radius), float(epsilon), float(strength))
        )
        return out

    def defringe(self, image, radius=10.0, edge_threshold=0.1, chroma_threshold=0.15, strength=10.0,
                 defringe_green=False, green_strength_scale=0.3):
        a = _rgb(image, "defringe")
        out = np.empty_like(a)
        self._check(
            self._lib.lre_defringe(
                self._h, _ptr(a), _ptr(out), a.shape[1], a.shape[0], float(radius), float(edge_threshold),
                float(chroma_threshold), float(strength), int(bool(defringe_green)), float(green_strength_scale),
            )
        )
        return out

    def black_level(self, raw4, cblack, black: int, maximum: int):
        r = np.ascontiguousarray(raw4, dtype=np.uint16).copy()
        cb = np.asarray(list(cblack) + [0] * max(0, 6 - len(cblack)), dtype=np.uint32)
        self._check(self._lib.lre_black_level(self._h, _ptr(r), r.shape[1], r.shape[0], _ptr(cb), cb.size, int(black), int(maximum)))
        return r

    def adjust_maximum(self, raw_rgb, filters: int, threshold: float, data_maximum: float, maximum: float):
        a = _rgb(raw_rgb, "adjust_maximum")
        dm = C.c_float(float(data_maximum))
        mx = C.c_float(float(maximum))
        self._check(self._lib.lre_adjust_maximum(self._h, _ptr(a), a.shape[1], a.shape[0], int(filters), float(threshold), C.byref(dm), C.byref(mx)))
        return float(mx.value), float(dm.value)

    def quantize(self, image, bits: int = 16):
        a = np.ascontiguousarray(image, dtype=np.float32)
        if bits == 16:
            out = np.empty(a.shape, np.uint16)
            self._check(self._lib.lre_quantize_u16(self._h, _ptr(a), _ptr(out), a.size))
        elif bits == 8:
            out = np.empty(a.shape, np.uint8)
            self._check(self._lib.lre_quantize_u8(self._h, _ptr(a), _ptr(out), a.size))
        else:
            raise ValueError("bits must be 8 or 16")
        return out

    # ------------------------------------------------------------ develop
    def develop(self, mosaic, params: DevelopParams, out=None):
        m = np.ascontiguousarray(mosaic, dtype=np.float32)
        if m.ndim != 2:
            raise ValueError("develop: mosaic must be a dense (H, W) float32 CFA image")
        h, w = m.shape
        if out is None:
            out = np.empty((h, w, 3), np.float32 if params.output_bits == 32 else np.uint16)
        self._check(self._lib.lre_develop(self._h, _ptr(m), _ptr(out), w, h, C.byref(params)))
        return out

    # ------------------------------------------------------------ device variants
    def dev_demosaic_bayer_amaze(self, raw, rgb, width, height, filters, cam_mul, maximum_value=1.0):
        cm = np.asarray(cam_mul, dtype=np.float32)
        self._check(self._lib.lre_dev_demosaic_bayer_amaze(self._h, _dptr(raw), _dptr(rgb), int(width), int(height), int(filters), _ptr(cm), float(maximum_value)))

    def dev_demosaic_bayer_linear(self, raw, rgb, width, height, filters, maximum_value=1.0):
        self._check(self._lib.lre_dev_demosaic_bayer_linear(self._h, _dptr(raw), _dptr(rgb), int(width), int(height),
                                                            int(filters), float(maximum_value)))

    def dev_demosaic_bayer_dcb(self, raw, rgb, width, height, filters, maximum_value=1.0, iterations=1,
                               dcb_enhance=True):
        self._check(self._lib.lre_dev_demosaic_bayer_dcb(self._h, _dptr(raw), _dptr(rgb), int(width), int(height),
                                                         int(filters), float(maximum_value), int(iterations),
                                                         int(bool(dcb_enhance))))

    def dev_recover_highlights(self, inp, out, width, height, saturation_threshold, mask=None, wb_rgb=None,
                               max_val=None):
        wb = None if wb_rgb is None else np.ascontiguousarray(wb_rgb, dtype=np.float32)
        self._check(self._lib.lre_dev_recover_highlights(self._h, _dptr(inp), _dptr(out), int(width), int(height),
                                                         float(saturation_threshold),
                                                         None if mask is None else _dptr(mask),
                                                         None if wb is None else _ptr(wb),
                                                         None if max_val is None else _dptr(max_val)))

    def dev_demosaic_bayer_aahd(self, raw, rgb, width, height, filters, maximum_value=1.0):
        self._check(self._lib.lre_dev_demosaic_bayer_aahd(self._h, _dptr(raw), _dptr(rgb), int(width), int(height),
                                                          int(filters), float(maximum_value)))

    def dev_demosaic_xtrans(self, raw, rgb, width, height, xtrans, maximum_value=1.0, passes=3):
        self._check(self._lib.lre_dev_demosaic_xtrans(self._h, _dptr(raw), _dptr(rgb), int(width), int(height), _xtrans_bytes(xtrans), float(maximum_value), int(passes)))

    def dev_tone_mapping(self, inp, out, width, height, after_scale=1.0):
        self._check(self._lib.lre_dev_tone_mapping(self._h, _dptr(inp), _dptr(out), int(width), int(height), float(after_scale)))

    def dev_detail_tonemap(self, inp, out, width, height):
        self._check(self._lib.lre_dev_detail_tonemap(self._h, _dptr(inp), _dptr(out), int(width), int(height)))

    def dev_enhance_micro_contrast(self, inp, out, width, height, threshold, strength=8.0, target_contrast=0.06, mask=None):
        mp = None if mask is None else _dptr(mask)
        self._check(self._lib.lre_dev_enhance_micro_contrast(self._h, _dptr(inp), _dptr(out), int(width), int(height), float(threshold), float(strength), float(target_contrast), mp))

    def dev_ca_register_lateral(self, inp, out, width, height, cell_size=96, max_iterations=3, max_shift=6.0, min_confidence=0.02, pyramid_levels=3):
        self._check(self._lib.lre_dev_ca_register_lateral(self._h, _dptr(inp), _dptr(out), int(width), int(height), int(cell_size), int(max_iterations), float(max_shift), float(min_confidence), int(pyramid_levels)))

    def dev_ca_axial_cleanup(self, inp, out, width, height, radius=6, epsilon=1e-4, strength=0.3):
        self._check(self._lib.lre_dev_ca_axial_cleanup(self._h, _dptr(inp), _dptr(out), int(width), int(height), int(radius), float(epsilon), float(strength)))

    def dev_defringe(self, inp, out, width, height, radius=10.0, edge_threshold=0.1, chroma_threshold=0.15, strength=10.0, defringe_green=False, green_strength_scale=0.3):
        self._check(self._lib.lre_dev_defringe(self._h, _dptr(inp), _dptr(out), int(width), int(height), float(radius), float(edge_threshold), float(chroma_threshold), float(strength), int(bool(defringe_green)), float(green_strength_scale)))

    def dev_develop(self, mosaic, out, width, height, params: DevelopParams):
        self._check(self._lib.lre_dev_develop(self._h, _dptr(mosaic), _dptr(out), int(width), int(height), C.byref(params)))

    # ------------------------------------------------------------ output end
    def convert_color_space(self, image, transform):
        """GPUAccelerator.convert_color_space: 3x4 row-major matrix."""
        img = _rgb(image, "convert_color_space")
        t = np.ascontiguousarray(transform, dtype=np.float32).reshape(12)
        out = np.empty_like(img)
        self._check(self._lib.lre_convert_color_space(self._h, _ptr(img), _ptr(out), img.shape[1], img.shape[0], _ptr(t)))
        return out

    def gamma_correct(self, image, gamma_power=0.0, gamma_slope=0.0, output_color_space=1):
        img = _rgb(image, "gamma_correct")
        out = np.empty_like(img)
        self._check(self._lib.lre_gamma_correct(self._h, _ptr(img), _ptr(out), img.shape[1], img.shape[0],
                                                float(gamma_power), float(gamma_slope), int(output_color_space)))
        return out

    def output_epilogue(self, image, transform, gamma_power=0.0, gamma_slope=0.0, output_color_space=1, bits=16):
        """Colour space + gamma + to_numpy quantisation in one pass."""
        img = _rgb(image, "output_epilogue")
        t = np.ascontiguousarray(transform, dtype=np.float32).reshape(12)
        dt = {8: np.uint8, 16: np.uint16, 32: np.float32}[int(bits)]
        out = np.empty(img.shape, dt)
        self._check(self._lib.lre_output_epilogue(self._h, _ptr(img), _ptr(out), img.shape[1], img.shape[0], _ptr(t),
                                                  float(gamma_power), float(gamma_slope), int(output_color_space),
                                                  int(bits)))
        return out

    # ------------------------------------------------------------ raw ingest
    def raw2image(self, raw_image, frame):
        """raw_image: (raw_height, raw_pitch // 2) uint16 (X-Trans: raw_width)."""
        r = np.ascontiguousarray(raw_image, dtype=np.uint16)
        s = 1 if frame.shrink else 0
        out = np.zeros(((frame.height + s) >> s, (frame.width + s) >> s, 4), np.uint16)
        self._check(self._lib.lre_raw2image(self._h, _ptr(r), C.byref(frame), _ptr(out)))
        return out

    def channel_sums(self, raw4, filters: int, xtrans=None):
        """Per-native-colour sums and counts of a uint16 (H, W, 4) image
        (the auto-WB statistics of scale_colors), reduced on the device."""
        a = np.ascontiguousarray(raw4, dtype=np.uint16)
        sums = np.zeros(4, np.uint64)
        counts = np.zeros(4, np.uint64)
        self._check(self._lib.lre_channel_sums(self._h, _ptr(a), a.shape[1], a.shape[0], int(filters),
                                               _xtrans_bytes(xtrans), _ptr(sums), _ptr(counts)))
        return sums, counts

    def scale_colors(self, raw4, filters: int, inputs, maximum: int, black: int, xtrans=None) -> dict:
        """scale_colors' multipliers for a black-subtracted uint16 (H, W, 4)
        image: the channel sums on the device when auto-WB needs them, then
        :func:`wb_multipliers`."""
        if wb_needs_channel_sums(inputs) and not inputs.no_auto_scale:
            sums, counts = self.channel_sums(raw4, filters, xtrans)
            return wb_multipliers(inputs, filters, maximum, black, sums, counts)
        return wb_multipliers(inputs, filters, maximum, black)

    def fuji_rotate(self, image, fuji_width: int, shrink: int = 0):
        """The 45-degree Fuji SuperCCD rotate after demosaic
        (core/libraw_wrapper.cpp:1709-1750)."""
        img = _rgb(image, "fuji_rotate")
        h, w = img.shape[:2]
        size = fuji_rotate_size(fuji_width, shrink, w, h)
        if size is None:
            raise ValueError("fuji_rotate: the reference leaves this image unrotated")
        out = np.empty((size[1], size[0], 3), np.float32)
        self._check(self._lib.lre_fuji_rotate(self._h, _ptr(img), w, h, int(fuji_width), int(shrink), _ptr(out)))
        return out

    def green_matching(self, raw4, filters: int, maximum: int):
        a = np.ascontiguousarray(raw4, dtype=np.uint16).copy()
        self._check(self._lib.lre_green_matching(self._h, _ptr(a), a.shape[1], a.shape[0], int(filters), int(maximum)))
        return a

    def develop_raw(self, raw_image, frame, params: DevelopParams, out=None):
        """process_raw_to_rgb from the 16-bit raw_image: returns (rgb, maximum_used)."""
        r = np.ascontiguousarray(raw_image, dtype=np.uint16)
        s = 1 if frame.shrink else 0
        h, w = (frame.height + s) >> s, (frame.width + s) >> s
        if out is None:
            out = np.empty((h, w, 3), np.float32 if params.output_bits == 32 else np.uint16)
        m = C.c_float()
        self._check(self._lib.lre_develop_raw(self._h, _ptr(r), C.byref(frame), _ptr(out), C.byref(params), C.byref(m)))
        return out, m.value

    # ------------------------------------------------------------ tuning
    def set_tuning(self, axial_strip=128, axial_rows=128, blur_tile=64) -> None:
        t = _lib.Tuning(1, int(axial_strip), int(axial_rows), int(blur_tile))
        self._check(self._lib.lre_set_tuning(self._h, C.byref(t)))

    def get_tuning(self) -> dict:
        t = _lib.Tuning()
        self._check(self._lib.lre_get_tuning(self._h, C.byref(t)))
        return {"axial_strip": t.axial_strip, "axial_rows": t.axial_rows, "blur_tile": t.blur_tile}


def _out_for(h, w, params):
    return np.empty((h, w, 3), np.float32 if params.output_bits == 32 else np.uint16)


class Batch:
    """Develop many images per call (``lre_batch_run``).

    ``lanes`` concurrent per-image pipelines (0: autotuned or 3), ``use_graph``
    captures the batch as one CUDA graph (replayed while the batch repeats),
    ``autotune`` times the kernel-shape choices on the first batch.
    """

    def __init__(self, device: int = 0, lanes: int = 0, use_graph: bool = True, autotune: bool = True):
        self._lib = _lib.load()
        cfg = _lib.BatchConfig(int(device), int(lanes), int(bool(use_graph)), int(bool(autotune)))
        h = C.c_void_p()
        st = self._lib.lre_batch_create(C.byref(cfg), C.byref(h))
        if st != _lib.LRE_OK:
            raise LibRawError(st, "lre_batch_create failed")
        self._h = h
        self.last_stats = None

    def close(self):
        if getattr(self, "_h", None):
            self._lib.lre_batch_destroy(self._h)
            self._h = None

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st):
        if st != _lib.LRE_OK:
            msg = self._lib.lre_batch_last_error(self._h)
            raise LibRawError(st, msg.decode() if msg else "")

    @staticmethod
    def _images(items, dev):
        arr = (_lib.Image * len(items))()
        for i, (m, o, w, h, p) in enumerate(items):
            arr[i].mosaic = (_dptr(m) if dev else _ptr(m)).value
            arr[i].out = (_dptr(o) if dev else _ptr(o)).value
            arr[i].width, arr[i].height = int(w), int(h)
            arr[i].params = p
        return arr

    def run(self, mosaics, params, outs=None):
        """Host numpy mosaics (H, W) float32 -> list of RGB outputs.

        ``params`` is one DevelopParams or a list (one per image)."""
        ps = params if isinstance(params, (list, tuple)) else [params] * len(mosaics)
        ms = [np.ascontiguousarray(m, dtype=np.float32) for m in mosaics]
        if outs is None:
            outs = [_out_for(m.shape[0], m.shape[1], p) for m, p in zip(ms, ps)]
        items = [(m, o, m.shape[1], m.shape[0], p) for m, o, p in zip(ms, outs, ps)]
        arr = self._images(items, False)
        stats = _lib.BatchStats()
        self._check(self._lib.lre_batch_run(self._h, arr, len(items), C.byref(stats)))
        self.last_stats = stats
        return outs

    def dev_run(self, mosaics, outs, params):
        """CUDA tensors in and out (synchronous)."""
        ps = params if isinstance(params, (list, tuple)) else [params] * len(mosaics)
        items = [(m, o, m.shape[1], m.shape[0], p) for m, o, p in zip(mosaics, outs, ps)]
        arr = self._images(items, True)
        stats = _lib.BatchStats()
        self._check(self._lib.lre_dev_batch_run(self._h, arr, len(items), C.byref(stats)))
        self.last_stats = stats
        return outs

    def get_tuning(self) -> dict:
        t = _lib.Tuning()
        self._check(self._lib.lre_batch_get_tuning(self._h, C.byref(t)))
        return {"lanes": t.lanes, "axial_strip": t.axial_strip, "axial_rows": t.axial_rows, "blur_tile": t.blur_tile}

    def set_tuning(self, lanes=3, axial_strip=128, axial_rows=128, blur_tile=64) -> None:
        t = _lib.Tuning(int(lanes), int(axial_strip), int(axial_rows), int(blur_tile))
        self._check(self._lib.lre_batch_set_tuning(self._h, C.byref(t)))


class Server:
    """Develop request server (``lre_server_*``): continuous batching under a
    device-memory budget.  ``submit`` queues a request and returns a ticket;
    ``wait`` returns the result and its latency record."""

    def __init__(self, device: int = 0, lanes: int = 4, budget_bytes: int = 150 * 10**9, decode_threads: int = 2):
        self._lib = _lib.load()
        cfg = _lib.ServerConfig(int(device), int(lanes), int(budget_bytes), int(decode_threads))
        h = C.c_void_p()
        st = self._lib.lre_server_create(C.byref(cfg), C.byref(h))
        if st != _lib.LRE_OK:
            raise LibRawError(st, "lre_server_create failed")
        self._h = h
        self._live = {}

    def close(self):
        if getattr(self, "_h", None):
            self._lib.lre_server_destroy(self._h)
            self._h = None
            self._live.clear()

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st):
        if st != _lib.LRE_OK:
            msg = self._lib.lre_server_last_error(self._h)
            raise LibRawError(st, msg.decode() if msg else "")

    def submit(self, mosaic, params: DevelopParams, out=None) -> int:
        m = np.ascontiguousarray(mosaic, dtype=np.float32)
        if m.ndim != 2:
            raise ValueError("submit: mosaic must be a dense (H, W) float32 CFA image")
        h, w = m.shape
        if out is None:
            out = _out_for(h, w, params)
        img = _lib.Image(m.ctypes.data, out.ctypes.data, w, h, params)
        t = C.c_uint64()
        self._check(self._lib.lre_server_submit(self._h, C.byref(img), C.byref(t)))
        self._live[t.value] = (m, out)
        return t.value

    def submit_decode(self, shape, params: DevelopParams, decode, out=None) -> int:
        """Queue a request whose mosaic is produced on the host first, the way
        the reference runs LibRaw's ``unpack`` before developing.
        ``decode(mosaic)`` receives a writable (H, W) float32 array and fills
        it; it runs on one of the server's decode threads while the device
        develops earlier requests.  An exception in ``decode`` fails the
        request and is raised again by ``wait``."""
        h, w = (int(shape[0]), int(shape[1]))
        m = np.empty((h, w), dtype=np.float32)
        if out is None:
            out = _out_for(h, w, params)
        errors = []

        def _run(user, ptr, width, height):
            try:
                decode(np.ctypeslib.as_array(ptr, shape=(int(height), int(width))))
                return _lib.LRE_OK
            except Exception as e:  # reported by wait()
                errors.append(e)
                return 1  # LRE_ERR_INVALID_ARGUMENT

        cb = _lib.DECODE_FN(_run)
        img = _lib.Image(m.ctypes.data, out.ctypes.data, w, h, params)
        t = C.c_uint64()
        self._check(self._lib.lre_server_submit_decode(self._h, C.byref(img), cb, None, C.byref(t)))
        self._live[t.value] = (m, out, cb, errors)
        return t.value

    def wait(self, ticket: int, timeout_ms: float = -1.0):
        st = _lib.RequestStats()
        r = self._lib.lre_server_wait(self._h, int(ticket), float(timeout_ms), C.byref(st))
        if r == 5:  # LRE_ERR_TIMEOUT: still running
            raise TimeoutError(f"request {ticket} not complete after {timeout_ms} ms")
        live = self._live.pop(int(ticket), (None, None))
        out = live[1]
        if len(live) > 2 and live[3]:
            raise live[3][0]
        self._check(r)
        return out, {"queue_ms": st.queue_ms, "run_ms": st.run_ms, "total_ms": st.total_ms, "lane": st.lane,
                     "device_bytes": st.device_bytes, "decode_ms": st.decode_ms}

    def memory(self):
        a, b = C.c_size_t(), C.c_size_t()
        self._check(self._lib.lre_server_memory(self._h, C.byref(a), C.byref(b)))
        return a.value, b.value


def wb_inputs(user_mul=(0.0, 0.0, 0.0, 0.0), pre_mul=(1.0, 1.0, 1.0, 1.0), cam_mul=(0.0, 0.0, 0.0, 0.0),
              white=None, cblack=(0, 0, 0, 0), use_auto_wb=False, use_camera_wb=False,
              camerawb_fallback_to_daylight=False, as_shot_wb_applied=False, colors=3,
              no_auto_scale=False) -> "_lib.WbInputs":
    """The imgdata fields LibRaw's scale_colors reads to choose the WB
    multipliers (core/libraw_wrapper.cpp:602-845)."""
    w = _lib.WbInputs()
    for i in range(4):
        w.user_mul[i] = float(user_mul[i])
        w.pre_mul[i] = float(pre_mul[i])
        w.cam_mul[i] = float(cam_mul[i])
        w.cblack[i] = int(cblack[i])
    if white is not None:
        wh = np.asarray(white, dtype=np.uint16).reshape(8, 8)
        for r in range(8):
            for c in range(8):
                w.white[r][c] = int(wh[r, c])
    w.use_auto_wb, w.use_camera_wb = int(bool(use_auto_wb)), int(bool(use_camera_wb))
    w.camerawb_fallback_to_daylight = int(bool(camerawb_fallback_to_daylight))
    w.as_shot_wb_applied, w.colors, w.no_auto_scale = int(bool(as_shot_wb_applied)), int(colors), int(bool(no_auto_scale))
    return w


def wb_multipliers(inputs: "_lib.WbInputs", filters: int, maximum: int, black: int, channel_sums=None,
                   channel_counts=None) -> dict:
    """scale_colors' multiplier logic (host, bit-exact): returns scale_mul,
    pre_mul, maximum - black, and the auto-WB / bad-camera-WB flags.  The
    channel sums (:meth:`CudaAccelerator.channel_sums`) are needed only when
    the inputs select auto-WB."""
    lib = _lib.load()
    r = _lib.WbResult()
    sp = cp = None
    if channel_sums is not None:
        sums = np.ascontiguousarray(channel_sums, dtype=np.uint64)
        counts = np.ascontiguousarray(channel_counts, dtype=np.uint64)
        sp, cp = _ptr(sums), _ptr(counts)
    st = lib.lre_wb_multipliers(C.byref(inputs), int(filters), int(maximum), int(black), sp, cp, C.byref(r))
    if st != _lib.LRE_OK:
        raise LibRawError(st, "wb_multipliers: the inputs select auto-WB, which needs the channel sums")
    return {"scale_mul": np.array(r.scale_mul, np.float32), "pre_mul": np.array(r.pre_mul, np.float32),
            "maximum": int(r.maximum), "auto_wb": bool(r.auto_wb), "bad_camera_wb": bool(r.bad_camera_wb)}


def wb_needs_channel_sums(inputs: "_lib.WbInputs") -> bool:
    return bool(_lib.load().lre_wb_needs_channel_sums(C.byref(inputs)))


def raw_frame(raw_width, raw_height, width, height, filters, raw_pitch=None, top_margin=0, left_margin=0,
              shrink=0, xtrans=None, cblack=(), black=0, maximum=65535, green_matching=0, wb=(1.0, 1.0, 1.0, 1.0),
              adjust_maximum_thr=0.0, data_maximum=0.0, wb_in=None, fuji_width=0,
              fuji_layout=0) -> "_lib.RawFrame":
    """A LibRaw-style frame description for the raw ingest entry points.
    With ``wb_in`` (:func:`wb_inputs`) the develop derives the WB multipliers
    on the device as scale_colors does and ``wb`` is ignored."""
    f = _lib.RawFrame()
    f.raw_width, f.raw_height = int(raw_width), int(raw_height)
    f.raw_pitch = int(raw_pitch if raw_pitch is not None else 2 * raw_width)
    f.top_margin, f.left_margin = int(top_margin), int(left_margin)
    f.width, f.height = int(width), int(height)
    f.shrink = int(shrink)
    f.filters = int(filters)
    if xtrans is not None:
        x = np.asarray(xtrans, dtype=np.int8).reshape(36)
        C.memmove(C.addressof(f) + _lib.RawFrame.xtrans.offset, x.ctypes.data, 36)
    for i, v in enumerate(cblack):
        f.cblack[i] = int(v)
    f.black, f.maximum = int(black), int(maximum)
    f.green_matching = int(green_matching)
    for i, v in enumerate(wb):
        f.wb[i] = float(v)
    f.adjust_maximum_thr = float(adjust_maximum_thr)
    f.data_maximum = float(data_maximum)
    if wb_in is not None:
        f.derive_wb = 1
        f.wb_in = wb_in
    f.fuji_width, f.fuji_layout = int(fuji_width), int(fuji_layout)
    return f


def fuji_rotate_size(fuji_width: int, shrink: int, width: int, height: int):
    """Output (width, height) of the Fuji SuperCCD rotate, or None when the
    reference leaves the image unrotated (core/libraw_wrapper.cpp:1709-1718)."""
    ow, oh = C.c_size_t(), C.c_size_t()
    _lib.load().lre_fuji_rotate_size(int(fuji_width), int(shrink), int(width), int(height), C.byref(ow), C.byref(oh))
    return None if ow.value == 0 else (ow.value, oh.value)


def develop_params(**kw) -> DevelopParams:
    """ProcessingParams-style develop settings (reference defaults), overridden by kw.

    ``cfa`` may be a Bayer layout name, a LibRaw filters word, or a 6x6 X-Trans
    pattern; ``tone_mapping`` is 0 (off), 1 (ACES) or 2 (detail-preserving).
    """
    lib = _lib.load()
    p = DevelopParams()
    lib.lre_develop_params_default(C.byref(p))
    cfa = kw.pop("cfa", None)
    if cfa is not None:
        if isinstance(cfa, str):
            p.filters = FILTERS[cfa]
        elif np.ndim(cfa) == 2:
            p.filters = FILTERS_XTRANS
            x = np.asarray(cfa, dtype=np.int8).reshape(36)
            # write through the struct's own storage (reading p.xtrans yields a copy)
            C.memmove(C.addressof(p) + DevelopParams.xtrans.offset, x.ctypes.data, 36)
        else:
            p.filters = int(cfa)
    if "cam_mul" in kw:
        for i, v in enumerate(kw.pop("cam_mul")):
            p.cam_mul[i] = float(v)
    for k, v in kw.items():
        if not hasattr(p, k):
            raise TypeError(f"unknown develop parameter {k!r}")
        setattr(p, k, v)
    return p


_default = None


def default_accelerator() -> CudaAccelerator:
    global _default
    if _default is None:
        _default = CudaAccelerator(0)
    return _default


def develop(mosaic, **kw):
    """Plain per-image develop of a dense float32 CFA mosaic (see develop_params)."""
    return default_accelerator().develop(mosaic, develop_params(**kw))


# ---------------------------------------------------------------- standalone
# RawImage.tone_mapping / enhance_micro_contrast / defringe
# (libraw_enhanced/high_level_api.py:465-546 -> core/libraw_wrapper.cpp:3098-3214)
def tone_mapping(image, after_scale: float = 1.0) -> np.ndarray:
    return default_accelerator().tone_mapping(image, after_scale)


def enhance_micro_contrast(image, threshold: float = -1.0, strength: float = 8.0, target_contrast: float = 0.06) -> np.ndarray:
    """``threshold < 0`` means maximum/data_maximum in the reference; without a
    loaded RAW the ratio is 1.0 (core/libraw_wrapper.cpp:3140-3142)."""
    if threshold < 0.0:
        threshold = 1.0
    return default_accelerator().enhance_micro_contrast(image, threshold, strength, target_contrast)


def defringe(image, radius: float = 10.0, strength: float = 10.0, defringe_green: bool = False) -> np.ndarray:
    """Edge / chroma thresholds fixed at 0.1 / 0.15 as in defringe_numpy."""
    return default_accelerator().defringe(image, radius, 0.1, 0.15, strength, defringe_green)
