"""TEST INFRASTRUCTURE -- the oracle the CUDA develop path is checked against.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg import this package.  The product (``libraw_enhanced_b200``) never does.

Two libraries back it, both built by ``oracle/Makefile``:

* ``ref``  -- ``oracle/_ref/liblre_ref.so``: uniuyuni/libraw_enhanced's own
  ``CPUAccelerator`` (core/cpu_accelerator.cpp) compiled from the reference
  sources, behind the C ABI in ``oracle/ref_capi.cpp``.  This is the parity
  reference for AMaZE, X-Trans, white balance, defringe, axial/lateral CA,
  ACES tone mapping and micro-contrast.
* ``port`` -- ``oracle/liblre_oracle.so``: a plain-C restatement
  (``oracle/lre_oracle.c``) of the LibRaw-dependent pieces that cannot be
  compiled here (black level, adjust_maximum, detail-preserving tone map,
  output quantization, WB-multiplier derivation) plus restatements of ACES,
  white balance, CFA indexing and border interpolation that are pinned against
  ``ref`` by the CPU test-suite.

All images are numpy arrays in the reference's layouts: float32 (H, W, 3)
interleaved, uint16 (H, W, 4) raw.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_SO = os.path.join(HERE, "_ref", "liblre_ref.so")
PORT_SO = os.path.join(HERE, "liblre_oracle.so")

_f = C.c_float
_sz = C.c_size_t
_p = C.c_void_p


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p)


def _img(a):
    a = np.ascontiguousarray(a, dtype=np.float32)
    assert a.ndim == 3 and a.shape[2] == 3, a.shape
    return a


class _Lib:
    def __init__(self, path, sigs):
        if not os.path.exists(path):
            raise FileNotFoundError(f"oracle library missing: {path} (run `make -C oracle`)")
        self.lib = C.CDLL(path)
        for name, (res, args) in sigs.items():
            fn = getattr(self.lib, name)
            fn.restype = res
            fn.argtypes = args


_REF_SIGS = {
    "ref_num_threads": (C.c_int, []),
    "ref_set_num_threads": (None, [C.c_int]),
    "ref_demosaic_bayer_amaze": (C.c_int, [_p, _p, _sz, _sz, C.c_uint32, _p, _f]),
    "ref_demosaic_bayer_linear": (C.c_int, [_p, _p, _sz, _sz, C.c_uint32, _f]),
    "ref_demosaic_bayer_dcb": (C.c_int, [_p, _p, _sz, _sz, C.c_uint32, _f, C.c_int, C.c_int]),
    "ref_demosaic_bayer_aahd": (C.c_int, [_p, _p, _sz, _sz, C.c_uint32, _f]),
    "ref_demosaic_xtrans": (C.c_int, [_p, _p, _sz, _sz, _p, _p, _f, C.c_int]),
    "ref_apply_white_balance": (C.c_int, [_p, _p, _sz, _sz, _p, C.c_uint32, _p]),
    "ref_tone_mapping": (C.c_int, [_p, _p, _sz, _sz, _f]),
    "ref_convert_color_space": (C.c_int, [_p, _p, _sz, _sz, _p]),
    "ref_gamma_correct": (C.c_int, [_p, _p, _sz, _sz, _f, _f, C.c_int]),
    "ref_enhance_micro_contrast": (C.c_int, [_p, _p, _sz, _sz, _f, _f, _f, _p]),
    "ref_defringe": (C.c_int, [_p, _p, _sz, _sz, _f, _f, _f, _f, C.c_int, _f]),
    "ref_ca_register_lateral": (C.c_int, [_p, _p, _sz, _sz, C.c_int, C.c_int, _f, _f, C.c_int]),
    "ref_ca_axial_cleanup": (C.c_int, [_p, _p, _sz, _sz, C.c_int, _f, _f]),
    "ref_pre_interpolate": (C.c_int, [_p, _sz, _sz, C.c_uint32, _p, C.c_int]),
}

_PORT_SIGS = {
    "port_fcol_bayer_native": (C.c_uint, [C.c_uint, C.c_uint, C.c_uint32]),
    "port_fcol_bayer": (C.c_uint, [C.c_uint, C.c_uint, C.c_uint32]),
    "port_fcol_xtrans": (C.c_uint, [C.c_uint, C.c_uint, _p]),
    "port_black_level": (None, [_p, _sz, _sz, _p, C.c_uint, C.c_uint]),
    "port_raw2image": (None, [_p, _sz, _sz, _sz, _sz, _sz, _sz, _sz, C.c_int, C.c_uint32, _p, _p]),
    "port_green_matching": (None, [_p, _sz, _sz, C.c_uint32, C.c_int]),
    "port_white_balance": (None, [_p, _p, _sz, _sz, _p, C.c_uint32, _p]),
    "port_adjust_maximum": (_f, [_p, _sz, _sz, C.c_uint32, _f, C.POINTER(_f), _f]),
    "port_tone_mapping": (None, [_p, _p, _sz, _f]),
    "port_detail_tonemap": (C.c_longlong, [_p, _sz, _sz]),
    "port_quantize_u16": (None, [_p, _p, _sz]),
    "port_quantize_u8": (None, [_p, _p, _sz]),
    "port_scale_mul": (None, [_p, C.c_int, _f, _p]),
    "port_auto_wb": (None, [_p, _sz, _sz, C.c_uint32, _p, _p]),
    "port_border_interpolate": (None, [_p, _sz, _sz, C.c_uint32, _sz]),
    "port_raw2image_fuji": (None, [_p, _sz, _sz, _sz, _sz, _sz, _sz, _sz, C.c_int, C.c_uint32, C.c_int, C.c_int,
                                    _p]),
    "port_fuji_rotate": (None, [_p, _sz, _sz, C.c_int, C.c_int, _p, C.POINTER(_sz), C.POINTER(_sz)]),
    "port_scale_colors": (C.c_int, [_p, _sz, _sz, C.c_uint32, _p, _p, _p, _p, _p, _p, C.c_int, C.c_int,
                                    C.POINTER(C.c_uint), C.c_uint, _p, _p]),
}

_ref = None
_port = None


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def ref():
    global _ref
    if _ref is None:
        _ref = _Lib(REF_SO, _REF_SIGS).lib
    return _ref


def port():
    global _port
    if _port is None:
        _port = _Lib(PORT_SO, _PORT_SIGS).lib
    return _port


def _xt(xtrans):
    if xtrans is None:
        return np.zeros(36, dtype=np.int8)
    return np.ascontiguousarray(np.asarray(xtrans, dtype=np.int8).reshape(36))


# ---------------------------------------------------------------- reference
def set_threads(n: int) -> None:
    ref().ref_set_num_threads(int(n))


def num_threads() -> int:
    return int(ref().ref_num_threads())


def amaze_tiles(h: int, w: int) -> int:
    """Tiles of the reference AMaZE tile loop (core/cpu_accelerator.cpp:1244-1245):
    160x160 tiles stepping by 128 from -16 in both directions."""
    return len(range(-16, h, 128)) * len(range(-16, w, 128))


def xtrans_tiles(h: int, w: int) -> int:
    """Tiles of the reference X-Trans 3-pass tile loop (core/cpu_accelerator.cpp:1968-1969):
    114x114 tiles stepping by 98 from 3 while below the size minus 19."""
    return len(range(3, h - 19, 98)) * len(range(3, w - 19, 98))


class _Threads:
    """Temporarily run the reference with `n` OpenMP threads."""

    def __init__(self, n):
        self.n = n

    def __enter__(self):
        self.saved = num_threads()
        if self.n:
            set_threads(self.n)

    def __exit__(self, *exc):
        set_threads(self.saved)


def amaze(raw_sparse, filters, cam_mul=(2.0, 1.0, 1.5, 1.0), maximum=1.0, fresh_tiles=False):
    """The reference AMaZE (core/cpu_accelerator.cpp:1145-1653).

    The reference allocates its tile scratch once per OpenMP thread
    (:1217-1218) and never fills the apron corners of tiles that touch two
    image edges (:1326), so those cells hold what the thread's previous tile
    left.  ``fresh_tiles=True`` runs one thread per tile (the static
    ``omp for`` then gives every thread exactly one tile), so every tile
    starts from a zero-filled buffer and the result is a function of the
    input alone -- the semantics the CUDA path implements."""
    raw = _img(raw_sparse)
    h, w, _ = raw.shape
    out = np.zeros_like(raw)
    cm = np.asarray(cam_mul, dtype=np.float32)
    with _Threads(amaze_tiles(h, w) if fresh_tiles else 0):
        ok = ref().ref_demosaic_bayer_amaze(_ptr(raw), _ptr(out), w, h, int(filters), _ptr(cm), float(maximum))
    assert ok
    return out


def bayer_linear(raw_sparse, filters, maximum=1.0):
    raw = _img(raw_sparse)
    h, w, _ = raw.shape
    out = np.zeros_like(raw)
    assert ref().ref_demosaic_bayer_linear(_ptr(raw), _ptr(out), w, h, int(filters), float(maximum))
    return out


def bayer_dcb(raw_sparse, filters, maximum=1.0, iterations=1, enhance=True, threads=1):
    """The reference's DCB demosaic (core/cpu_accelerator.cpp:1043-1137).

    ``threads=1`` (the default) gives the sequential result of DCB's in-place
    passes; with more OpenMP threads the reference's row-parallel nyquist, pp
    and color_full loops read rows that other threads are rewriting, so rows
    at each thread's chunk boundary depend on timing."""
    raw = _img(raw_sparse)
    h, w, _ = raw.shape
    out = np.zeros_like(raw)
    saved = num_threads()
    set_threads(threads)
    try:
        assert ref().ref_demosaic_bayer_dcb(_ptr(raw), _ptr(out), w, h, int(filters), float(maximum),
                                            int(iterations), int(bool(enhance)))
    finally:
        set_threads(saved)
    return out


REF_HL_SO = os.path.join(HERE, "_ref", "liblre_ref_hl.so")
REF_DT_SO = os.path.join(HERE, "_ref", "liblre_ref_dt.so")
_ref_hl = None
_ref_dt = None


def ref_detail_tonemap(img):
    """The reference's detail-preserving tone map, compiled from its own lines
    (core/libraw_wrapper.cpp:45-116 box_filter_normalized and :1389-1471
    aces_tone_map_scalar + apply_detail_preserving_tonemap) into
    oracle/_ref/liblre_ref_dt.so.  Returns the tone-mapped copy."""
    global _ref_dt
    if _ref_dt is None:
        if not os.path.exists(REF_DT_SO):
            raise FileNotFoundError(f"oracle library missing: {REF_DT_SO} (run `make -C oracle ref`)")
        _ref_dt = C.CDLL(REF_DT_SO)
        _ref_dt.ref_detail_tonemap.restype = C.c_int
        _ref_dt.ref_detail_tonemap.argtypes = [_p, _sz, _sz]
    a = _img(img).copy()
    _ref_dt.ref_detail_tonemap(_ptr(a), a.shape[1], a.shape[0])
    return a


def recover_highlights(rgb, saturation_threshold, want_mask=False, wb_rgb=None):
    """The reference's highlight recovery (core/libraw_wrapper.cpp:1095-1383),
    compiled from those lines alone.  Returns (recovered copy, mask or None)."""
    global _ref_hl
    if _ref_hl is None:
        _ref_hl = C.CDLL(REF_HL_SO)
        _ref_hl.ref_recover_highlights.restype = C.c_int
        _ref_hl.ref_recover_highlights.argtypes = [_p, _sz, _sz, _f, _p, _p]
    img = np.ascontiguousarray(rgb, dtype=np.float32).copy()
    h, w, _ = img.shape
    mask = np.zeros((h, w), np.float32) if want_mask else None
    wb = None if wb_rgb is None else np.asarray(wb_rgb, np.float32)
    _ref_hl.ref_recover_highlights(_ptr(img), w, h, float(saturation_threshold),
                                   None if mask is None else _ptr(mask), None if wb is None else _ptr(wb))
    return img, mask


def bayer_aahd(raw_sparse, filters, maximum=1.0, threads=1):
    """The reference's AAHD demosaic (core/cpu_accelerator.cpp:617-633), by
    default single-threaded: its in-place row loops and channel min/max scan
    are order-dependent under OpenMP."""
    raw = _img(raw_sparse)
    h, w, _ = raw.shape
    out = np.zeros_like(raw)
    saved = num_threads()
    set_threads(threads)
    try:
        assert ref().ref_demosaic_bayer_aahd(_ptr(raw), _ptr(out), w, h, int(filters), float(maximum))
    finally:
        set_threads(saved)
    return out


def xtrans(raw_sparse, xtrans_pattern, passes=3, maximum=1.0, color_matrix=None, fresh_tiles=False):
    """The reference X-Trans demosaic (core/cpu_accelerator.cpp:1870-2762).

    The 3-pass tile buffers are allocated once per OpenMP thread (:1953-1959)
    and the homogeneity maps of edge tiles read cells their tile never
    writes; ``fresh_tiles=True`` runs one thread per tile so that every tile
    starts from zero-filled buffers (see :func:`amaze`)."""
    raw = _img(raw_sparse)
    h, w, _ = raw.shape
    out = np.zeros_like(raw)
    cm = np.zeros(12, np.float32) if color_matrix is None else np.asarray(color_matrix, np.float32).reshape(12)
    xt = _xt(xtrans_pattern)
    n = xtrans_tiles(h, w) if (fresh_tiles and passes != 1) else 0
    with _Threads(n):
        ok = ref().ref_demosaic_xtrans(_ptr(raw), _ptr(out), w, h, _ptr(xt), _ptr(cm), float(maximum), int(passes))
    assert ok
    return out


def white_balance(raw4, wb, filters, xtrans_pattern=None, out=None):
    raw4 = np.ascontiguousarray(raw4, dtype=np.uint16)
    h, w, _ = raw4.shape
    out = np.zeros((h, w, 3), np.float32) if out is None else np.ascontiguousarray(out, np.float32)
    wbv = np.asarray(wb, dtype=np.float32)
    ok = ref().ref_apply_white_balance(_ptr(raw4), _ptr(out), w, h, _ptr(wbv), int(filters), _ptr(_xt(xtrans_pattern)))
    assert ok
    return out


def tone_mapping(img, after_scale=1.0):
    a = _img(img)
    out = np.empty_like(a)
    assert ref().ref_tone_mapping(_ptr(a), _ptr(out), a.shape[1], a.shape[0], float(after_scale))
    return out


def micro_contrast(img, threshold=0.5, strength=8.0, target=0.06, mask=None):
    a = _img(img)
    out = np.empty_like(a)
    mp = None
    if mask is not None:
        mask = np.ascontiguousarray(mask, dtype=np.float32)
        mp = _ptr(mask)
    assert ref().ref_enhance_micro_contrast(
        _ptr(a), _ptr(out), a.shape[1], a.shape[0], float(threshold), float(strength), float(target), mp
    )
    return out


def defringe(img, radius=10.0, edge=0.1, chroma=0.15, strength=10.0, green=False, green_scale=0.3):
    a = _img(img)
    out = np.empty_like(a)
    assert ref().ref_defringe(
        _ptr(a), _ptr(out), a.shape[1], a.shape[0], float(radius), float(edge), float(chroma),
        float(strength), int(bool(green)), float(green_scale),
    )
    return out


def lateral_ca(img, cell=96, iters=3, max_shift=6.0, min_conf=0.02, levels=3):
    a = _img(img)
    out = np.empty_like(a)
    assert ref().ref_ca_register_lateral(
        _ptr(a), _ptr(out), a.shape[1], a.shape[0], int(cell), int(iters), float(max_shift), float(min_conf), int(levels)
    )
    return out


def axial_ca(img, radius=6, eps=1e-4, strength=0.3):
    a = _img(img)
    out = np.empty_like(a)
    assert ref().ref_ca_axial_cleanup(_ptr(a), _ptr(out), a.shape[1], a.shape[0], int(radius), float(eps), float(strength))
    return out


def convert_color_space(img, transform):
    a = _img(img)
    out = np.empty_like(a)
    t = np.ascontiguousarray(transform, dtype=np.float32).reshape(12)
    assert ref().ref_convert_color_space(_ptr(a), _ptr(out), a.shape[1], a.shape[0], _ptr(t))
    return out


def gamma_correct(img, gamma_power=0.0, gamma_slope=0.0, color_space=1):
    a = _img(img)
    out = np.empty_like(a)
    assert ref().ref_gamma_correct(_ptr(a), _ptr(out), a.shape[1], a.shape[0], float(gamma_power), float(gamma_slope),
                                   int(color_space))
    return out


# ---------------------------------------------------------------- restatement
def black_level(raw4, cblack, black, maximum):
    """cblack: sequence of 6 + n ints (LibRaw layout)."""
    a = np.ascontiguousarray(raw4, dtype=np.uint16).copy()
    cb = np.zeros(6 + 4104, dtype=np.uint32)
    cb[: len(cblack)] = np.asarray(cblack, dtype=np.uint32)
    port().port_black_level(_ptr(a), a.shape[1], a.shape[0], _ptr(cb), int(black), int(maximum))
    return a


def raw2image(raw, raw_pitch, top_margin, left_margin, width, height, filters, xtrans_pattern=None, shrink=0):
    """raw: (raw_height, raw_width) uint16 (Bayer rows raw_pitch bytes apart)."""
    raw = np.ascontiguousarray(raw, dtype=np.uint16)
    rh, rw = raw.shape
    iw, ih = (width + shrink) >> shrink, (height + shrink) >> shrink
    out = np.zeros((ih, iw, 4), np.uint16)
    port().port_raw2image(_ptr(raw), rw, rh, int(raw_pitch), int(top_margin), int(left_margin), int(width),
                          int(height), int(shrink), int(filters), _ptr(_xt(xtrans_pattern)), _ptr(out))
    return out


def raw2image_fuji(raw, raw_pitch, top_margin, left_margin, width, height, filters, fuji_width, fuji_layout,
                   shrink=0, raw_width=None):
    """The Fuji SuperCCD honeycomb raw2image (core/libraw_wrapper.cpp:2342-2392).
    raw: (raw_height, raw_pitch // 2) uint16; raw_width defaults to the row length."""
    raw = np.ascontiguousarray(raw, dtype=np.uint16)
    rh, rw = raw.shape
    if raw_width is not None:
        rw = int(raw_width)
    iw, ih = (width + shrink) >> shrink, (height + shrink) >> shrink
    out = np.zeros((ih, iw, 4), np.uint16)
    port().port_raw2image_fuji(_ptr(raw), rw, rh, int(raw_pitch), int(top_margin), int(left_margin), int(width),
                               int(height), int(shrink), int(filters), int(fuji_width), int(fuji_layout), _ptr(out))
    return out


def fuji_rotate(rgb, fuji_width, shrink=0):
    """The 45-degree Fuji rotate after demosaic (core/libraw_wrapper.cpp:1709-1750);
    returns the input unchanged when the reference would not rotate."""
    a = _img(rgb)
    h, w, _ = a.shape
    ow, oh = _sz(0), _sz(0)
    port().port_fuji_rotate(_ptr(a), w, h, int(fuji_width), int(shrink), None, C.byref(ow), C.byref(oh))
    if ow.value == 0:
        return a.copy()
    out = np.empty((oh.value, ow.value, 3), np.float32)
    port().port_fuji_rotate(_ptr(a), w, h, int(fuji_width), int(shrink), _ptr(out), C.byref(ow), C.byref(oh))
    return out


def green_matching(raw4, filters, maximum):
    a = np.ascontiguousarray(raw4, dtype=np.uint16).copy()
    port().port_green_matching(_ptr(a), a.shape[1], a.shape[0], int(filters), int(maximum))
    return a


def port_white_balance(raw4, wb, filters, xtrans_pattern=None, out=None):
    raw4 = np.ascontiguousarray(raw4, dtype=np.uint16)
    h, w, _ = raw4.shape
    out = np.zeros((h, w, 3), np.float32) if out is None else np.ascontiguousarray(out, np.float32).copy()
    wbv = np.asarray(wb, dtype=np.float32)
    port().port_white_balance(_ptr(raw4), _ptr(out), w, h, _ptr(wbv), int(filters), _ptr(_xt(xtrans_pattern)))
    return out


def adjust_maximum(rgb, filters, threshold, data_maximum, maximum):
    a = _img(rgb)
    dm = C.c_float(float(data_maximum))
    m = port().port_adjust_maximum(_ptr(a), a.shape[1], a.shape[0], int(filters), float(threshold), C.byref(dm), float(maximum))
    return float(m), float(dm.value)


def port_tone_mapping(img, after_scale=1.0):
    a = _img(img)
    out = np.empty_like(a)
    port().port_tone_mapping(_ptr(a), _ptr(out), a.shape[0] * a.shape[1], float(after_scale))
    return out


def detail_tonemap(img):
    a = _img(img).copy()
    port().port_detail_tonemap(_ptr(a), a.shape[1], a.shape[0])
    return a


def quantize_u16(img):
    a = np.ascontiguousarray(img, dtype=np.float32)
    out = np.empty(a.shape, np.uint16)
    port().port_quantize_u16(_ptr(a), _ptr(out), a.size)
    return out


def quantize_u8(img):
    a = np.ascontiguousarray(img, dtype=np.float32)
    out = np.empty(a.shape, np.uint8)
    port().port_quantize_u8(_ptr(a), _ptr(out), a.size)
    return out


def scale_mul(pre_mul, colors=3, maximum=1.0):
    pm = np.asarray(pre_mul, dtype=np.float32)
    out = np.empty(4, np.float32)
    port().port_scale_mul(_ptr(pm), int(colors), float(maximum), _ptr(out))
    return out


def auto_wb(raw4, filters, xtrans_pattern=None):
    a = np.ascontiguousarray(raw4, dtype=np.uint16)
    out = np.empty(4, np.float32)
    port().port_auto_wb(_ptr(a), a.shape[1], a.shape[0], int(filters), _ptr(_xt(xtrans_pattern)), _ptr(out))
    return out


def scale_colors(raw4, filters, xtrans_pattern=None, *, user_mul=(0, 0, 0, 0), pre_mul=(1, 1, 1, 1),
                 cam_mul=(0, 0, 0, 0), white=None, cblack=(0, 0, 0, 0), colors=3, use_auto_wb=False,
                 use_camera_wb=False, fallback_daylight=False, as_shot_wb_applied=False, no_auto_scale=False,
                 maximum=16383, black=0):
    """scale_colors' multiplier derivation (core/libraw_wrapper.cpp:602-845).
    Returns (scale_mul[4], pre_mul[4], maximum - black, bad_camera_wb)."""
    a = np.zeros((1, 1, 4), np.uint16) if raw4 is None else np.ascontiguousarray(raw4, dtype=np.uint16)
    h, w = a.shape[:2]
    f4 = lambda v: np.ascontiguousarray(np.asarray(v, np.float32).reshape(4))  # noqa: E731
    um, pm, cm = f4(user_mul), f4(pre_mul), f4(cam_mul)
    wh = np.zeros(64, np.uint16) if white is None else np.ascontiguousarray(np.asarray(white, np.uint16).reshape(64))
    cb = np.ascontiguousarray(np.asarray(cblack, np.uint32).reshape(4))
    flags = (int(bool(use_auto_wb)) | int(bool(use_camera_wb)) << 1 | int(bool(fallback_daylight)) << 2
             | int(bool(as_shot_wb_applied)) << 3 | int(bool(no_auto_scale)) << 4)
    mx = C.c_uint(int(maximum))
    sm = np.empty(4, np.float32)
    po = np.empty(4, np.float32)
    warn = port().port_scale_colors(_ptr(a), w, h, int(filters), _ptr(_xt(xtrans_pattern)), _ptr(um), _ptr(pm),
                                    _ptr(cm), _ptr(wh), _ptr(cb), int(colors), flags, C.byref(mx), int(black),
                                    _ptr(sm), _ptr(po))
    return sm, po, int(mx.value), bool(warn)


def border_interpolate(rgb, filters, border=4):
    a = _img(rgb).copy()
    port().port_border_interpolate(_ptr(a), a.shape[1], a.shape[0], int(filters), int(border))
    return a
