"""On-device raw ingest against the oracle's restatements: raw2image, green
matching and the whole develop_raw chain (raw2image -> black level -> green
matching -> WB -> adjust_maximum -> develop), bit-exact."""
import numpy as np
import pytest

import oracle
from libraw_enhanced_b200 import scenes

pytestmark = pytest.mark.gpu

RGGB = 0x94949494
RGGB_G2 = 0xB4B4B4B4  # second green coded as colour 3


@pytest.fixture(scope="module")
def lre():
    import libraw_enhanced_b200 as m

    return m


@pytest.fixture(scope="module")
def acc(lre):
    a = lre.CudaAccelerator(0)
    yield a
    a.close()


def _raw_from_scene(h, w, cfa, seed, black=256, white=16383, margins=(3, 5), pad=7):
    """A raw_image with margins and row padding holding a scene mosaic."""
    mos = scenes.bayer_scene(h, w, seed, cfa=cfa, wb=(1, 1, 1, 1)) if not isinstance(cfa, np.ndarray) else \
        scenes.mosaic(scenes.scene_rgb(h, w, seed), cfa, (1, 1, 1, 1), seed)
    top, left = margins
    rh, rw = h + top + 2, w + left + 3
    pitch_px = rw + pad
    raw = np.full((rh, pitch_px), black // 2, np.uint16)
    vals = np.clip(np.round(mos * (white - black) * 0.8) + black, 0, 65535).astype(np.uint16)
    raw[top:top + h, left:left + w] = vals
    return raw, rw, rh, pitch_px * 2, top, left


@pytest.mark.parametrize("filters,shrink", [(RGGB, 0), (RGGB_G2, 0), (RGGB, 1), ("xtrans", 0)])
def test_raw2image_matches_oracle(lre, acc, filters, shrink):
    h, w = 130, 198
    xt = scenes.XTRANS_STD if filters == "xtrans" else None
    filt = 9 if filters == "xtrans" else filters
    raw, rw, rh, pitch, top, left = _raw_from_scene(h, w, "RGGB", 11)
    if filt == 9:
        raw = np.ascontiguousarray(raw[:, :rw])  # X-Trans rows are raw_width apart
    f = lre.raw_frame(rw, rh, w, h, filt, raw_pitch=pitch, top_margin=top, left_margin=left, shrink=shrink, xtrans=xt)
    got = acc.raw2image(raw, f)
    ref = oracle.raw2image(raw, pitch, top, left, w, h, filt, xt, shrink=shrink)
    assert np.array_equal(got, ref)


def test_green_matching_matches_oracle(lre, acc):
    h, w = 160, 224
    raw, rw, rh, pitch, top, left = _raw_from_scene(h, w, "RGGB", 12)
    img = oracle.raw2image(raw, pitch, top, left, w, h, RGGB_G2)
    for maximum in (16383, 4000):
        got = acc.green_matching(img, RGGB_G2, maximum)
        ref = oracle.green_matching(img, RGGB_G2, maximum)
        assert np.array_equal(got, ref)
        assert (got != img).any() or maximum == 4000
    assert np.array_equal(acc.green_matching(img, 9, 16383), img)


@pytest.mark.parametrize("filters", [RGGB_G2, RGGB])
def test_develop_raw_matches_composed_oracle_ingest(lre, acc, filters):
    h, w = 256, 384
    raw, rw, rh, pitch, top, left = _raw_from_scene(h, w, "RGGB", 13)
    cblack = (10, 4, 12, 6, 0, 0)
    wb = (2.0, 1.0, 1.5, 1.0)
    maximum = 16383 - 256
    f = lre.raw_frame(rw, rh, w, h, filters, raw_pitch=pitch, top_margin=top, left_margin=left, cblack=cblack,
                      black=256, maximum=maximum, green_matching=1, wb=wb, adjust_maximum_thr=0.75)
    p = lre.develop_params(cam_mul=wb, defringe=1, axial_ca_correction=1, tone_mapping=1, stage_order=1)
    got, used = acc.develop_raw(raw, f, p)
    # the reference's steps, restated on the CPU
    img = oracle.raw2image(raw, pitch, top, left, w, h, filters)
    img = oracle.black_level(img, cblack, 256, maximum)
    img = oracle.green_matching(img, filters, maximum)
    sparse = oracle.port_white_balance(img, wb, filters)
    adopted, _ = oracle.adjust_maximum(sparse, filters, 0.75, 0.0, float(maximum))
    assert used == adopted
    ch = scenes.cfa_map(h, w, filters)
    ch = np.where(ch == 3, 1, ch)
    dense = np.take_along_axis(sparse, ch[:, :, None], axis=2)[:, :, 0]
    p.filters = filters
    p.maximum_value = adopted
    ref = acc.develop(np.ascontiguousarray(dense), p)
    assert np.array_equal(got, ref)


def test_develop_raw_rejects_bad_frames(lre, acc):
    raw = np.zeros((40, 40), np.uint16)
    f = lre.raw_frame(40, 40, 40, 40, RGGB, raw_pitch=41)  # odd pitch
    with pytest.raises(lre.LibRawError):
        acc.develop_raw(raw, f, lre.develop_params())
    f = lre.raw_frame(40, 40, 40, 40, RGGB, top_margin=40)
    with pytest.raises(lre.LibRawError):
        acc.develop_raw(raw, f, lre.develop_params())


@pytest.mark.parametrize("filters", [RGGB_G2, "xtrans"])
def test_channel_sums_match_numpy(lre, acc, filters):
    """The auto-WB statistics (core/libraw_wrapper.cpp:632-661) reduced on
    the device: exact 64-bit sums and counts per native colour."""
    rng = np.random.default_rng(21)
    raw4 = rng.integers(0, 65536, size=(301, 517, 4), dtype=np.uint16)
    xt = scenes.XTRANS_STD if filters == "xtrans" else None
    filt = 9 if filters == "xtrans" else filters
    sums, counts = acc.channel_sums(raw4, filt, xt)
    idx = scenes.cfa_map(301, 517, xt if xt is not None else filt)
    vals = np.take_along_axis(raw4.astype(np.uint64), idx[:, :, None], axis=2)[:, :, 0]
    assert sums.tolist() == [int(vals[idx == c].sum()) for c in range(4)]
    assert counts.tolist() == [int((idx == c).sum()) for c in range(4)]


@pytest.mark.parametrize("mode", ["auto", "camera", "daylight"])
def test_develop_raw_derives_wb_like_scale_colors(lre, acc, mode):
    """develop_raw with frame.wb_in: the multipliers come from scale_colors'
    logic (core/libraw_wrapper.cpp:602-845) after black level and green
    matching, and adjust_maximum compares against maximum - black, as the
    reference pipeline does (:1515-1575)."""
    h, w = 256, 384
    raw, rw, rh, pitch, top, left = _raw_from_scene(h, w, "RGGB", 14)
    cblack = (10, 4, 12, 6, 0, 0)
    black, maximum = 256, 16383
    white = np.full((8, 8), 900, np.uint16)
    white[::2, ::2] = 500  # R sites of RGGB
    kw = {"auto": dict(use_auto_wb=True),
          "camera": dict(use_camera_wb=True, cam_mul=(2.0, 1.0, 1.5, 0.0), white=white, cblack=cblack[:4]),
          "daylight": dict(pre_mul=(2.2, 1.0, 1.4, 0.0))}[mode]
    inputs = lre.wb_inputs(**kw)
    f = lre.raw_frame(rw, rh, w, h, RGGB_G2, raw_pitch=pitch, top_margin=top, left_margin=left, cblack=cblack,
                      black=black, maximum=maximum, green_matching=1, adjust_maximum_thr=0.75, wb_in=inputs)
    p = lre.develop_params(cam_mul=(2.0, 1.0, 1.5, 1.0), defringe=1, axial_ca_correction=1, stage_order=1)
    got, used = acc.develop_raw(raw, f, p)
    # the reference's steps, restated on the CPU
    img = oracle.raw2image(raw, pitch, top, left, w, h, RGGB_G2)
    img = oracle.black_level(img, cblack, black, maximum)
    img = oracle.green_matching(img, RGGB_G2, maximum)
    okw = dict(kw)
    if "cblack" in okw:
        okw["cblack"] = tuple(okw["cblack"])
    scale_mul, _, mx_after, _ = oracle.scale_colors(img, RGGB_G2, maximum=maximum, black=black, **okw)
    sparse = oracle.port_white_balance(img, scale_mul, RGGB_G2)
    adopted, _ = oracle.adjust_maximum(sparse, RGGB_G2, 0.75, 0.0, float(mx_after))
    assert used == adopted
    # the same multipliers through the standalone entry points
    r = acc.scale_colors(img, RGGB_G2, inputs, maximum, black)
    assert r["scale_mul"].view(np.uint32).tolist() == scale_mul.view(np.uint32).tolist()
    ch = scenes.cfa_map(h, w, RGGB_G2)
    ch = np.where(ch == 3, 1, ch)
    dense = np.take_along_axis(sparse, ch[:, :, None], axis=2)[:, :, 0]
    p.filters = RGGB_G2
    p.maximum_value = adopted
    ref = acc.develop(np.ascontiguousarray(dense), p)
    assert np.array_equal(got, ref)


@pytest.mark.parametrize("fuji_layout,shrink", [(1, 0), (0, 0), (1, 1), (0, 1)])
def test_raw2image_fuji_honeycomb(lre, acc, fuji_layout, shrink):
    """Fuji SuperCCD honeycomb raw2image (core/libraw_wrapper.cpp:2342-2392):
    raw rows and columns mapped onto the 45-degree frame, bit-exact against
    the oracle's forward scan (the device inverts the map per pixel)."""
    rng = np.random.default_rng(31 + 2 * fuji_layout + shrink)
    fuji_width = 181
    copy_cols = fuji_width << (0 if fuji_layout else 1)
    top, left = 4, 3
    rh, rw = 260 + 2 * top, copy_cols + left + 5
    pitch_px = rw + 6
    raw = rng.integers(0, 16384, size=(rh, pitch_px), dtype=np.uint16)
    width, height = 420, 400
    for filters in (RGGB, RGGB_G2):
        f = lre.raw_frame(rw, rh, width, height, filters, raw_pitch=pitch_px * 2, top_margin=top, left_margin=left,
                          shrink=shrink, fuji_width=fuji_width, fuji_layout=fuji_layout)
        got = acc.raw2image(raw, f)
        ref = oracle.raw2image_fuji(raw, pitch_px * 2, top, left, width, height, filters, fuji_width, fuji_layout,
                                    shrink, raw_width=rw)
        assert np.array_equal(got, ref)
        assert (ref != 0).any(axis=2).mean() > 0.2


def test_fuji_rotate_bit_exact(lre, acc):
    """The 45-degree Fuji rotate after demosaic (core/libraw_wrapper.cpp:
    1709-1750): same output size and values as the reference's loop."""
    rgb = np.random.default_rng(33).random((403, 371, 3), dtype=np.float32) * np.float32(1.2)
    for fuji_width, shrink in ((180, 0), (181, 1)):
        ref = oracle.fuji_rotate(rgb, fuji_width, shrink)
        assert lre.fuji_rotate_size(fuji_width, shrink, 371, 403) == (ref.shape[1], ref.shape[0])
        got = acc.fuji_rotate(rgb, fuji_width, shrink)
        assert np.array_equal(got, ref)
    assert lre.fuji_rotate_size(0, 0, 371, 403) is None
