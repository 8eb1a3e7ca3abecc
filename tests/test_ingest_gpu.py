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
