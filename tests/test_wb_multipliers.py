"""White-balance multiplier derivation (LibRaw's scale_colors,
core/libraw_wrapper.cpp:602-845) in the product (lre_wb_multipliers, host
code of liblre_cuda.so) against the oracle's restatement (port_scale_colors),
bit for bit, over seeded inputs that reach every branch: user multipliers,
auto-WB (grey world, Bayer and X-Trans), camera WB from the white block, the
as-shot and Nikon sRAW daylight cases, the pre_mul defaults, the unsigned
maximum - black, and no_auto_scale.  No GPU is used: the multiplier logic is
host code, and the auto-WB channel sums are formed here with numpy (the
device reduction is checked against the same sums in tests/test_ingest_gpu.py).
"""
import numpy as np
import pytest

import oracle
from libraw_enhanced_b200 import scenes

lre = pytest.importorskip("libraw_enhanced_b200")


def _sums(raw4, filters, xtrans=None):
    h, w = raw4.shape[:2]
    if filters == scenes.FILTERS_XTRANS:
        idx = scenes.cfa_map(h, w, np.asarray(xtrans))
    else:
        idx = scenes.cfa_map(h, w, int(filters))
    vals = np.take_along_axis(raw4.astype(np.uint64), idx[:, :, None], axis=2)[:, :, 0]
    sums = np.array([vals[idx == c].sum() for c in range(4)], np.uint64)
    counts = np.array([(idx == c).sum() for c in range(4)], np.uint64)
    return sums, counts


def _case(rng, filters, xtrans=None):
    h, w = int(rng.integers(2, 40)), int(rng.integers(2, 40))
    raw4 = rng.integers(0, 16384, size=(h, w, 4), dtype=np.uint16)
    if rng.random() < 0.1:
        raw4[..., 0] = 0  # an all-dark red channel: G / R = inf
    kw = dict(
        user_mul=tuple(rng.uniform(0.5, 3.0, 4)) if rng.random() < 0.2 else (0.0, 0.0, 0.0, 0.0),
        pre_mul=tuple(float(v) for v in rng.choice([0.0, 1.0, 1.7, 2.3, 0.000005], 4)),
        cam_mul=tuple(float(v) for v in rng.choice([-1.0, 0.0, 0.000001, 1.0, 1.4, 2.2], 4)),
        white=rng.integers(0, 2000, size=(8, 8)) if rng.random() < 0.7 else np.zeros((8, 8), np.int64),
        cblack=tuple(int(v) for v in rng.integers(0, 700, 4)),
        colors=int(rng.choice([3, 4])),
        use_auto_wb=bool(rng.random() < 0.3),
        use_camera_wb=bool(rng.random() < 0.6),
        fallback_daylight=bool(rng.random() < 0.3),
        as_shot_wb_applied=bool(rng.random() < 0.2),
        no_auto_scale=bool(rng.random() < 0.1),
    )
    maximum = int(rng.choice([16383, 4095, 300, 0]))
    black = int(rng.choice([0, 256, 512, 400]))
    return raw4, kw, maximum, black


def _product(raw4, filters, xtrans, kw, maximum, black):
    inputs = lre.wb_inputs(user_mul=kw["user_mul"], pre_mul=kw["pre_mul"], cam_mul=kw["cam_mul"], white=kw["white"],
                           cblack=kw["cblack"], use_auto_wb=kw["use_auto_wb"], use_camera_wb=kw["use_camera_wb"],
                           camerawb_fallback_to_daylight=kw["fallback_daylight"],
                           as_shot_wb_applied=kw["as_shot_wb_applied"], colors=kw["colors"],
                           no_auto_scale=kw["no_auto_scale"])
    if lre.wb_needs_channel_sums(inputs):
        sums, counts = _sums(raw4, filters, xtrans)
        return lre.wb_multipliers(inputs, filters, maximum, black, sums, counts)
    return lre.wb_multipliers(inputs, filters, maximum, black)


@pytest.mark.parametrize("cfa", ["RGGB", "BGGR", "GRBG", "GBRG", "xtrans"])
def test_wb_multipliers_match_restatement(cfa):
    rng = np.random.default_rng(300 + len(cfa) + (7 if cfa == "xtrans" else 0))
    filters = scenes.FILTERS_XTRANS if cfa == "xtrans" else scenes.FILTERS[cfa]
    xt = scenes.XTRANS_STD if cfa == "xtrans" else None
    branches = set()
    with np.errstate(all="ignore"):
        for _ in range(400):
            raw4, kw, maximum, black = _case(rng, filters, xt)
            got = _product(raw4, filters, xt, kw, maximum, black)
            sm, pm, mx, warn = oracle.scale_colors(raw4, filters, xt, maximum=maximum, black=black, **kw)
            np.testing.assert_array_equal(got["scale_mul"].view(np.uint32), sm.view(np.uint32))
            np.testing.assert_array_equal(got["pre_mul"].view(np.uint32), pm.view(np.uint32))
            assert got["maximum"] == mx and got["bad_camera_wb"] == warn
            branches.add((got["auto_wb"], warn, kw["as_shot_wb_applied"], kw["no_auto_scale"]))
    assert len(branches) >= 5, branches


def test_wb_known_answers():
    f = scenes.FILTERS["RGGB"]
    # camera WB from metadata only (white block empty): pre_mul = cam_mul,
    # pre_mul[3] = pre_mul[1] for 3 colours, normalised by the minimum
    r = lre.wb_multipliers(lre.wb_inputs(cam_mul=(2.0, 1.0, 1.5, 0.0), use_camera_wb=True), f, 16383, 512)
    assert r["scale_mul"].tolist() == [2.0, 1.0, 1.5, 1.0] and r["maximum"] == 16383 - 512
    # daylight multipliers (float fields), divided by their minimum in double
    r = lre.wb_multipliers(lre.wb_inputs(pre_mul=(2.4, 1.2, 1.8, 1.2)), f, 16383, 0)
    q = lambda a, b: np.float32(np.float64(np.float32(a)) / np.float64(np.float32(b)))  # noqa: E731
    assert r["scale_mul"].tolist() == [q(2.4, 1.2), 1.0, q(1.8, 1.2), 1.0]
    # auto-WB: grey-world means, G2 folded into G, not normalised
    raw4 = np.zeros((2, 2, 4), np.uint16)
    raw4[0, 0, 0] = 100
    raw4[0, 1, 1] = 200
    raw4[1, 0, 1] = 200  # RGGB codes both greens as colour 1
    raw4[1, 1, 2] = 50
    inp = lre.wb_inputs(use_auto_wb=True)
    sums, counts = _sums(raw4, f)
    r = lre.wb_multipliers(inp, f, 1000, 0, sums, counts)
    assert r["auto_wb"] and r["scale_mul"].tolist() == [2.0, 1.0, 4.0, 1.0]
    # auto-WB without the sums is refused
    with pytest.raises(lre.LibRawError):
        lre.wb_multipliers(inp, f, 1000, 0)
    # maximum - black is LibRaw's unsigned field: it wraps
    r = lre.wb_multipliers(lre.wb_inputs(pre_mul=(2.0, 1.0, 1.5, 1.0)), f, 100, 200)
    assert r["maximum"] == (100 - 200) % 2**32
