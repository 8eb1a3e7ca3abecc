"""Parity of every develop stage on the GPU against the reference's own CPU
accelerator (oracle/_ref, compiled from the reference sources) and the C
restatement of the LibRaw-dependent pieces (oracle/liblre_oracle.so).

Tolerances: float stages max-abs <= 1e-4 and PSNR >= 90 dB (peak 1.0);
integer stages (black level, quantisation, CFA packing) bit-exact.
Inputs are seeded synthetic scenes (no RAW fixtures exist for this path).
"""
import numpy as np
import pytest

import oracle
from libraw_enhanced_b200 import scenes
from tests._util import amaze_stale_mask, assert_parity, frame_mask, report

pytestmark = pytest.mark.gpu

WB = (2.0, 1.0, 1.5, 1.0)


@pytest.fixture(scope="module")
def acc():
    import libraw_enhanced_b200 as lre

    a = lre.CudaAccelerator(0)
    yield a
    a.close()


@pytest.fixture(scope="module", autouse=True)
def _oracle_threads():
    # fixed thread count: the reference AMaZE / X-Trans read per-thread scratch
    # near image corners / edges, which depends on the tile-to-thread split
    oracle.set_threads(4)


_cache = {}


def bayer_case(h, w, seed, cfa="RGGB"):
    key = ("bayer", h, w, seed, cfa)
    if key not in _cache:
        rgb = scenes.scene_rgb(h, w, seed)
        mos = scenes.mosaic(rgb, cfa, WB, seed)
        sp = scenes.sparse_rgb(mos, cfa)
        _cache[key] = (mos, sp)
    return _cache[key]


def rgb_case(h, w, seed):
    """A demosaiced RGB image (reference AMaZE of a seeded scene)."""
    key = ("rgb", h, w, seed)
    if key not in _cache:
        _, sp = bayer_case(h, w, seed)
        _cache[key] = oracle.amaze(sp, scenes.FILTERS["RGGB"], WB, 1.0)
    return _cache[key]


def corner_mask(h, w, n=32):
    m = np.ones((h, w), bool)
    m[:n, :n] = m[:n, -n:] = m[-n:, :n] = m[-n:, -n:] = False
    return m


# ------------------------------------------------------------------ AMaZE
@pytest.mark.parametrize(
    "h,w,cfa",
    [(1024, 1536, "RGGB"), (384, 512, "BGGR"), (384, 512, "GRBG"), (384, 512, "GBRG"), (203, 301, "RGGB"), (64, 80, "RGGB")],
)
def test_amaze_parity(acc, h, w, cfa):
    """Bit-exact over the whole frame against the reference run one OpenMP
    thread per tile (every tile starts from a zeroed scratch buffer)."""
    _, sp = bayer_case(h, w, 11, cfa)
    f = scenes.FILTERS[cfa]
    ref = oracle.amaze(sp, f, WB, 1.0, fresh_tiles=True)
    gpu = acc.demosaic_bayer_amaze(sp, f, WB, 1.0)
    assert np.array_equal(gpu, ref), report(gpu, ref)
    # for information: the reference under a shared-thread split differs from
    # both only inside the cells whose value is whatever a previous tile left
    shared = oracle.amaze(sp, f, WB, 1.0)
    m = np.repeat(amaze_stale_mask(h, w)[:, :, None], 3, 2)
    assert np.array_equal(gpu[~m], shared[~m])
    print("amaze", cfa, w, h, "vs 4-thread reference in the scratch-dependent cells:", report(gpu, shared, mask=m))


def test_amaze_dense_device_path(acc):
    torch = pytest.importorskip("torch")
    mos, sp = bayer_case(256, 320, 12)
    f = scenes.FILTERS["RGGB"]
    ref = acc.demosaic_bayer_amaze(sp, f, WB, 1.0)
    d_in = torch.from_numpy(mos).cuda()
    d_out = torch.empty((256, 320, 3), device="cuda", dtype=torch.float32)
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    acc.set_stream(s.cuda_stream)
    assert acc.stream == s.cuda_stream
    acc.dev_demosaic_bayer_amaze(d_in, d_out, 320, 256, f, WB, 1.0)
    s.synchronize()
    acc.set_stream(None)
    assert np.array_equal(d_out.cpu().numpy(), ref)


# ------------------------------------------------------------------ X-Trans
@pytest.mark.parametrize("h,w", [(1024, 1536), (240, 360), (131, 211)])
def test_xtrans_3pass_parity(acc, h, w):
    """Whole frame against the reference run one OpenMP thread per tile."""
    rgb = scenes.scene_rgb(h, w, 21)
    mos = scenes.mosaic(rgb, scenes.XTRANS_STD, (1.8, 1.0, 1.6, 1.0), 21)
    sp = scenes.sparse_rgb(mos, scenes.XTRANS_STD)
    ref = oracle.xtrans(sp, scenes.XTRANS_STD, 3, fresh_tiles=True)
    gpu = acc.demosaic_xtrans_3pass(sp, scenes.XTRANS_STD)
    r = assert_parity(gpu, ref, what=f"xtrans3 {w}x{h}")
    m = np.repeat(frame_mask(h, w, 12)[:, :, None], 3, 2)
    print("xtrans3", w, h, r, "12-px frame:", report(gpu, ref, mask=~m))


@pytest.mark.parametrize("h,w", [(1024, 1536), (131, 211)])
def test_xtrans_3pass_rowscan_kernel(acc, monkeypatch, h, w):
    """The row-scan kernel (the fallback for 6x6 patterns whose scans are
    not site-parallel), forced on the X-Trans layout, against the same
    reference run and bit for bit against the plane-resident kernel."""
    rgb = scenes.scene_rgb(h, w, 23)
    mos = scenes.mosaic(rgb, scenes.XTRANS_STD, (1.8, 1.0, 1.6, 1.0), 23)
    sp = scenes.sparse_rgb(mos, scenes.XTRANS_STD)
    ref = oracle.xtrans(sp, scenes.XTRANS_STD, 3, fresh_tiles=True)
    planes = acc.demosaic_xtrans_3pass(sp, scenes.XTRANS_STD)
    monkeypatch.setenv("LRE_XTRANS_ROWSCAN", "1")
    rowscan = acc.demosaic_xtrans_3pass(sp, scenes.XTRANS_STD)
    assert_parity(rowscan, ref, what=f"xtrans3 row-scan {w}x{h}")
    assert np.array_equal(rowscan, planes)


@pytest.mark.parametrize("h,w", [(1024, 1536), (131, 211)])
def test_xtrans_1pass_parity(acc, h, w):
    rgb = scenes.scene_rgb(h, w, 22)
    mos = scenes.mosaic(rgb, scenes.XTRANS_STD, (1.8, 1.0, 1.6, 1.0), 22)
    sp = scenes.sparse_rgb(mos, scenes.XTRANS_STD)
    ref = oracle.xtrans(sp, scenes.XTRANS_STD, 1)
    gpu = acc.demosaic_xtrans_1pass(sp, scenes.XTRANS_STD)
    assert_parity(gpu, ref, what=f"xtrans1 {w}x{h}")


# ------------------------------------------------------------------ post-demosaic
@pytest.mark.parametrize("h,w", [(1024, 1536), (203, 301)])
def test_tone_mapping_parity(acc, h, w):
    img = rgb_case(h, w, 31)
    ref = oracle.tone_mapping(img, 1.0)
    gpu = acc.tone_mapping(img, 1.0)
    assert np.array_equal(gpu, ref), report(gpu, ref)
    assert np.array_equal(acc.tone_mapping(img, 0.8), oracle.tone_mapping(img, 0.8))


@pytest.mark.parametrize("h,w", [(1024, 1536), (203, 301), (40, 37)])
def test_axial_ca_parity(acc, h, w):
    img = rgb_case(h, w, 32)
    ref = oracle.axial_ca(img, 6, 1e-4, 0.3)
    gpu = acc.ca_axial_cleanup(img, 6, 1e-4, 0.3)
    r = assert_parity(gpu, ref, what=f"axial {w}x{h}")
    print("axial", w, h, r)


@pytest.mark.parametrize("radius,eps,strength", [(3, 1e-3, 1.0), (12, 1e-4, 0.5)])
def test_axial_ca_params(acc, radius, eps, strength):
    img = rgb_case(203, 301, 33)
    ref = oracle.axial_ca(img, radius, eps, strength)
    gpu = acc.ca_axial_cleanup(img, radius, eps, strength)
    assert_parity(gpu, ref, what=f"axial r={radius}")


@pytest.mark.parametrize("h,w", [(1024, 1536), (203, 301), (40, 37)])
def test_defringe_parity(acc, h, w):
    img = rgb_case(h, w, 34)
    ref = oracle.defringe(img)
    gpu = acc.defringe(img)
    r = assert_parity(gpu, ref, what=f"defringe {w}x{h}")
    print("defringe", w, h, r, "changed px:", int((np.abs(ref - img) > 0).any(2).sum()))


@pytest.mark.parametrize("green,strength,radius", [(True, 10.0, 10.0), (False, 2.0, 6.0), (True, 4.0, 14.0)])
def test_defringe_params(acc, green, strength, radius):
    img = rgb_case(203, 301, 35)
    ref = oracle.defringe(img, radius=radius, strength=strength, green=green)
    gpu = acc.defringe(img, radius=radius, strength=strength, defringe_green=green)
    assert_parity(gpu, ref, what=f"defringe g={green} s={strength} r={radius}")


@pytest.mark.parametrize("h,w", [(1024, 1536), (203, 301)])
def test_lateral_ca_parity(acc, h, w):
    rgb = scenes.radial_ca(scenes.scene_rgb(h, w, 36), 1.003, 0.997)
    ref = oracle.lateral_ca(rgb)
    gpu = acc.ca_register_lateral(rgb)
    r = assert_parity(gpu, ref, what=f"lateral {w}x{h}")
    print("lateral", w, h, r)


@pytest.mark.parametrize("h,w", [(1024, 1536), (203, 301)])
def test_detail_tonemap_parity(acc, h, w):
    """Against the reference's own detail tone map lines
    (core/libraw_wrapper.cpp:45-116, 1389-1471, compiled into oracle/_ref)."""
    img = rgb_case(h, w, 37)
    ref = oracle.ref_detail_tonemap(img)
    gpu = acc.apply_detail_preserving_tonemap(img)
    assert_parity(gpu, ref, what=f"detail tonemap {w}x{h}")


@pytest.mark.parametrize("use_mask", [False, True])
def test_micro_contrast_parity(acc, use_mask):
    img = rgb_case(203, 301, 38)
    mask = None
    if use_mask:
        mask = np.clip((img.max(axis=2) - 0.5) * 2.0, 0.0, 1.0).astype(np.float32)
    ref = oracle.micro_contrast(img, 0.6, 8.0, 0.04, mask)
    gpu = acc.enhance_micro_contrast(img, 0.6, 8.0, 0.04, mask)
    assert_parity(gpu, ref, what="micro contrast")


# ------------------------------------------------------------------ integer pieces
def test_white_balance_bit_exact(acc):
    rng = np.random.default_rng(5)
    raw4 = rng.integers(0, 16384, size=(67, 93, 4), dtype=np.uint16)
    wb = (2.1, 1.0, 1.7, 1.02)
    for filters, xt in ((scenes.FILTERS["GRBG"], None), (scenes.FILTERS_XTRANS, scenes.XTRANS_STD)):
        base = rng.random((67, 93, 3), dtype=np.float32)
        ref = oracle.white_balance(raw4, wb, filters, xt, out=base.copy())
        gpu = acc.apply_white_balance(raw4, wb, filters, xt, out=base.copy())
        assert np.array_equal(gpu, ref)


def test_black_level_bit_exact(acc):
    rng = np.random.default_rng(6)
    raw4 = rng.integers(0, 16384, size=(41, 53, 4), dtype=np.uint16)
    cases = [
        ([0, 0, 0, 0, 0, 0], 512, 15000),
        ([510, 512, 514, 511, 0, 0], 0, 16000),
        ([10, 12, 14, 11, 2, 2, 100, 101, 102, 103], 0, 16383),
    ]
    for cblack, black, maximum in cases:
        ref = oracle.black_level(raw4, cblack, black, maximum)
        gpu = acc.black_level(raw4, cblack, black, maximum)
        assert np.array_equal(gpu, ref), cblack


def test_quantize_bit_exact(acc):
    rng = np.random.default_rng(7)
    x = (rng.random((33, 47, 3), dtype=np.float32) * 1.4 - 0.2).astype(np.float32)
    x[0, 0] = [0.5 / 65535, 1.0, -0.0]
    assert np.array_equal(acc.quantize(x, 16), oracle.quantize_u16(x))
    assert np.array_equal(acc.quantize(x, 8), oracle.quantize_u8(x))


def test_adjust_maximum(acc):
    _, sp = bayer_case(203, 301, 8)
    f = scenes.FILTERS["RGGB"]
    for thr, dm, mx in ((0.75, 0.0, 2.0), (0.2, 0.0, 1.5), (0.9, 1.7, 2.0), (0.0, 0.0, 2.0)):
        assert acc.adjust_maximum(sp, f, thr, dm, mx) == oracle.adjust_maximum(sp, f, thr, dm, mx)
