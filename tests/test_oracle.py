"""CPU tests of the oracle itself: the C restatement against the compiled
reference, both against the committed golden vectors, and known answers for
the integer pieces.  No GPU is used here."""
import os

import numpy as np
import pytest

import oracle
from libraw_enhanced_b200 import scenes

GOLD = os.path.join(os.path.dirname(__file__), "golden", "develop_golden.npz")
WB = (2.0, 1.0, 1.5, 1.0)

needs_ref = pytest.mark.skipif(not oracle.ref_available(), reason="oracle/_ref not built (make -C oracle)")


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLD)


def test_fcol_matches_scene_generator():
    for name, f in scenes.FILTERS.items():
        for r in range(4):
            for c in range(4):
                assert oracle.port().port_fcol_bayer_native(r, c, f) == scenes.fcol_bayer_native(r, c, f)
    # RGGB word decodes to R at (0,0), B at (1,1)
    f = scenes.FILTERS["RGGB"]
    assert [oracle.port().port_fcol_bayer(r, c, f) for r in (0, 1) for c in (0, 1)] == [0, 1, 1, 2]


def test_quantize_known_answers():
    x = np.array([-1.0, 0.0, 0.5 / 65535, 1.0 / 65535, 0.5, 1.0, 2.0], np.float32)
    assert oracle.quantize_u16(x).tolist() == [0, 0, 1, 1, 32768, 65535, 65535]
    assert oracle.quantize_u8(x).tolist() == [0, 0, 0, 0, 128, 255, 255]


def test_black_level_known_answers():
    raw4 = np.array([[[100, 200, 300, 400], [5, 6, 7, 8]]], np.uint16)
    out = oracle.black_level(raw4, [0, 0, 0, 0, 0, 0], 50, 300)
    assert out.tolist() == [[[50, 150, 250, 300], [0, 0, 0, 0]]]
    out = oracle.black_level(raw4, [10, 20, 30, 40, 0, 0], 0, 1000)
    assert out.tolist() == [[[90, 180, 270, 360], [0, 0, 0, 0]]]
    out = oracle.black_level(raw4, [0, 0, 0, 0, 1, 2, 5, 7], 0, 1000)
    assert out.tolist() == [[[95, 195, 295, 395], [0, 0, 0, 1]]]


def test_scale_mul_and_auto_wb():
    assert oracle.scale_mul([2.0, 1.0, 1.5, 0.0], 3, 1.0).tolist() == [2.0, 1.0, 1.5, 1.0]
    raw4 = np.zeros((2, 2, 4), np.uint16)
    raw4[0, 0, 0] = 100
    raw4[0, 1, 1] = 200
    raw4[1, 0, 1] = 200  # 0x94949494 codes both greens as colour 1
    raw4[1, 1, 2] = 50
    pm = oracle.auto_wb(raw4, scenes.FILTERS["RGGB"])
    assert pm.tolist() == [2.0, 1.0, 4.0, 1.0]


@needs_ref
def test_port_tone_mapping_matches_reference():
    img = np.random.default_rng(0).random((37, 53, 3), dtype=np.float32) * 1.5
    assert np.array_equal(oracle.port_tone_mapping(img, 0.9), oracle.tone_mapping(img, 0.9))


@needs_ref
def test_port_white_balance_matches_reference():
    rng = np.random.default_rng(1)
    raw4 = rng.integers(0, 65535, size=(29, 31, 4), dtype=np.uint16)
    for f, xt in ((scenes.FILTERS["BGGR"], None), (scenes.FILTERS_XTRANS, scenes.XTRANS_STD)):
        base = rng.random((29, 31, 3), dtype=np.float32)
        a = oracle.white_balance(raw4, (1.9, 1.0, 1.3, 1.05), f, xt, out=base.copy())
        b = oracle.port_white_balance(raw4, (1.9, 1.0, 1.3, 1.05), f, xt, out=base.copy())
        assert np.array_equal(a, b)


@needs_ref
def test_port_border_interpolate_matches_reference_amaze_frame():
    # the reference AMaZE ends with border_interpolate(4): applying the
    # restated border fill to its output must be a no-op on the 4-px frame
    mos = scenes.bayer_scene(64, 80, 5)
    sp = scenes.sparse_rgb(mos, "RGGB")
    out = oracle.amaze(sp, scenes.FILTERS["RGGB"], WB, 1.0)
    again = oracle.border_interpolate(out, scenes.FILTERS["RGGB"], 4)
    assert np.array_equal(out, again)


@needs_ref
@pytest.mark.parametrize(
    "key,fn",
    [
        ("amaze_rggb", lambda g: oracle.amaze(scenes.sparse_rgb(g["bayer_mosaic"], "RGGB"), scenes.FILTERS["RGGB"], WB, 1.0)),
        ("defringe", lambda g: oracle.defringe(g["amaze_rggb"])),
        ("defringe_green_s4", lambda g: oracle.defringe(g["amaze_rggb"], strength=4.0, green=True)),
        ("axial", lambda g: oracle.axial_ca(g["amaze_rggb"])),
        ("tone", lambda g: oracle.tone_mapping(g["amaze_rggb"], 1.0)),
        ("micro", lambda g: oracle.micro_contrast(g["amaze_rggb"], 0.6, 8.0, 0.04)),
        ("lateral", lambda g: oracle.lateral_ca(g["lateral_in"], cell=32)),
        ("xtrans3", lambda g: oracle.xtrans(scenes.sparse_rgb(g["xtrans_mosaic"], scenes.XTRANS_STD), scenes.XTRANS_STD, 3)),
        ("xtrans1", lambda g: oracle.xtrans(scenes.sparse_rgb(g["xtrans_mosaic"], scenes.XTRANS_STD), scenes.XTRANS_STD, 1)),
        ("wb_grbg", lambda g: oracle.white_balance(g["raw4"], (2.1, 1.0, 1.7, 1.02), scenes.FILTERS["GRBG"])),
    ],
)
def test_reference_build_reproduces_golden(gold, key, fn):
    oracle.set_threads(4)
    got = fn(gold)
    assert np.array_equal(got, gold[key]), key


needs_ref_dt = pytest.mark.skipif(not os.path.exists(oracle.REF_DT_SO), reason="oracle/_ref not built (make -C oracle)")


@needs_ref_dt
def test_detail_tonemap_reference_lines_reproduce_golden(gold):
    """The golden `detail` vector is written by the reference's own lines
    (core/libraw_wrapper.cpp:45-116, :1389-1471 compiled into
    oracle/_ref/liblre_ref_dt.so); rebuilding them reproduces it."""
    assert np.array_equal(oracle.ref_detail_tonemap(gold["amaze_rggb"]), gold["detail"])


@needs_ref_dt
@pytest.mark.parametrize("threads", [1, 3, 8])
def test_detail_tonemap_restatement_matches_reference_lines(threads):
    """The C restatement of the detail tone map equals the reference's own
    compiled lines bit for bit, at several OpenMP thread counts (the
    reference's sliding box sums run per row / per column, so its result does
    not depend on the thread split)."""
    img = np.random.default_rng(40).random((83, 131, 3), dtype=np.float32) * np.float32(1.3)
    oracle.set_threads(threads)
    try:
        assert np.array_equal(oracle.detail_tonemap(img), oracle.ref_detail_tonemap(img))
    finally:
        oracle.set_threads(4)


def test_restatement_reproduces_golden(gold):
    assert np.array_equal(oracle.detail_tonemap(gold["amaze_rggb"]), gold["detail"])
    assert np.array_equal(oracle.quantize_u16(gold["tone"]), gold["u16"])
    assert np.array_equal(oracle.port_tone_mapping(gold["amaze_rggb"], 1.0), gold["tone"])
    assert np.array_equal(
        oracle.black_level(gold["raw4"], [10, 12, 14, 11, 2, 2, 100, 101, 102, 103], 0, 16383), gold["black_pos"]
    )
    assert np.array_equal(oracle.black_level(gold["raw4"], [510, 512, 514, 511, 0, 0], 0, 16000), gold["black_chan"])
    assert np.array_equal(oracle.port_white_balance(gold["raw4"], (2.1, 1.0, 1.7, 1.02), scenes.FILTERS["GRBG"]), gold["wb_grbg"])


def test_reference_dcb_flat_field_and_thread_dependence():
    """The reference DCB (core/cpu_accelerator.cpp:1043-1137) keeps a flat
    field flat; single-threaded it is deterministic.  (With several OpenMP
    threads its in-place row-parallel passes read rows other threads are
    rewriting, which is why parity is taken against one thread.)"""
    import numpy as np
    from libraw_enhanced_b200 import scenes

    if not oracle.ref_available():
        pytest.skip("reference not built")
    f = scenes.FILTERS["RGGB"]
    flat = scenes.sparse_rgb(np.full((40, 72), 700.0, np.float32), "RGGB")
    out = oracle.bayer_dcb(flat, f, 4095.0)
    assert np.array_equal(out, np.full_like(out, np.float32(700.0) / np.float32(4095.0)))
    sp = scenes.sparse_rgb(scenes.bayer_scene(64, 96, 3) * np.float32(4095.0), "RGGB")
    a = oracle.bayer_dcb(sp, f, 4095.0, threads=1)
    b = oracle.bayer_dcb(sp, f, 4095.0, threads=1)
    assert np.array_equal(a, b) and np.isfinite(a).all()


@needs_ref
def test_reference_amaze_depends_on_thread_split_only_in_stale_cells():
    """The reference AMaZE is not a function of its input near image corners:
    its tile scratch is allocated once per OpenMP thread
    (core/cpu_accelerator.cpp:1217-1218) and the apron corners of tiles that
    touch two image edges are never filled (:1326).  Between thread splits
    the output moves inside tests._util.amaze_stale_mask and nowhere else;
    with one thread per tile (every tile starts from a zeroed buffer, the
    semantics the CUDA path implements) the result is reproducible."""
    from tests._util import amaze_stale_mask

    h, w = 1024, 1536
    sp = scenes.sparse_rgb(scenes.bayer_scene(h, w, 1), "RGGB")
    f = scenes.FILTERS["RGGB"]
    saved = oracle.num_threads()
    try:
        outs = {}
        for t in (1, 9, oracle.amaze_tiles(h, w)):
            oracle.set_threads(t)
            outs[t] = oracle.amaze(sp, f, WB, 1.0)
        fresh = oracle.amaze(sp, f, WB, 1.0, fresh_tiles=True)
    finally:
        oracle.set_threads(saved)
    stale = amaze_stale_mask(h, w)
    assert np.array_equal(fresh, outs[oracle.amaze_tiles(h, w)])
    moved_anywhere = False
    for t in (1, 9):
        d = np.abs(outs[t] - fresh).max(axis=2)
        assert d[~stale].max() == 0.0, t
        moved_anywhere |= bool(d[stale].max() > 0)
    assert moved_anywhere  # the thread split does change the stale cells


@needs_ref
def test_reference_xtrans_depends_on_thread_split_only_in_frame():
    """The reference X-Trans 3-pass reads per-thread tile buffers
    (core/cpu_accelerator.cpp:1953-1959) in cells its edge tiles never write,
    so the thread split moves the output within 12 px of the image edge and
    nowhere else; one thread per tile makes it reproducible."""
    h, w = 240, 360
    rgb = scenes.scene_rgb(h, w, 21)
    sp = scenes.sparse_rgb(scenes.mosaic(rgb, scenes.XTRANS_STD, (1.8, 1.0, 1.6, 1.0), 21), scenes.XTRANS_STD)
    saved = oracle.num_threads()
    try:
        outs = {}
        for t in (1, 4):
            oracle.set_threads(t)
            outs[t] = oracle.xtrans(sp, scenes.XTRANS_STD, 3)
        fresh = oracle.xtrans(sp, scenes.XTRANS_STD, 3, fresh_tiles=True)
        fresh2 = oracle.xtrans(sp, scenes.XTRANS_STD, 3, fresh_tiles=True)
    finally:
        oracle.set_threads(saved)
    assert np.array_equal(fresh, fresh2)
    inner = np.zeros((h, w), bool)
    inner[12:-12, 12:-12] = True
    moved = False
    for t in (1, 4):
        d = np.abs(outs[t] - fresh).max(axis=2)
        assert d[inner].max() == 0.0, t
        moved |= bool(d[~inner].max() > 0)
    assert moved
