"""End-to-end develop on the GPU against the oracle chain of the same stages,
plus the failure paths of the C ABI (host-side fault injection; no GPU fault
is ever provoked)."""
import numpy as np
import pytest

import oracle
from libraw_enhanced_b200 import scenes
from tests._util import amaze_stale_mask, assert_parity, dilate, report

pytestmark = pytest.mark.gpu

WB = (2.0, 1.0, 1.5, 1.0)


@pytest.fixture(scope="module")
def lre():
    import libraw_enhanced_b200 as m

    return m


@pytest.fixture(scope="module")
def acc(lre):
    a = lre.CudaAccelerator(0)
    yield a
    a.close()


@pytest.fixture(scope="module", autouse=True)
def _oracle_threads():
    oracle.set_threads(4)


def _corner_mask3(h, w):
    return np.ones((h, w, 3), bool)


def test_develop_51mp_chain_order_small(acc, lre):
    """The 51 MP workload's chain (AMaZE -> defringe -> axial -> ACES) on the
    1536x1024 seeded scene, float and 16-bit outputs."""
    h, w = 1024, 1536
    mos = scenes.bayer_scene(h, w, 1)
    sp = scenes.sparse_rgb(mos, "RGGB")
    ref_dm = oracle.amaze(sp, scenes.FILTERS["RGGB"], WB, 1.0, fresh_tiles=True)
    ours_dm = acc.demosaic_bayer_amaze(sp, scenes.FILTERS["RGGB"], WB, 1.0)
    # one reference thread per tile: every tile starts from a zeroed buffer,
    # and AMaZE is bit-exact over the whole frame
    assert np.array_equal(ours_dm, ref_dm)
    ref = oracle.defringe(ref_dm)
    ref = oracle.axial_ca(ref, 6, 1e-4, 0.3)
    ref = oracle.tone_mapping(ref, 1.0)
    p = lre.develop_params(cfa="RGGB", cam_mul=WB, defringe=1, axial_ca_correction=1, tone_mapping=1, stage_order=1)
    out = acc.develop(mos, p)
    r = assert_parity(out, ref, mask=_corner_mask3(h, w), what="develop chain")
    print("develop", r)
    p.output_bits = 16
    out16 = acc.develop(mos, p)
    ref16 = oracle.quantize_u16(ref)
    d = np.abs(out16.astype(np.int64) - ref16.astype(np.int64))
    m = _corner_mask3(h, w)
    # 1e-4 on [0,1] is 6.55 counts of 65535: quantising after a <=1e-4 float
    # difference moves a code by at most 7
    assert d[m].max() <= 7
    assert np.array_equal(out16, acc.quantize(out, 16))


def test_develop_reference_order_xtrans(acc, lre):
    """Reference stage order on X-Trans: 3-pass -> lateral CA -> axial -> defringe."""
    h, w = 600, 900
    rgb = scenes.radial_ca(scenes.scene_rgb(h, w, 3), 1.002, 0.998)
    xw = (1.8, 1.0, 1.6, 1.0)
    mos = scenes.mosaic(rgb, scenes.XTRANS_STD, xw, 3)
    sp = scenes.sparse_rgb(mos, scenes.XTRANS_STD)
    ref_dm = oracle.xtrans(sp, scenes.XTRANS_STD, 3, fresh_tiles=True)
    ours_dm = acc.demosaic_xtrans_3pass(sp, scenes.XTRANS_STD)
    assert_parity(ours_dm, ref_dm, what="xtrans3")
    ref = oracle.lateral_ca(ref_dm)
    ref = oracle.axial_ca(ref)
    ref = oracle.defringe(ref)
    p = lre.develop_params(cfa=scenes.XTRANS_STD, lateral_ca_correction=1, axial_ca_correction=1, defringe=1)
    out = acc.develop(mos, p)
    r = assert_parity(out, ref, what="develop xtrans")
    print("develop xtrans", r)


def test_in_place_alias_matches_out_of_place(acc):
    torch = pytest.importorskip("torch")
    img = oracle.amaze(scenes.sparse_rgb(scenes.bayer_scene(192, 256, 4), "RGGB"), scenes.FILTERS["RGGB"], WB, 1.0)
    t = torch.from_numpy(img).cuda()
    for name, kw in (("dev_ca_axial_cleanup", {}), ("dev_defringe", {}), ("dev_ca_register_lateral", {}),
                     ("dev_detail_tonemap", {}), ("dev_tone_mapping", {})):
        out = torch.empty_like(t)
        getattr(acc, name)(t, out, 256, 192, **kw)
        same = t.clone()
        getattr(acc, name)(same, same, 256, 192, **kw)
        acc.synchronize()
        assert torch.equal(out, same), name


def test_invalid_arguments_raise(acc, lre):
    with pytest.raises(ValueError):
        acc.tone_mapping(np.zeros((4, 4), np.float32))
    with pytest.raises(lre.LibRawError) as e:
        acc.ca_axial_cleanup(np.zeros((16, 16, 3), np.float32), radius=40)
    assert e.value.status == 1
    with pytest.raises(lre.LibRawError):
        acc.demosaic_bayer_amaze(np.zeros((16, 16, 3), np.float32), 9, WB)
    with pytest.raises(ValueError):
        lre.defringe(np.zeros((8, 8, 4), np.float32))


def test_host_fault_injection_leaves_context_usable(acc, lre):
    img = np.random.default_rng(3).random((64, 64, 3), dtype=np.float32)
    acc.inject_fault(1)
    with pytest.raises(lre.LibRawError) as e:
        acc.tone_mapping(img)
    assert e.value.status == 6
    # the next call runs normally
    assert np.array_equal(acc.tone_mapping(img), oracle.tone_mapping(img))


def test_launch_counter_counts_own_kernels(acc):
    img = np.random.default_rng(4).random((64, 64, 3), dtype=np.float32)
    n0 = acc.launch_count
    acc.tone_mapping(img)
    assert acc.launch_count - n0 == 1
    acc.defringe(img)
    # init + max G + prep, blur with the support seed fused, blur of the
    # seed, line-link, blur of the solo seeds, main pass
    assert acc.launch_count - n0 == 1 + 8


def test_defringe_unaligned_views_match(acc):
    """The defringe main pass reads and writes four pixels per float4 when
    the RGB buffers are 16-byte aligned and falls back to one pixel per step
    otherwise (and for the last W*H % 4 pixels); both forms must agree."""
    torch = pytest.importorskip("torch")
    h, w = 203, 301  # W*H % 4 == 3: the scalar tail runs too
    img = torch.from_numpy(oracle.amaze(scenes.sparse_rgb(scenes.bayer_scene(h, w, 5), "RGGB"),
                                        scenes.FILTERS["RGGB"], WB, 1.0)).cuda()
    aligned = torch.empty_like(img)
    acc.dev_defringe(img, aligned, w, h)
    src_buf = torch.empty(h * w * 3 + 1, device="cuda")
    dst_buf = torch.empty(h * w * 3 + 1, device="cuda")
    src = src_buf[1:].view(h, w, 3)  # 4-byte offset: not 16-byte aligned
    dst = dst_buf[1:].view(h, w, 3)
    src.copy_(img)
    acc.synchronize()
    torch.cuda.synchronize()
    acc.dev_defringe(src, dst, w, h)
    acc.synchronize()
    assert torch.equal(dst, aligned)
