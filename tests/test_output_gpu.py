"""Output end of the pipeline against the reference's own CPU accelerator:
convert_color_space (bit-exact), gamma_correct (std::pow evaluated in double
and rounded once: within 2 float ulps of glibc's powf) and the fused
colour-space + gamma + to_numpy quantisation epilogue (16/8-bit codes equal
except where the float input sits on a rounding boundary)."""
import numpy as np
import pytest

import oracle
from libraw_enhanced_b200 import scenes

pytestmark = pytest.mark.gpu

XFORM = np.array([[1.65, -0.52, -0.13, 0.0], [-0.18, 1.42, -0.24, 0.0], [0.02, -0.41, 1.39, 0.001]], np.float32)


@pytest.fixture(scope="module")
def lre():
    import libraw_enhanced_b200 as m

    return m


@pytest.fixture(scope="module")
def acc(lre):
    a = lre.CudaAccelerator(0)
    yield a
    a.close()


@pytest.fixture(scope="module")
def img():
    rgb = scenes.scene_rgb(192, 256, 21)
    rgb[0, :8] = [-0.01, 0.0, 1e-8]  # negatives, zeros, tiny values
    rgb[1, :8] = [1.2, 0.0031308, 0.018]  # above 1 and on the encoders' breakpoints
    return np.ascontiguousarray(rgb, np.float32)


def test_convert_color_space_bit_exact(acc, img):
    assert np.array_equal(acc.convert_color_space(img, XFORM), oracle.convert_color_space(img, XFORM))


@pytest.mark.parametrize("cs,gp,gs", [(1, 0, 0), (2, 0, 0), (3, 0, 0), (4, 0, 0), (7, 0, 0), (8, 0, 0),
                                      (0, 2.222, 4.5), (5, 2.4, 0.0), (6, 1.0, 1.0)])
def test_gamma_correct(acc, img, cs, gp, gs):
    got = acc.gamma_correct(img, gp, gs, cs)
    ref = oracle.gamma_correct(img, gp, gs, cs)
    assert np.array_equal(np.isnan(got), np.isnan(ref))
    ok = ~np.isnan(ref)
    d = np.abs(got[ok].astype(np.float64) - ref[ok])
    tol = 2 * np.spacing(np.abs(ref[ok]).astype(np.float32)).astype(np.float64)
    assert (d <= tol).all(), float(d.max())
    assert (got[ok] != ref[ok]).mean() < 0.01


@pytest.mark.parametrize("bits", [16, 8])
def test_fused_epilogue(acc, img, bits):
    got = acc.output_epilogue(img, XFORM, 0.0, 0.0, 1, bits)
    lin = oracle.convert_color_space(img, XFORM)
    enc = oracle.gamma_correct(lin, 0.0, 0.0, 1)
    ref = oracle.quantize_u16(enc) if bits == 16 else oracle.quantize_u8(enc)
    d = np.abs(got.astype(np.int64) - ref.astype(np.int64))
    assert d.max() <= 1
    assert (d > 0).mean() < 1e-3
    # the float form of the epilogue equals the two stages run separately
    f32 = acc.output_epilogue(img, XFORM, 0.0, 0.0, 1, 32)
    assert np.array_equal(f32, acc.gamma_correct(acc.convert_color_space(img, XFORM), 0.0, 0.0, 1))


@pytest.mark.parametrize("cfa", ["RGGB", "BGGR", "GRBG", "GBRG"])
def test_bayer_linear_demosaic_bit_exact(acc, cfa):
    h, w = 130, 197
    mos = scenes.bayer_scene(h, w, 31, cfa=cfa)
    sp = scenes.sparse_rgb(mos, cfa)
    got = acc.demosaic_bayer_linear(sp, scenes.FILTERS[cfa], 1.7)
    ref = oracle.bayer_linear(sp, scenes.FILTERS[cfa], 1.7)
    assert np.array_equal(got, ref)
