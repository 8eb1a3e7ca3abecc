"""Host-buffer develop against device-buffer develop, bit for bit.

The host-buffer entry point (lre_develop) overlaps the mosaic upload with
AMaZE and, when the chain ends with the axial guided filter and a pointwise
tone map, runs the filter, the tone map and the download in row bands.  The
device-buffer entry point (lre_dev_develop) runs every stage whole.  Both
must give the same bytes, on ragged sizes whose last band is short, with a
pinned or a pageable destination."""
import numpy as np
import pytest

from libraw_enhanced_b200 import scenes

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


def _device_develop(acc, mos, p):
    import torch

    h, w = mos.shape
    d_in = torch.from_numpy(mos).cuda()
    dt = torch.float32 if p.output_bits == 32 else torch.int16
    d_out = torch.empty((h, w, 3), dtype=dt, device="cuda")
    acc.dev_develop(d_in, d_out, w, h, p)
    acc.synchronize()
    got = d_out.cpu().numpy()
    return got if p.output_bits == 32 else got.view(np.uint16)


@pytest.mark.parametrize("hw", [(517, 1203), (1024, 1536), (33, 40), (300, 64)])
@pytest.mark.parametrize("bits", [32, 16])
def test_banded_tail_matches_device_develop(acc, lre, hw, bits):
    h, w = hw
    mos = scenes.bayer_scene(h, w, 11)
    p = lre.develop_params(cfa="RGGB", cam_mul=WB, defringe=1, axial_ca_correction=1, tone_mapping=1, stage_order=1,
                           output_bits=bits)
    host = acc.develop(mos, p)
    dev = _device_develop(acc, mos, p)
    assert np.array_equal(host, dev)


@pytest.mark.parametrize("algo,tone", [(0, 0), (1, 1), (4, 1), (1, 2)])
def test_banded_tail_other_routes(acc, lre, algo, tone):
    # bilinear and DCB upload before the chain; tone 0 downloads the axial
    # output as is; tone 2 (local, not pointwise) keeps the whole-image tail
    h, w = 389, 611
    mos = (scenes.bayer_scene(h, w, 12) * np.float32(4095.0)).astype(np.float32)
    p = lre.develop_params(cfa="GRBG", cam_mul=WB, maximum_value=4095.0, demosaic_algorithm=algo, defringe=1,
                           axial_ca_correction=1, tone_mapping=tone, stage_order=1)
    assert np.array_equal(acc.develop(mos, p), _device_develop(acc, mos, p))


def test_banded_tail_pinned_destination(acc, lre):
    import torch

    h, w = 700, 900
    mos = scenes.bayer_scene(h, w, 13)
    p = lre.develop_params(cfa="RGGB", cam_mul=WB, defringe=1, axial_ca_correction=1, tone_mapping=1, stage_order=1)
    pinned = torch.empty((h, w, 3), dtype=torch.float32, pin_memory=True)
    out = pinned.numpy()
    acc.develop(mos, p, out=out)
    assert np.array_equal(out, acc.develop(mos, p))
    assert np.array_equal(out, _device_develop(acc, mos, p))
    # a second call into the same pinned buffer after a smaller image
    acc.develop(scenes.bayer_scene(64, 96, 14), p)
    out[:] = 0
    acc.develop(mos, p, out=out)
    assert np.array_equal(out, _device_develop(acc, mos, p))


def _standalone_chain(acc, mos, p, w, h):
    """The 51 MP order as separate device calls, each stage reducing its own
    input maximum (AMaZE -> defringe -> axial CA -> ACES)."""
    import torch

    from libraw_enhanced_b200 import scenes as sc

    d_in = torch.from_numpy(mos).cuda()
    a = torch.empty((h, w, 3), dtype=torch.float32, device="cuda")
    b = torch.empty_like(a)
    acc.dev_demosaic_bayer_amaze(d_in, a, w, h, sc.FILTERS["RGGB"], WB, 1.0)
    if p.defringe:
        acc.dev_defringe(a, a, w, h)
    if p.axial_ca_correction:
        acc.dev_ca_axial_cleanup(a, b, w, h)
        a, b = b, a
    if p.tone_mapping == 1:
        acc.dev_tone_mapping(a, a, w, h, 1.0)
    acc.synchronize()
    return a.cpu().numpy()


@pytest.mark.parametrize("hw", [(517, 1203), (33, 40), (96, 64)])
@pytest.mark.parametrize("defringe", [1, 0])
def test_fused_maxima_match_standalone_stages(acc, lre, hw, defringe):
    """AMaZE and the defringe main pass hand the next stage its input's max G
    (reduced in their own kernels, the 4-px border included); the result must
    equal the stages run one by one, each reducing its own input."""
    h, w = hw
    mos = scenes.bayer_scene(h, w, 15)
    # the brightest samples sit in the border frame, so the border pass's
    # share of the maximum decides it
    mos[:2, :] = np.float32(0.97)
    mos[:, -3:] = np.float32(0.99)
    p = lre.develop_params(cfa="RGGB", cam_mul=WB, defringe=defringe, axial_ca_correction=1, tone_mapping=1,
                           stage_order=1)
    ref = _standalone_chain(acc, mos, p, w, h)
    assert np.array_equal(_device_develop(acc, mos, p), ref)
    assert np.array_equal(acc.develop(mos, p), ref)
