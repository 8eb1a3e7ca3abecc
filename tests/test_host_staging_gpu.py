"""Host-buffer entry points with pageable (ordinary numpy) buffers, the way
the reference's pipeline passes its std::vector-backed ImageBufferFloat.
Above a few MB those copies go through the context's pinned chunk ring with
a parallel host memcpy (csrc/host_stage.cu); results must be the same bytes
as with page-locked buffers and as the device-buffer entry points, for
sizes that span several ring chunks and end in a partial chunk."""
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


def _pinned_like(a):
    import torch

    t = torch.empty(a.nbytes, dtype=torch.uint8).pin_memory()
    return t.numpy().view(a.dtype).reshape(a.shape)


@pytest.mark.parametrize("bits", [32, 16])
def test_develop_pageable_matches_pinned_and_device(lre, acc, bits):
    import torch

    h, w = 2101, 3007  # 25 MB mosaic, 76 MB f32 RGB: several 16 MB chunks plus a partial one
    mos = scenes.mosaic_upscaled_torch(7, h, w, "RGGB", WB).cpu().numpy()
    p = lre.develop_params(cfa="RGGB", cam_mul=WB, defringe=1, axial_ca_correction=1, tone_mapping=1,
                           stage_order=1, output_bits=bits)
    pageable = acc.develop(np.array(mos, copy=True), p)
    pm = _pinned_like(mos)
    pm[...] = mos
    po = _pinned_like(pageable)
    acc.develop(pm, p, out=po)
    d_out = torch.empty((h, w, 3), dtype=torch.float32 if bits == 32 else torch.int16, device="cuda")
    acc.dev_develop(torch.from_numpy(mos).cuda(), d_out, w, h, p)
    acc.synchronize()
    dev = d_out.cpu().numpy().view(pageable.dtype)
    assert np.array_equal(pageable, po)
    assert np.array_equal(pageable, dev)


def test_stage_pageable_matches_device(lre, acc):
    import torch

    h, w = 1500, 2300  # 41 MB of RGB each way
    img = np.random.default_rng(8).random((h, w, 3), dtype=np.float32)
    out = acc.defringe(img)
    d_in = torch.from_numpy(img).cuda()
    d_out = torch.empty_like(d_in)
    acc.dev_defringe(d_in, d_out, w, h)
    acc.synchronize()
    assert np.array_equal(out, d_out.cpu().numpy())
    # reusing the same context and ring for a second, differently sized call
    img2 = img[: h - 77].copy()
    out2 = acc.tone_mapping(img2, 0.9)
    d2 = torch.from_numpy(img2).cuda()
    d2o = torch.empty_like(d2)
    acc.dev_tone_mapping(d2, d2o, w, h - 77, 0.9)
    acc.synchronize()
    assert np.array_equal(out2, d2o.cpu().numpy())
