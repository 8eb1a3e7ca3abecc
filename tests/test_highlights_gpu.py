"""Highlight recovery on the GPU against the reference's own code
(core/libraw_wrapper.cpp:1095-1383, compiled from those lines alone into
oracle/_ref/liblre_ref_hl.so): bit-exact image and mask, with and without the
WB-undone chroma edges, across many sweep bands."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lre():
    import libraw_enhanced_b200 as m

    return m


@pytest.fixture(scope="module")
def acc(lre):
    a = lre.CudaAccelerator(0)
    yield a
    a.close()


def highlight_scene(h, w, seed):
    """Smooth colour field with bright blobs: some clipped (white), some
    tinted (purple/magenta rims), some just over the threshold."""
    rng = np.random.default_rng(seed)
    yy, xx = np.mgrid[0:h, 0:w].astype(np.float32)
    img = np.empty((h, w, 3), np.float32)
    for c in range(3):
        img[..., c] = 0.35 + 0.25 * np.sin(xx / (17 + 5 * c) + rng.random() * 6) * np.cos(yy / (23 + 3 * c))
    for _ in range(max(3, h * w // 4000)):
        cy, cx = rng.random() * h, rng.random() * w
        rad = 4 + rng.random() * 20
        amp = 0.5 + rng.random() * 0.9
        tint = np.array([1.0 + 0.4 * rng.random(), 1.0 - 0.3 * rng.random(), 1.0 + 0.4 * rng.random()], np.float32)
        blob = np.exp(-((yy - cy) ** 2 + (xx - cx) ** 2) / (2 * rad * rad)).astype(np.float32)
        img += (amp * blob)[..., None] * tint[None, None, :]
    img += rng.normal(0, 0.003, img.shape).astype(np.float32)
    return np.clip(img, 0.0, 1.6).astype(np.float32)


@pytest.mark.parametrize("wb", [None, (2.1, 1.0, 1.6)])
@pytest.mark.parametrize("thr", [0.9, 0.97])
def test_recover_highlights_bit_exact(acc, wb, thr):
    img = highlight_scene(150, 230, 80)
    got, gmask, gmax = acc.recover_highlights(img, thr, want_mask=True, wb_rgb=wb)
    ref, rmask = oracle.recover_highlights(img, thr, want_mask=True, wb_rgb=wb)
    assert (ref != img).any()  # the scene exercises the recovery
    assert np.array_equal(gmask, rmask)
    assert np.array_equal(got, ref)
    hl = (img[..., 0] >= thr) & (img[..., 2] >= thr)
    assert gmax == img[hl].max()


def test_recover_highlights_many_bands(acc):
    img = highlight_scene(517, 1203, 81)
    got, _, _ = acc.recover_highlights(img, 0.92)
    ref, _ = oracle.recover_highlights(img, 0.92)
    assert np.array_equal(got, ref)


@pytest.mark.parametrize("hw", [(4, 9), (6, 6), (33, 7)])
def test_recover_highlights_tiny(acc, hw):
    img = highlight_scene(*hw, 82) + np.float32(0.4)
    got, _, _ = acc.recover_highlights(img, 0.9)
    ref, _ = oracle.recover_highlights(img, 0.9)
    assert np.array_equal(got, ref)


def test_recover_highlights_none_and_device(acc):
    import torch

    img = np.full((40, 64, 3), 0.3, np.float32)  # nothing reaches the threshold
    got, _, gmax = acc.recover_highlights(img, 0.9)
    assert np.array_equal(got, img) and gmax == 0.0
    img = highlight_scene(200, 260, 83)
    d_in = torch.from_numpy(img).cuda()
    d_out = torch.empty_like(d_in)
    d_mask = torch.empty((200, 260), dtype=torch.float32, device="cuda")
    acc.dev_recover_highlights(d_in, d_out, 260, 200, 0.93, mask=d_mask, wb_rgb=(1.9, 1.0, 1.4))
    ref, rmask = oracle.recover_highlights(img, 0.93, want_mask=True, wb_rgb=(1.9, 1.0, 1.4))
    assert np.array_equal(d_out.cpu().numpy(), ref)
    assert np.array_equal(d_mask.cpu().numpy(), rmask)
    # in place
    acc.dev_recover_highlights(d_in, d_in, 260, 200, 0.93, wb_rgb=(1.9, 1.0, 1.4))
    assert np.array_equal(d_in.cpu().numpy(), ref)
