"""AAHD Bayer demosaic on the GPU against the reference's own CPU AAHD
(core/cpu_accelerator.cpp:617-633) run with one OpenMP thread.

The reference's hide_hots and refine_hv_dirs rewrite in place inside
row-parallel OpenMP loops, and its channel min/max scan is an unsynchronised
parallel loop, so its multi-threaded result depends on timing; the
single-thread (sequential) result is the defined one and the CUDA path must
reproduce it bit for bit."""
import numpy as np
import pytest

import oracle
from libraw_enhanced_b200 import scenes

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


def _mosaic(h, w, seed, cfa, scale):
    return (scenes.bayer_scene(h, w, seed, cfa=cfa) * np.float32(scale)).astype(np.float32)


def _check(acc, mos, cfa, maximum):
    sp = scenes.sparse_rgb(mos, cfa)
    f = scenes.FILTERS[cfa]
    got = acc.demosaic_bayer_aahd(sp, f, maximum)
    ref = oracle.bayer_aahd(sp, f, maximum, threads=1)
    assert np.array_equal(got, ref)


@pytest.mark.parametrize("cfa", ["RGGB", "BGGR", "GRBG", "GBRG"])
def test_aahd_bit_exact(acc, cfa):
    _check(acc, _mosaic(131, 197, 51, cfa, 4095.0), cfa, 4095.0)


def test_aahd_hot_and_dead_sites_in_order(acc):
    mos = _mosaic(96, 160, 52, "RGGB", 2000.0)
    mos[20, 30] = 60000.0  # isolated hot R site
    mos[41, 61] = 0.25     # isolated dead B site
    # a hot pair on one row: the right one only tests hot after the left one
    # has been replaced, which is what the in-order pass must reproduce
    mos[60, 40] = 60000.0
    mos[60, 42] = 30000.0
    mos[70, 80] = 65000.0  # two hot sites shielding each other
    mos[70, 82] = 65000.0
    _check(acc, mos, "RGGB", 65535.0)


def test_aahd_many_bands(acc):
    mos = _mosaic(517, 1203, 53, "GBRG", 16383.0)
    rng = np.random.default_rng(7)
    for r, c in rng.integers(8, (509, 1195), size=(40, 2)):
        mos[r, c] = 16000.0 if rng.random() < 0.5 else 0.5
    _check(acc, mos, "GBRG", 16383.0)


@pytest.mark.parametrize("hw", [(9, 11), (16, 5), (3, 33)])
def test_aahd_tiny_images(acc, hw):
    h, w = hw
    _check(acc, _mosaic(h, w, 54, "GRBG", 255.0), "GRBG", 255.0)


def test_aahd_device_entry(acc):
    import torch

    mos = _mosaic(200, 260, 55, "BGGR", 4095.0)
    f = scenes.FILTERS["BGGR"]
    d_in = torch.from_numpy(mos).cuda()
    d_out = torch.empty((200, 260, 3), dtype=torch.float32, device="cuda")
    acc.dev_demosaic_bayer_aahd(d_in, d_out, 260, 200, f, 4095.0)
    ref = oracle.bayer_aahd(scenes.sparse_rgb(mos, "BGGR"), f, 4095.0, threads=1)
    assert np.array_equal(d_out.cpu().numpy(), ref)


def test_aahd_rejects_non_bayer(lre, acc):
    sp = scenes.sparse_rgb(_mosaic(64, 64, 56, "RGGB", 100.0), "RGGB")
    for bad in (scenes.FILTERS_XTRANS, 0x55555555, 0x61949494):
        with pytest.raises(lre.LibRawError) as ei:
            acc.demosaic_bayer_aahd(sp, bad, 100.0)
        assert ei.value.status == 1
