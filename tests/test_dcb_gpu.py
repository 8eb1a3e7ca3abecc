"""DCB Bayer demosaic on the GPU against the reference's own CPU DCB
(core/cpu_accelerator.cpp:1043-1137) run with one OpenMP thread.

The reference's nyquist, pp and last color_full loops are row-parallel
OpenMP loops whose rows read rows the same loop rewrites, so the reference's
result depends on its thread count; the single-thread result is the defined
(sequential) one and the CUDA path must reproduce it bit for bit."""
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


def _raw(h, w, seed, cfa, scale):
    mos = scenes.bayer_scene(h, w, seed, cfa=cfa) * np.float32(scale)
    return mos.astype(np.float32), scenes.sparse_rgb(mos.astype(np.float32), cfa)


@pytest.mark.parametrize("cfa", ["RGGB", "BGGR", "GRBG", "GBRG"])
def test_dcb_bit_exact_defaults(acc, cfa):
    # raw-scale samples (12-bit range) so the refinement's "sample > 1" branch
    # is taken; ragged size
    _, sp = _raw(131, 197, 41, cfa, 4095.0)
    got = acc.demosaic_bayer_dcb(sp, scenes.FILTERS[cfa], 4095.0)
    ref = oracle.bayer_dcb(sp, scenes.FILTERS[cfa], 4095.0, iterations=1, enhance=True, threads=1)
    assert np.array_equal(got, ref)


@pytest.mark.parametrize("iterations,enhance", [(0, False), (0, True), (2, False), (3, True)])
def test_dcb_bit_exact_options(acc, iterations, enhance):
    _, sp = _raw(96, 160, 43, "GRBG", 1000.0)
    f = scenes.FILTERS["GRBG"]
    got = acc.demosaic_bayer_dcb(sp, f, 1000.0, iterations=iterations, dcb_enhance=enhance)
    ref = oracle.bayer_dcb(sp, f, 1000.0, iterations=iterations, enhance=enhance, threads=1)
    assert np.array_equal(got, ref)


def test_dcb_unit_scale_and_clipping(acc):
    # samples in [0, ~1.9] with maximum 1.0: CLIP saturates, the refinement
    # takes its "sample <= 1" branch almost everywhere
    _, sp = _raw(80, 112, 44, "RGGB", 1.0)
    got = acc.demosaic_bayer_dcb(sp, scenes.FILTERS["RGGB"], 1.0)
    ref = oracle.bayer_dcb(sp, scenes.FILTERS["RGGB"], 1.0, threads=1)
    assert np.array_equal(got, ref)


def test_dcb_many_bands_and_columns(acc):
    # several 32-row bands chained through their progress counters and many
    # 128-column ring wraps
    _, sp = _raw(517, 1203, 45, "BGGR", 16383.0)
    got = acc.demosaic_bayer_dcb(sp, scenes.FILTERS["BGGR"], 16383.0)
    ref = oracle.bayer_dcb(sp, scenes.FILTERS["BGGR"], 16383.0, threads=1)
    assert np.array_equal(got, ref)


@pytest.mark.parametrize("hw", [(7, 9), (12, 13), (3, 40)])
def test_dcb_tiny_images(acc, hw):
    h, w = hw
    _, sp = _raw(h, w, 46, "RGGB", 255.0)
    got = acc.demosaic_bayer_dcb(sp, scenes.FILTERS["RGGB"], 255.0)
    ref = oracle.bayer_dcb(sp, scenes.FILTERS["RGGB"], 255.0, threads=1)
    assert np.array_equal(got, ref)


def test_dcb_flat_field(acc):
    # a flat field stays flat through every DCB pass
    sp = scenes.sparse_rgb(np.full((40, 72), 700.0, np.float32), "RGGB")
    got = acc.demosaic_bayer_dcb(sp, scenes.FILTERS["RGGB"], 4095.0)
    assert np.array_equal(got, np.full_like(got, np.float32(700.0) / np.float32(4095.0)))


def test_dcb_device_entry(acc):
    import torch

    mos, sp = _raw(200, 260, 47, "GBRG", 4095.0)
    f = scenes.FILTERS["GBRG"]
    d_in = torch.from_numpy(mos).cuda()
    d_out = torch.empty((200, 260, 3), dtype=torch.float32, device="cuda")
    acc.dev_demosaic_bayer_dcb(d_in, d_out, 260, 200, f, 4095.0)
    ref = oracle.bayer_dcb(sp, f, 4095.0, threads=1)
    assert np.array_equal(d_out.cpu().numpy(), ref)


def test_dcb_rejects_non_bayer(lre, acc):
    _, sp = _raw(64, 64, 48, "RGGB", 1.0)
    # X-Trans marker, all-green word, rows 6/7 laid out unlike rows 0/1
    for bad in (scenes.FILTERS_XTRANS, 0x55555555, 0x61949494):
        with pytest.raises(lre.LibRawError) as ei:
            acc.demosaic_bayer_dcb(sp, bad, 1.0)
        assert ei.value.status == 1
    with pytest.raises(lre.LibRawError):
        acc.demosaic_bayer_dcb(sp, scenes.FILTERS["RGGB"], 1.0, iterations=-1)


def test_sweep_wait_runs_out_and_context_recovers(lre, acc):
    """The in-order sweeps' bounded wait, driven to its limit without any GPU
    fault: host-side injection makes band 0 of the next sweep drop its
    progress reports, so band 1 waits until a short bound (2e7 SM cycles,
    ~10 ms) runs out, raises the error flag and finishes; the call returns
    LRE_ERR_TIMEOUT.  The next call, with the default bound, is bit-exact."""
    _, sp = _raw(128, 96, 45, "RGGB", 4095.0)  # 4 bands of 32 rows
    f = scenes.FILTERS["RGGB"]
    acc.set_wait_limit(20_000_000)
    acc.inject_sweep_stall(0)
    try:
        with pytest.raises(lre.LibRawError) as e:
            acc.demosaic_bayer_dcb(sp, f, 4095.0)
        assert e.value.status == 5  # LRE_ERR_TIMEOUT
    finally:
        acc.set_wait_limit(0)
        acc.inject_sweep_stall(-1)
    got = acc.demosaic_bayer_dcb(sp, f, 4095.0)
    assert np.array_equal(got, oracle.bayer_dcb(sp, f, 4095.0, threads=1))
