"""The develop chain routes ProcessingParams::demosaic_algorithm as
Accelerator::demosaic_compute does (core/accelerator.cpp:90-129): Bayer 0 ->
bilinear, 4 -> DCB (1 iteration, enhanced), 12 -> AAHD, anything else ->
AMaZE.  A develop with every later stage off must equal the standalone
demosaic; with stages on, the plain, batched (graph-captured) and served
paths must agree."""
import numpy as np
import pytest

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


@pytest.mark.parametrize("algo", [0, 4, 12, 10, 1])
def test_develop_demosaic_only_matches_standalone(lre, acc, algo):
    h, w = 160, 224
    mos = (scenes.bayer_scene(h, w, 61, cfa="GRBG") * np.float32(4095.0)).astype(np.float32)
    f = scenes.FILTERS["GRBG"]
    p = lre.develop_params(cfa="GRBG", maximum_value=4095.0, cam_mul=(2.0, 1.0, 1.5, 1.0), demosaic_algorithm=algo)
    got = acc.develop(mos, p)
    sp = scenes.sparse_rgb(mos, "GRBG")
    if algo == 0:
        ref = acc.demosaic_bayer_linear(sp, f, 4095.0)
    elif algo == 4:
        ref = acc.demosaic_bayer_dcb(sp, f, 4095.0, iterations=1, dcb_enhance=True)
    elif algo == 12:
        ref = acc.demosaic_bayer_aahd(sp, f, 4095.0)
    else:
        ref = acc.demosaic_bayer_amaze(sp, f, (2.0, 1.0, 1.5, 1.0), 4095.0)
    assert np.array_equal(got, ref)


def test_develop_algorithms_batched_and_served(lre, acc):
    ms, ps = [], []
    for i, algo in enumerate([4, 12, 0, 10, 12, 4]):
        h, w = 128 + 16 * i, 192 - 8 * i
        cfa = ["RGGB", "BGGR", "GBRG", "GRBG", "RGGB", "GBRG"][i]
        ms.append((scenes.bayer_scene(h, w, 70 + i, cfa=cfa) * np.float32(4095.0)).astype(np.float32))
        ps.append(lre.develop_params(cfa=cfa, maximum_value=4095.0, demosaic_algorithm=algo, defringe=1,
                                     axial_ca_correction=1, stage_order=1, output_bits=16))
    refs = [acc.develop(m, p) for m, p in zip(ms, ps)]

    import torch

    def pinned(a):
        t = torch.empty(a.nbytes, dtype=torch.uint8).pin_memory()
        v = t.numpy().view(a.dtype).reshape(a.shape)
        v[...] = a
        return v

    b = lre.Batch(0, lanes=3, use_graph=True, autotune=False)
    try:
        pms = [pinned(m) for m in ms]
        outs = [pinned(np.zeros_like(r)) for r in refs]
        b.run(pms, ps, outs=outs)
        assert b.last_stats.graph == 1
        for o, r in zip(outs, refs):
            assert np.array_equal(o, r)
    finally:
        b.close()
    srv = lre.Server(0, lanes=2)
    try:
        tickets = [srv.submit(m, p) for m, p in zip(ms, ps)]
        for t, r in zip(tickets, refs):
            o, _ = srv.wait(t)
            assert np.array_equal(o, r)
    finally:
        srv.close()


def test_develop_dcb_aahd_need_2x2_bayer(lre, acc):
    mos = np.ones((64, 64), np.float32)
    for algo in (4, 12):
        p = lre.develop_params(demosaic_algorithm=algo)
        p.filters = 0x61949494
        with pytest.raises(lre.LibRawError) as ei:
            acc.develop(mos, p)
        assert ei.value.status == 1


@pytest.mark.parametrize("algo", [10, 4])
def test_develop_highlight_recovery_matches_standalone(lre, acc, algo):
    # recover_highlights right after the demosaic, as the pipeline runs it
    h, w = 150, 210
    mos = scenes.bayer_scene(h, w, 64, cfa="RGGB")
    p = lre.develop_params(cfa="RGGB", cam_mul=(2.0, 1.0, 1.5, 1.0), demosaic_algorithm=algo,
                           highlight_recovery=1, highlight_threshold=0.9)
    got = acc.develop(mos, p)
    sp = scenes.sparse_rgb(mos, "RGGB")
    f = scenes.FILTERS["RGGB"]
    dem = (acc.demosaic_bayer_dcb(sp, f, 1.0) if algo == 4
           else acc.demosaic_bayer_amaze(sp, f, (2.0, 1.0, 1.5, 1.0), 1.0))
    ref, _, _ = acc.recover_highlights(dem, 0.9)
    assert not np.array_equal(ref, dem)
    assert np.array_equal(got, ref)
