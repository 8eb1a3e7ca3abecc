"""Batched develop (lre_batch_run / lre_dev_batch_run): many images of uneven
sizes, CFA layouts, WB gains and option sets in one call must give each
image the result the plain per-image path gives it alone.  Kernel-shape
choices (autotuned) may change double-precision summation order inside the
guided filter, so float outputs are compared within 1e-5 and 16-bit outputs
within one code."""
import numpy as np
import pytest

from libraw_enhanced_b200 import scenes

pytestmark = pytest.mark.gpu

SIZES = [(192, 256), (130, 203), (384, 512), (256, 320), (97, 161), (320, 224)]
CFAS = ["RGGB", "BGGR", "GRBG", "GBRG", "RGGB", "GBRG"]


@pytest.fixture(scope="module")
def lre():
    import libraw_enhanced_b200 as m

    return m


@pytest.fixture(scope="module")
def acc(lre):
    a = lre.CudaAccelerator(0)
    yield a
    a.close()


def _workload(lre, bits=16):
    rng = np.random.default_rng(100)
    ms, ps = [], []
    for i, ((h, w), cfa) in enumerate(zip(SIZES, CFAS)):
        wb = (float(rng.uniform(1.5, 2.5)), 1.0, float(rng.uniform(1.2, 2.0)), 1.0)
        ms.append(scenes.bayer_scene(h, w, 100 + i, cfa=cfa, wb=wb))
        ps.append(lre.develop_params(cfa=cfa, cam_mul=wb, defringe=1, axial_ca_correction=1,
                                     tone_mapping=i % 2, stage_order=1, output_bits=bits))
    return ms, ps


def _compare(out, ref):
    if out.dtype == np.uint16:
        d = np.abs(out.astype(np.int32) - ref.astype(np.int32))
        assert d.max() <= 1, d.max()
        assert (d > 0).mean() < 1e-3
    else:
        assert np.abs(out - ref).max() <= 1e-5


def _pinned_like(a):
    import torch

    t = torch.empty(a.nbytes, dtype=torch.uint8).pin_memory()
    return t.numpy().view(a.dtype).reshape(a.shape)


def _pinned_copy(a):
    b = _pinned_like(a)
    b[...] = a
    return b


@pytest.mark.parametrize("use_graph", [False, True])
def test_batch_matches_plain(lre, acc, use_graph):
    ms, ps = _workload(lre)
    b = lre.Batch(0, lanes=0, use_graph=use_graph, autotune=True)
    try:
        # pageable numpy buffers: page-locked for the call, never a graph
        outs = b.run(ms, ps)
        st = b.last_stats
        assert st.launches > 0 and st.lanes >= 1
        assert st.graph == 0
        tune = b.get_tuning()
        acc.set_tuning(tune["axial_strip"], tune["axial_rows"], tune["blur_tile"])
        for m, p, o in zip(ms, ps, outs):
            _compare(o, acc.develop(m, p))
        # page-locked buffers: captured once, then replayed
        pms = [_pinned_copy(m) for m in ms]
        pouts = [_pinned_like(o) for o in outs]
        b.run(pms, ps, outs=pouts)
        assert b.last_stats.graph == (1 if use_graph else 0)
        for a, c in zip(outs, pouts):
            assert np.array_equal(a, c)
        pouts2 = [_pinned_like(o) for o in outs]
        b.run(pms, ps, outs=pouts2)  # new outputs: a new signature
        assert b.last_stats.graph == (1 if use_graph else 0)
        for a in pouts2:
            a[...] = 0
        b.run(pms, ps, outs=pouts2)  # same signature: replay
        assert b.last_stats.graph == (2 if use_graph else 0)
        for a, c in zip(outs, pouts2):
            assert np.array_equal(a, c)
    finally:
        acc.set_tuning()
        b.close()


def test_batch_float_output_and_tuning_choices(lre, acc):
    ms, ps = _workload(lre, bits=32)
    b = lre.Batch(0, lanes=2, use_graph=False, autotune=False)
    try:
        for tune in ({"lanes": 2, "axial_strip": 128, "axial_rows": 128, "blur_tile": 32},
                     {"lanes": 3, "axial_strip": 64, "axial_rows": 64, "blur_tile": 64},
                     {"lanes": 1, "axial_strip": 128, "axial_rows": 64, "blur_tile": 64}):
            b.set_tuning(**tune)
            assert b.get_tuning() == tune
            outs = b.run(ms, ps)
            for m, p, o in zip(ms, ps, outs):
                _compare(o, acc.develop(m, p))
    finally:
        b.close()


def test_dev_batch_run(lre, acc):
    import torch

    ms, ps = _workload(lre)
    dm = [torch.from_numpy(m).cuda() for m in ms]
    do = [torch.empty((m.shape[0], m.shape[1], 3), dtype=torch.int16, device="cuda") for m in ms]
    b = lre.Batch(0, lanes=3, use_graph=True, autotune=False)
    try:
        b.dev_run(dm, do, ps)
        for m, p, o in zip(ms, ps, do):
            got = o.cpu().numpy().view(np.uint16)
            assert np.array_equal(got, acc.develop(m, p))
    finally:
        b.close()


def test_batch_rejects_bad_image(lre):
    ms, ps = _workload(lre)
    ms[2] = np.zeros((16, 16), np.float32)
    b = lre.Batch(0, lanes=2, use_graph=False, autotune=False)
    try:
        with pytest.raises(lre.LibRawError) as ei:
            b.run(ms, ps)
        assert ei.value.status == 1
        assert "image 2" in str(ei.value)
    finally:
        b.close()
