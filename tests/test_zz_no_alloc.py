"""The allocation-free axial CA entry point, called through the C ABI.

It exists for callers that cannot allocate device memory mid-frame (hosts
that only lend pre-reserved pools, capture threads that must not block in
cudaMalloc).  Its output must match both the regular entry point,
lre_dev_ca_axial_cleanup, and the reference's own CPU axial CA (oracle/_ref)
within the float-stage tolerance, on two calls in a row (the shared scratch
is reused across calls), in place as well as out of place, for both tile
variants of its kernel (radius <= 8: 32-px tiles; radius > 8: 16-px tiles)
and at exactly its maximum image size.  This file is named to be collected
last.
"""
import ctypes as C

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

MAX_ABS = 1e-4  # the float-stage tolerance of every parity test
MAX_PIXELS = 2048 * 1024  # the entry point's fixed scratch limit


def _scene(h, w):
    from libraw_enhanced_b200 import scenes

    # a demosaic-like RGB image: smooth scene with per-channel texture
    rgb = scenes.scene_rgb(h, w, 77)
    rng = np.random.default_rng(77)
    rgb = rgb * (1.0 + 0.02 * rng.standard_normal(rgb.shape).astype(np.float32))
    return np.ascontiguousarray(rgb, dtype=np.float32)


@pytest.fixture(scope="module")
def env():
    torch = pytest.importorskip("torch")
    import libraw_enhanced_b200 as lre
    from libraw_enhanced_b200 import _lib

    oracle.set_threads(4)
    acc = lre.CudaAccelerator(0)
    stream = torch.cuda.Stream()
    acc.set_stream(stream.cuda_stream)
    yield torch, _lib.load(), acc, stream
    acc.close()


def _noalloc(lib, stream, d_in, d_out, w, h, radius, eps=1e-4, strength=0.3):
    return lib.lre_dev_ca_axial_cleanup_noalloc(
        C.c_void_p(d_in.data_ptr()), C.c_void_p(d_out.data_ptr()), w, h, radius, eps, strength,
        C.c_void_p(stream.cuda_stream),
    )


@pytest.mark.parametrize("h,w,radius", [(480, 640, 6), (301, 203, 12), (256, 384, 16)])
def test_noalloc_axial_matches_regular_entry_point_and_oracle(env, h, w, radius):
    torch, lib, acc, stream = env
    img = _scene(h, w)
    ref = oracle.axial_ca(img, radius, 1e-4, 0.3)
    d_in = torch.from_numpy(img).cuda()
    d_reg = torch.empty_like(d_in)
    acc.dev_ca_axial_cleanup(d_in, d_reg, w, h, radius, 1e-4, 0.3)
    stream.synchronize()
    reg = d_reg.cpu().numpy()
    assert float(np.abs(reg - ref).max()) <= MAX_ABS

    for call in range(2):
        d_out = torch.full_like(d_in, float("nan"))
        assert _noalloc(lib, stream, d_in, d_out, w, h, radius) == 0, f"call {call}"
        stream.synchronize()
        got = d_out.cpu().numpy()
        assert np.isfinite(got).all()
        assert float(np.abs(got - reg).max()) <= MAX_ABS, f"call {call} vs regular entry point"
        assert float(np.abs(got - ref).max()) <= MAX_ABS, f"call {call} vs oracle"

    # in place (the input is copied into the fixed scratch first)
    d_io = d_in.clone()
    assert _noalloc(lib, stream, d_io, d_io, w, h, radius) == 0
    stream.synchronize()
    assert float(np.abs(d_io.cpu().numpy() - ref).max()) <= MAX_ABS


def test_noalloc_axial_in_place_at_maximum_size(env):
    """2048 x 1024 = 2,097,152 px fills the whole scratch copy of the input."""
    torch, lib, acc, stream = env
    h, w = 1024, 2048
    assert h * w == MAX_PIXELS
    img = _scene(h, w)
    ref = oracle.axial_ca(img, 6, 1e-4, 0.3)
    for call in range(2):
        d_io = torch.from_numpy(img).cuda()
        assert _noalloc(lib, stream, d_io, d_io, w, h, 6) == 0, f"call {call}"
        stream.synchronize()
        got = d_io.cpu().numpy()
        assert float(np.abs(got - ref).max()) <= MAX_ABS, f"call {call}"


def test_noalloc_axial_rejects_oversize_before_any_work(env):
    torch, lib, acc, stream = env
    d_in = torch.zeros((8, 8, 3), device="cuda")
    d_out = torch.full_like(d_in, 7.0)
    # one pixel row beyond the limit, and a radius beyond 16
    assert _noalloc(lib, stream, d_in, d_out, 2048, 1025, 6) == 1  # LRE_ERR_INVALID_ARGUMENT
    assert _noalloc(lib, stream, d_in, d_out, 8, 8, 17) == 1
    stream.synchronize()
    assert bool((d_out == 7.0).all())
