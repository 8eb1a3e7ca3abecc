"""The allocation-free axial CA entry point, called through the C ABI.

It exists for callers that cannot allocate device memory mid-frame (pre-
reserved pool hosts, capture threads that must not block in cudaMalloc).
Its output must equal that of the regular entry point, lre_dev_ca_axial_cleanup,
on two calls in a row (the shared scratch is reused across calls), in place
as well as out of place.  This file is named to be collected last.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_ABS = 1e-4  # the float-stage tolerance of every parity test


def _scene(h, w):
    from libraw_enhanced_b200 import scenes

    # a demosaic-like RGB image: smooth scene with per-channel texture
    rgb = scenes.scene_rgb(h, w, 77)
    rng = np.random.default_rng(77)
    rgb = rgb * (1.0 + 0.02 * rng.standard_normal(rgb.shape).astype(np.float32))
    return np.ascontiguousarray(rgb, dtype=np.float32)


def test_noalloc_axial_matches_regular_entry_point():
    torch = pytest.importorskip("torch")
    import libraw_enhanced_b200 as lre
    from libraw_enhanced_b200 import _lib

    lib = _lib.load()
    acc = lre.CudaAccelerator(0)
    h, w = 480, 640
    img = _scene(h, w)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    try:
        acc.set_stream(stream.cuda_stream)
        d_in = torch.from_numpy(img).cuda()
        d_ref = torch.empty_like(d_in)
        acc.dev_ca_axial_cleanup(d_in, d_ref, w, h, 6, 1e-4, 0.3)
        stream.synchronize()
        ref = d_ref.cpu().numpy()

        for call in range(2):
            d_out = torch.full_like(d_in, float("nan"))
            st = lib.lre_dev_ca_axial_cleanup_noalloc(
                C.c_void_p(d_in.data_ptr()), C.c_void_p(d_out.data_ptr()), w, h, 6, 1e-4, 0.3,
                C.c_void_p(stream.cuda_stream),
            )
            assert st == 0, f"call {call}: status {st}"
            stream.synchronize()
            got = d_out.cpu().numpy()
            assert np.isfinite(got).all()
            assert float(np.abs(got - ref).max()) <= MAX_ABS, f"call {call}"

        # in place (input copied into the fixed scratch first)
        d_io = d_in.clone()
        st = lib.lre_dev_ca_axial_cleanup_noalloc(
            C.c_void_p(d_io.data_ptr()), C.c_void_p(d_io.data_ptr()), w, h, 6, 1e-4, 0.3, C.c_void_p(stream.cuda_stream)
        )
        assert st == 0
        stream.synchronize()
        assert float(np.abs(d_io.cpu().numpy() - ref).max()) <= MAX_ABS

        # beyond the fixed scratch size: rejected before any work
        st = lib.lre_dev_ca_axial_cleanup_noalloc(
            C.c_void_p(d_in.data_ptr()), C.c_void_p(d_out.data_ptr()), 2048, 1025, 6, 1e-4, 0.3,
            C.c_void_p(stream.cuda_stream),
        )
        assert st == 1  # LRE_ERR_INVALID_ARGUMENT
    finally:
        torch.cuda.set_stream(torch.cuda.default_stream())
        acc.close()
