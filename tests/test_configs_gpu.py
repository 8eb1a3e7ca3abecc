"""Parity at the exact benchmarked workloads, against the reference's own CPU
accelerator (oracle/_ref), on the very inputs bench.py times:

* the 51 MP fringed Bayer develop (8736x5856 RGGB, seed 2):
  AMaZE -> defringe(10, 0.1, 0.15, 10, green off, 0.3) -> axial CA
  (r 6, eps 1e-4, strength 0.3) -> ACES tone map (after_scale 1.0)
  (core/cpu_accelerator.cpp:1145-1653, 3939-5064, 3799-3928, 3034-3068);
* the 6240x4160 X-Trans scene with radial lateral CA (R x1.0008,
  B x0.9992), 3-pass demosaic -> pyramidal LK (cell 96, 3 levels,
  3 iterations, max shift 6, min confidence 0.02)
  (core/cpu_accelerator.cpp:1870-2676, 3496-3673);
* the 32-image batched set: one image of each Bayer layout, through
  lre_batch_run, AMaZE -> defringe -> axial CA, float and 16-bit output.

Each stage is checked on the reference's own input for that stage and the
whole chain end to end.  Tolerances: max-abs <= 1e-4 and PSNR >= 90 dB for
float stages (peak 1.0), bit-exact for AMaZE and the ACES curve; 16-bit
output within 7 codes (1e-4 of 65535 is 6.55 codes).

The reference's AMaZE and X-Trans read tile scratch that is allocated once
per OpenMP thread; the oracle runs them one thread per tile
(``fresh_tiles=True``) so that every tile starts from a zeroed buffer, which
is the CUDA path's semantics.  The comparison is then over the whole frame.
"""
import numpy as np
import pytest

import oracle
from libraw_enhanced_b200 import scenes
from tests._util import assert_parity, report

pytestmark = pytest.mark.gpu

WB = (2.0, 1.0, 1.5, 1.0)
RGGB = scenes.FILTERS["RGGB"]


@pytest.fixture(scope="module")
def lre():
    import libraw_enhanced_b200 as m

    return m


@pytest.fixture(scope="module")
def acc(lre):
    a = lre.CudaAccelerator(0)
    yield a
    a.close()


@pytest.fixture(scope="module", autouse=True)
def _oracle_threads():
    import os

    oracle.set_threads(os.cpu_count() or 4)


def _u16_close(out16, ref_f32):
    ref16 = oracle.quantize_u16(ref_f32)
    d = np.abs(out16.astype(np.int64) - ref16.astype(np.int64))
    assert d.max() <= 7, d.max()
    return int(d.max()), float((d > 0).mean())


def test_bayer_51mp_fringed_develop(acc, lre):
    h, w = 5856, 8736
    mos = scenes.bayer_51mp_fringed(2, h, w)  # the bench input
    sp = scenes.sparse_rgb(mos, "RGGB")

    ref_dm = oracle.amaze(sp, RGGB, WB, 1.0, fresh_tiles=True)
    gpu_dm = acc.demosaic_bayer_amaze(sp, RGGB, WB, 1.0)
    assert np.array_equal(gpu_dm, ref_dm), report(gpu_dm, ref_dm)
    del sp, gpu_dm

    ref_df = oracle.defringe(ref_dm, 10.0, 0.1, 0.15, 10.0, False, 0.3)
    gpu_df = acc.defringe(ref_dm)
    changed = float((ref_df != ref_dm).any(axis=2).mean())
    r_df = assert_parity(gpu_df, ref_df, what="defringe 51 MP")
    del gpu_df

    ref_ax = oracle.axial_ca(ref_df, 6, 1e-4, 0.3)
    gpu_ax = acc.ca_axial_cleanup(ref_df, 6, 1e-4, 0.3)
    r_ax = assert_parity(gpu_ax, ref_ax, what="axial 51 MP")
    del gpu_ax, ref_df

    ref = oracle.tone_mapping(ref_ax, 1.0)
    assert np.array_equal(acc.tone_mapping(ref_ax, 1.0), ref)
    del ref_ax

    p = lre.develop_params(cfa="RGGB", cam_mul=WB, defringe=1, axial_ca_correction=1, tone_mapping=1,
                           tone_after_scale=1.0, stage_order=1)
    out = acc.develop(mos, p)
    r_e2e = assert_parity(out, ref, what="51 MP develop end to end")
    p.output_bits = 16
    u16 = _u16_close(acc.develop(mos, p), ref)
    print(f"51 MP fringed: defringe changed {changed:.3%} of pixels; defringe {r_df}; axial {r_ax}; "
          f"end to end {r_e2e}; u16 max code diff / fraction {u16}")


def test_xtrans_26mp_lateral_ca(acc, lre):
    h, w = 4160, 6240
    d = scenes.xtrans_lateral_ca_torch(3, h, w)  # the bench input (generated on the GPU)
    mos = d.cpu().numpy()
    del d
    xt = scenes.XTRANS_STD
    sp = scenes.sparse_rgb(mos, xt)

    ref_dm = oracle.xtrans(sp, xt, 3, fresh_tiles=True)
    gpu_dm = acc.demosaic_xtrans_3pass(sp, xt)
    r_dm = assert_parity(gpu_dm, ref_dm, what="X-Trans 3-pass 26 MP")
    del sp, gpu_dm

    ref = oracle.lateral_ca(ref_dm, 96, 3, 6.0, 0.02, 3)
    gpu_lk = acc.ca_register_lateral(ref_dm, 96, 3, 6.0, 0.02, 3)
    r_lk = assert_parity(gpu_lk, ref, what="lateral CA 26 MP")
    moved = float((ref != ref_dm).any(axis=2).mean())
    del gpu_lk, ref_dm

    p = lre.develop_params(cfa=xt, cam_mul=(1.8, 1.0, 1.6, 1.0), xtrans_passes=3, lateral_ca_correction=1,
                           lateral_ca_cell_size=96, lateral_ca_pyramid_levels=3, lateral_ca_max_iterations=3,
                           lateral_ca_max_shift=6.0, lateral_ca_min_confidence=0.02)
    out = acc.develop(mos, p)
    r_e2e = assert_parity(out, ref, what="X-Trans develop end to end")
    print(f"X-Trans 26 MP: 3-pass {r_dm}; lateral CA moved {moved:.3%} of pixels, {r_lk}; end to end {r_e2e}")


def test_batch_one_image_per_cfa(lre):
    """One image of each Bayer layout from the 32-image batched set (seeds
    100..131, the bench's draws of size, CFA and WB), developed together in
    one lre_batch_run call and compared with the reference chain."""
    first = {}
    for spec in scenes.batch_specs(32, 100):
        first.setdefault(spec[3], spec)
    specs = [first[c] for c in ("RGGB", "BGGR", "GRBG", "GBRG")]
    mos = []
    for seed, h, w, cfa, wb in specs:
        d = scenes.mosaic_upscaled_torch(seed, h, w, cfa, wb)  # the bench input
        mos.append(d.cpu().numpy())
        del d
    p32 = [lre.develop_params(cfa=cfa, cam_mul=wb, defringe=1, axial_ca_correction=1, stage_order=1,
                              output_bits=32) for _, _, _, cfa, wb in specs]
    p16 = [lre.develop_params(cfa=cfa, cam_mul=wb, defringe=1, axial_ca_correction=1, stage_order=1,
                              output_bits=16) for _, _, _, cfa, wb in specs]
    b = lre.Batch(0, lanes=0, use_graph=True, autotune=True)
    try:
        outs32 = b.run(mos, p32)
        outs16 = b.run(mos, p16)
    finally:
        b.close()
    for (seed, h, w, cfa, wb), m, o32, o16 in zip(specs, mos, outs32, outs16):
        sp = scenes.sparse_rgb(m, cfa)
        ref = oracle.amaze(sp, scenes.FILTERS[cfa], wb, 1.0, fresh_tiles=True)
        ref = oracle.defringe(ref)
        ref = oracle.axial_ca(ref, 6, 1e-4, 0.3)
        r = assert_parity(o32, ref, what=f"batch {cfa} {w}x{h}")
        u16 = _u16_close(o16, ref)
        print(f"batch {cfa} {w}x{h} seed {seed}: {r}; u16 max code diff / fraction {u16}")
