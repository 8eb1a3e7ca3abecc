"""The seeded synthetic scene generator is deterministic and produces the
layouts the develop path consumes."""
import numpy as np

from libraw_enhanced_b200 import scenes


def test_scene_deterministic():
    a = scenes.bayer_scene(64, 96, 7)
    b = scenes.bayer_scene(64, 96, 7)
    assert np.array_equal(a, b)
    assert not np.array_equal(a, scenes.bayer_scene(64, 96, 8))
    assert a.dtype == np.float32 and a.shape == (64, 96)


def test_sparse_layout_holds_only_native_channel():
    mos = scenes.bayer_scene(16, 16, 1, cfa="GBRG")
    sp = scenes.sparse_rgb(mos, "GBRG")
    idx = scenes.cfa_map(16, 16, "GBRG")
    ch = np.where(idx == 3, 1, idx)
    assert np.array_equal(np.take_along_axis(sp, ch[:, :, None], 2)[:, :, 0], mos)
    assert int((sp != 0).sum(axis=2).max()) <= 1


def test_xtrans_pattern_counts():
    x = scenes.XTRANS_STD
    assert (x == 1).sum() == 20 and (x == 0).sum() == 8 and (x == 2).sum() == 8


def test_wb_applied_per_site():
    rgb = np.full((4, 4, 3), 0.25, np.float32)
    m = scenes.mosaic(rgb, "RGGB", (2.0, 1.0, 1.5, 1.0), 0, noise=False)
    assert m[0, 0] == 0.5 and m[0, 1] == 0.25 and m[1, 1] == np.float32(0.375)
