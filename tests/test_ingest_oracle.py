"""Known-answer checks of the oracle's raw-ingest restatements (raw2image,
green matching) on hand-built frames, CPU only."""
import numpy as np

import oracle

RGGB = 0x94949494
RGGB_G2 = 0xB4B4B4B4  # the same layout with the second green coded as colour 3


def test_raw2image_margins_pitch_and_channels():
    raw = np.arange(10 * 16, dtype=np.uint16).reshape(10, 16)  # raw_pitch 32 bytes, raw_width 12
    img = oracle.raw2image(raw, 32, 1, 2, 8, 6, RGGB)
    assert img.shape == (6, 8, 4)
    # sample (row, col) comes from raw[row + 1, col + 2] and lands in its colour
    assert list(img[0, 0]) == [raw[1, 2], 0, 0, 0]
    assert list(img[0, 1]) == [0, raw[1, 3], 0, 0]
    assert list(img[1, 0]) == [0, raw[2, 2], 0, 0]
    assert list(img[1, 1]) == [0, 0, raw[2, 3], 0]
    # a colour-3 second green is also copied into channel 1
    g2 = oracle.raw2image(raw, 32, 1, 2, 8, 6, RGGB_G2)
    assert list(g2[1, 0]) == [0, raw[2, 2], 0, raw[2, 2]]


def test_raw2image_half_size_keeps_last_sample():
    raw = np.arange(8 * 8, dtype=np.uint16).reshape(8, 8)
    img = oracle.raw2image(raw, 16, 0, 0, 8, 8, RGGB, shrink=1)
    assert img.shape == (4, 4, 4)
    # R (0,0); G (0,1) then overwritten by G (1,0); B (1,1)
    assert list(img[0, 0]) == [raw[0, 0], raw[1, 0], raw[1, 1], 0]


def test_raw2image_xtrans_rows_are_raw_width_apart():
    from libraw_enhanced_b200 import scenes

    raw = np.arange(9 * 12, dtype=np.uint16).reshape(9, 12)
    img = oracle.raw2image(raw, 0, 1, 1, 10, 7, 9, scenes.XTRANS_STD)
    for row in range(7):
        for col in range(10):
            c = scenes.XTRANS_STD[row % 6, col % 6]
            assert img[row, col, c] == raw[row + 1, col + 1]
            assert int(img[row, col].sum()) == int(raw[row + 1, col + 1])


def test_green_matching_flat_patch():
    h, w, maximum = 12, 12, 4000
    img = np.zeros((h, w, 4), np.uint16)
    # G1 = 1000 at colour-1 sites, G2 = 800 at colour-3 sites of RGGB_G2
    for r in range(h):
        for c in range(w):
            f = (RGGB_G2 >> ((((r << 1) & 14) | (c & 1)) << 1)) & 3
            if f == 1:
                img[r, c, 1] = 1000
            elif f == 3:
                img[r, c, 3] = 800
                img[r, c, 1] = 800
    out = oracle.green_matching(img, RGGB_G2, maximum)
    # flat neighbourhoods: G2 at (3..8 odd rows, 2..8 even cols) scaled by 1000/800
    assert out[3, 2, 3] == 1000 and out[5, 4, 3] == 1000
    # outside the candidate range nothing changes
    assert out[1, 0, 3] == 800 and out[11, 10, 3] == 800
    # a textured G1 neighbourhood (spread above 1% of maximum) is left alone
    img2 = img.copy()
    img2[4, 5, 1] = 1100
    out2 = oracle.green_matching(img2, RGGB_G2, maximum)
    assert out2[5, 4, 3] == 800 and out2[3, 4, 3] == 800
    # X-Trans frames are untouched
    assert np.array_equal(oracle.green_matching(img, 9, maximum), img)
