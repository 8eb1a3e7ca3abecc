"""Generate the golden vectors in tests/golden/ from the reference itself.

    make -C oracle && python tests/golden/make_golden.py

Every output is produced by uniuyuni/libraw_enhanced's own code: its CPU
accelerator (compiled from the reference sources into
oracle/_ref/liblre_ref.so), its detail-preserving tone map (the reference's
own lines compiled into oracle/_ref/liblre_ref_dt.so) or, for the
LibRaw-dependent integer pieces, the oracle's C restatement.  Inputs are small
seeded synthetic scenes and are stored beside the outputs, so the fixtures do
not depend on the scene generator staying unchanged.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from libraw_enhanced_b200 import scenes  # noqa: E402

WB = (2.0, 1.0, 1.5, 1.0)


def main():
    oracle.set_threads(4)
    out = {}
    h, w = 96, 128
    mos = scenes.bayer_scene(h, w, 101)
    sp = scenes.sparse_rgb(mos, "RGGB")
    out["bayer_mosaic"] = mos
    out["amaze_rggb"] = oracle.amaze(sp, scenes.FILTERS["RGGB"], WB, 1.0)
    rgb = out["amaze_rggb"]
    out["defringe"] = oracle.defringe(rgb)
    out["defringe_green_s4"] = oracle.defringe(rgb, strength=4.0, green=True)
    out["axial"] = oracle.axial_ca(rgb)
    out["tone"] = oracle.tone_mapping(rgb, 1.0)
    out["detail"] = oracle.ref_detail_tonemap(rgb)
    out["micro"] = oracle.micro_contrast(rgb, 0.6, 8.0, 0.04)
    lat_in = scenes.radial_ca(scenes.scene_rgb(h, w, 102), 1.004, 0.996)
    out["lateral_in"] = lat_in
    out["lateral"] = oracle.lateral_ca(lat_in, cell=32)
    xm = scenes.mosaic(scenes.scene_rgb(h, w, 103), scenes.XTRANS_STD, (1.8, 1.0, 1.6, 1.0), 103)
    xs = scenes.sparse_rgb(xm, scenes.XTRANS_STD)
    out["xtrans_mosaic"] = xm
    out["xtrans3"] = oracle.xtrans(xs, scenes.XTRANS_STD, 3)
    out["xtrans1"] = oracle.xtrans(xs, scenes.XTRANS_STD, 1)
    out["u16"] = oracle.quantize_u16(out["tone"])
    rng = np.random.default_rng(104)
    raw4 = rng.integers(0, 16384, size=(24, 30, 4), dtype=np.uint16)
    out["raw4"] = raw4
    out["black_pos"] = oracle.black_level(raw4, [10, 12, 14, 11, 2, 2, 100, 101, 102, 103], 0, 16383)
    out["black_chan"] = oracle.black_level(raw4, [510, 512, 514, 511, 0, 0], 0, 16000)
    out["wb_grbg"] = oracle.white_balance(raw4, (2.1, 1.0, 1.7, 1.02), scenes.FILTERS["GRBG"])
    path = os.path.join(HERE, "develop_golden.npz")
    np.savez_compressed(path, **out)
    print(path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
