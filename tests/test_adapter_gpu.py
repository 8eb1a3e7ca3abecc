"""The C++ drop-in (csrc/cuda_accelerator.h, the GPUAccelerator method set
over the C ABI) run on the device the way libraw_enhanced's pipeline calls a
GPUAccelerator: host ImageBufferFloat buffers, post-demosaic stages aliased
in == out (core/cpu_accelerator.h:137,167).  The harness
(tests/adapter_harness.cpp) is the build compiled against the reference's own
core/accelerator.h types (oracle/_ref/adapter_harness_ref, made by
`make -C oracle ref`) when present, else compiled here against the adapter's
layout-identical structs.  Outputs are compared with the reference CPU
accelerator: AMaZE bit-exact, defringe and axial CA within max-abs 1e-4."""
import os
import shutil
import subprocess

import numpy as np
import pytest

import oracle
from libraw_enhanced_b200 import scenes
from tests._util import assert_parity

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_HARNESS = os.path.join(ROOT, "oracle", "_ref", "adapter_harness_ref")


def _harness(tmp_path):
    if os.path.exists(REF_HARNESS):
        return REF_HARNESS, "reference types"
    cxx = shutil.which("g++")
    assert cxx, "no C++ compiler to build the adapter harness"
    lib_dir = os.path.join(ROOT, "libraw_enhanced_b200")
    exe = str(tmp_path / "adapter_harness")
    r = subprocess.run([cxx, "-std=c++17", "-O2", "-I", ROOT, os.path.join(ROOT, "tests", "adapter_harness.cpp"),
                        "-o", exe, "-L", lib_dir, "-l:liblre_cuda.so", "-Wl,-rpath," + lib_dir],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe, "layout-identical types"


def test_adapter_runs_pipeline_calls_on_host_buffers(tmp_path):
    h, w = 384, 512
    mos = scenes.bayer_scene(h, w, 41)
    sp = scenes.sparse_rgb(mos, "RGGB")
    raw_path = tmp_path / "raw.f32"
    sp.tofile(raw_path)
    exe, kind = _harness(tmp_path)
    prefix = str(tmp_path / "out_")
    r = subprocess.run([exe, str(raw_path), str(w), str(h), hex(scenes.FILTERS["RGGB"]), prefix],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, (kind, r.returncode, r.stderr)

    def load(name):
        return np.fromfile(prefix + name + ".f32", np.float32).reshape(h, w, 3)

    oracle.set_threads(4)
    ref = oracle.amaze(sp, scenes.FILTERS["RGGB"], (2.0, 1.0, 1.5, 1.0), 1.0, fresh_tiles=True)
    assert np.array_equal(load("amaze"), ref), kind
    ref = oracle.defringe(ref, 10.0, 0.1, 0.15, 10.0, False, 0.3)
    assert_parity(load("defringe"), ref, what=f"adapter defringe ({kind})")
    ref = oracle.axial_ca(ref, 6, 1e-4, 0.3)
    assert_parity(load("axial"), ref, what=f"adapter axial ({kind})")
    # gamma_correct(in, out) with the reference's default arguments
    g = oracle.gamma_correct(load("axial"), 0.0, 0.0, 1)
    d = np.abs(load("gamma").astype(np.float64) - g)
    assert d.max() <= 2 * np.spacing(np.float32(1.0)), d.max()
    print("adapter harness:", kind)
