"""CPU checks of the C ABI library: it loads without a GPU and exports every
entry point include/lre_cuda.h declares (no compute call is made here)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "lre_cuda.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"^[A-Za-z_][\w\s\*]*?\b(lre_\w+)\s*\(", src, flags=re.M)
    return sorted(set(names))


def test_header_declares_entry_points():
    names = declared_functions()
    for must in ("lre_create", "lre_destroy", "lre_defringe", "lre_ca_axial_cleanup", "lre_demosaic_bayer_amaze",
                 "lre_develop", "lre_dev_develop", "lre_tone_mapping"):
        assert must in names


def test_library_exports_every_declared_symbol():
    from libraw_enhanced_b200 import _lib

    if not os.path.exists(_lib.LIB_PATH):
        pytest.skip("liblre_cuda.so not built")
    lib = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing
    # the Python binding declares a signature for every header entry point
    assert set(declared_functions()) <= set(_lib.SIGNATURES), set(declared_functions()) - set(_lib.SIGNATURES)


def test_loader_binds_without_gpu():
    from libraw_enhanced_b200 import _lib

    if not os.path.exists(_lib.LIB_PATH):
        pytest.skip("liblre_cuda.so not built")
    lib = _lib.load()
    assert lib.lre_abi_version() == 1
    # no device here: creation must fail cleanly, not crash or fall back
    import torch

    if not torch.cuda.is_available():
        h = ctypes.c_void_p()
        assert lib.lre_create(0, ctypes.byref(h)) == 4  # LRE_ERR_NO_DEVICE
        assert lib.lre_is_available() == 0
