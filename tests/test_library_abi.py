"""The C-ABI library loads and exports every entry point include/otmap_b200.h declares
(no compute: this runs without a GPU)."""

import ctypes
import os
import re

import pytest

from otmap_b200 import build, native

HEADER = os.path.join(build.INCLUDE, "otmap_b200.h")


def declared_symbols():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(otm_[a-z_0-9]+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(native.LIB_PATH):
        build.build_library()
    return native.lib()


def test_header_declares_entry_points():
    syms = declared_symbols()
    assert "otm_solve" in syms and "otm_map_inverse" in syms and "otm_rasterize" in syms


def test_library_exports_every_declared_symbol(lib):
    for s in declared_symbols():
        assert hasattr(lib, s), s
        assert s in native.SIGNATURES, f"{s} has no ctypes signature"


def test_abi_version_and_defaults(lib):
    assert lib.otm_abi_version() == 1
    o = native.default_options()
    assert o.beta == 1 and o.max_iter == 1000 and o.threshold == 1e-7 and o.max_ratio > 1e300


def test_create_without_device_fails_cleanly(lib):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    h = ctypes.c_void_p()
    rc = lib.otm_create(0, ctypes.byref(h))
    assert rc == native.ERR_NO_DEVICE
    assert b"device" in lib.otm_last_error()
