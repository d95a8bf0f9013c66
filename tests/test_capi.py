"""The C ABI: the library loads without a GPU, exports every entry point include/rsx.h declares, and rejects bad
arguments with RSX_E_ARG (no CUDA call is needed for that)."""
import ctypes
import os
import re

import pytest

from conftest import ROOT, gpu_available


def declared_symbols():
    with open(os.path.join(ROOT, "include", "rsx.h")) as f:
        src = f.read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(rsx_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol(rsx):
    L = rsx.lib()
    names = declared_symbols()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_bad_arguments_are_rejected(rsx):
    L = rsx.lib()
    assert L.rsx_sim8_raw(None, 10, None, None, None, 32, None, None) == -1
    assert L.rsx_build_static(None, 1, 0, 0) == -1
    assert L.rsx_device_destroy(None) == -1
    assert L.rsx_static_upload(None, None, 1, None) == -1


@pytest.mark.skipif(gpu_available(), reason="checks the no-device path")
def test_no_device_is_reported(rsx):
    L = rsx.lib()
    h = ctypes.c_void_p()
    assert L.rsx_device_create(0, ctypes.byref(h)) == -3
    assert b"device" in L.rsx_last_error()
