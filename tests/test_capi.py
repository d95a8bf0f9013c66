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


def test_queue_limits_are_refused_before_any_launch(rsx):
    """The queue-driven entry points refuse sizes whose 32-bit queue counter could wrap (a granularity of 2^27 would
    make every claim step 32 x granularity wrap to zero, so the warps would never leave), with a message and before any
    CUDA call: dummy non-null pointers are never touched."""
    L = rsx.lib()
    vp, u32 = ctypes.c_void_p, ctypes.c_uint32
    L.rsx_sim8_persistent_ex.argtypes = [vp, u32, vp, vp, vp, vp, vp, vp, vp, u32, u32, u32, u32, vp, vp]
    L.rsx_sim8_lockstep_raw.argtypes = [vp, u32, vp, vp, vp, vp, vp, vp, vp, u32, u32, u32, vp]
    p = vp(256)
    for n, grid, block, gran in ((1000, 148, 32, 1 << 27), (1000, 148, 32, 257), (1000, 65536, 32, 1), ((1 << 24) + 1, 148, 32, 1)):
        assert L.rsx_sim8_persistent_ex(p, n, p, None, p, p, None, None, p, grid, block, gran, 1, None, None) == -1, (n, grid, gran)
        assert b"wrap" in L.rsx_last_error() or b"granularity" in L.rsx_last_error()
    for n, grid in (((1 << 24) + 1, 148), (1000, 65536)):
        assert L.rsx_sim8_lockstep_raw(p, n, p, None, p, p, None, None, p, grid, 448, 7, None) == -1
        assert b"wrap" in L.rsx_last_error()


@pytest.mark.skipif(gpu_available(), reason="checks the no-device path")
def test_no_device_is_reported(rsx):
    L = rsx.lib()
    h = ctypes.c_void_p()
    assert L.rsx_device_create(0, ctypes.byref(h)) == -3
    assert b"device" in L.rsx_last_error()
