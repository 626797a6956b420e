"""The C-ABI library loads and exports every entry point include/xk.h
declares; host-side argument checks work without a GPU."""
import os
import re

import numpy as np
import pytest

import xrt_rs
from xrt_rs import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", fn)).read()
            txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
            names |= set(re.findall(r"\b(xk_[a-z0-9_]+)\s*\(", txt))
    return names


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    declared = _declared()
    assert declared, "no declarations parsed"
    missing = [n for n in sorted(declared) if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_header():
    assert set(_lib.exported_names()) == _declared()


def test_version_and_status_strings():
    lib = _lib.load()
    assert b"sm_100a" in lib.xk_version()
    for code in range(10):
        assert lib.xk_status_string(code)
    assert xrt_rs.route_reason(0) == ""
    assert xrt_rs.route_reason(1) == "no rays"
    assert xrt_rs.route_reason(7) == "non-finite ray or screen values"
    assert xrt_rs.route_reason(8) == "amplitudes outside the FP32 range of the phase-reduced sums"
    assert xrt_rs.route_reason(9) == "unknown"


def test_length_mismatch_raises_value_error():
    # crates/xrt-python/src/lib.rs:31-45: ValueError before any compute.
    with pytest.raises(ValueError, match="array length mismatch"):
        xrt_rs.diffraction_integral_rs([0.0, 1.0], [0.0], [0.0], [0.0], [0.0], [1.0], [1.0],
                                       [1.0], [0.0], [0.0], [0.0], [1e4], [0.0], [0.0], [1.0])
    with pytest.raises(ValueError, match="array length mismatch"):
        xrt_rs.diffraction_integral_rs([0.0], [0.0], [0.0], [0.0], [0.0], [1.0], [1.0], [1.0],
                                       [0.0], [0.0], [0.0], [1e4], [0.0, 1.0], [0.0], [1.0])


def test_unknown_path_rejected():
    with pytest.raises(ValueError):
        xrt_rs.diffraction_integral([[0.0]] * 12, [[0.0], [0.0], [1.0]], path="f16")


def test_no_device_is_an_error_not_a_fallback():
    import ctypes
    lib = _lib.load()
    h = ctypes.c_void_p()
    rc = lib.xk_init(0, ctypes.byref(h))
    if rc == _lib.XK_OK:
        lib.xk_destroy(h)
        pytest.skip("a CUDA device is present")
    assert rc == _lib.XK_ERR_NO_DEVICE
    assert xrt_rs.GpuContext.new() is None
    with pytest.raises(xrt_rs.XkError) as ei:
        xrt_rs.kirchhoff_auto(np.zeros(1, xrt_rs.GPU_RAY_DTYPE), np.zeros(1, xrt_rs.GPU_PIXEL_DTYPE))
    assert ei.value.code == _lib.XK_ERR_NO_DEVICE


def test_gpu_record_layouts_match_reference():
    # GpuRay is 48 bytes, GpuPixel 16 bytes (src/gpu/kirchhoff.rs:20-45).
    import ctypes
    assert xrt_rs.GPU_RAY_DTYPE.itemsize == 48 == ctypes.sizeof(_lib.XkGpuRay)
    assert xrt_rs.GPU_PIXEL_DTYPE.itemsize == 16 == ctypes.sizeof(_lib.XkGpuPixel)
