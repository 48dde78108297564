"""CPU: libdfft loads and exports every entry point include/dfft.h declares;
argument validation that needs no GPU returns the documented statuses."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADERS = [os.path.join(ROOT, "include", f) for f in sorted(os.listdir(os.path.join(ROOT, "include")))
           if f.endswith(".h")]


def declared_symbols():
    syms = []
    for h in HEADERS:
        txt = open(h).read()
        syms += re.findall(r"DFFT_API\s+[\w\s\*]+?\b(dfft_\w+)\s*\(", txt)
    return sorted(set(syms))


def test_header_declares_entry_points():
    syms = declared_symbols()
    for s in ("dfft_plan_create", "dfft_execute", "dfft_plan_destroy", "dfft_last_error"):
        assert s in syms


def test_library_exports_every_declared_symbol():
    import dfft
    L = dfft.lib()
    missing = [s for s in declared_symbols() if not hasattr(L, s)]
    assert not missing, missing


def test_status_strings_and_version():
    import dfft
    L = dfft.lib()
    assert L.dfft_status_string(2) == b"Unknown transform type"
    assert L.dfft_version().decode().count(".") == 2


def test_unknown_transform_without_gpu():
    import dfft
    from dfft import _lib
    L = dfft.lib()
    h = ctypes.c_void_p()
    shape = _lib.i64_array([4, 4, 4])
    dims = _lib.i32_array([1, 2, 3])
    st = L.dfft_plan_create(ctypes.byref(h), 3, shape, 0, 99, 3, dims, None, 0, 0, 0, 0)
    assert st == _lib.ERROR_UNKNOWN_TRANSFORM
    assert L.dfft_last_error() == b"Unknown transform type"
    st = L.dfft_plan_create(ctypes.byref(h), 4, shape, 0, 0, 3, dims, None, 0, 0, 0, 0)
    assert st == _lib.ERROR_INVALID_VALUE
    st = L.dfft_plan_create(None, 3, shape, 0, 0, 3, dims, None, 0, 0, 0, 0)
    assert st == _lib.ERROR_INVALID_VALUE


def test_python_tags_mirror_reference():
    import dfft
    assert repr(dfft.FFT_()) == "FFT!()"
    assert dfft.Pencil() == dfft.Pencil() and dfft.Pencil() != dfft.Slab()
    with pytest.raises(dfft.ArgumentError, match="Unknown transform type"):
        dfft.R2R((99,))


def _noalloc_status(shape):
    """dfft_irfft_noalloc_f32 with placeholder pointers: every length check
    runs before the device is touched, so a rejected shape returns its
    status here without a GPU (the pointers are never dereferenced)."""
    import dfft
    from dfft import _lib
    L = dfft.lib()
    L.dfft_irfft_noalloc_f32.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                         ctypes.POINTER(ctypes.c_int64), ctypes.c_void_p]
    L.dfft_irfft_noalloc_f32.restype = ctypes.c_int
    return L.dfft_irfft_noalloc_f32(ctypes.c_void_p(256), ctypes.c_void_p(512), len(shape),
                                    _lib.i64_array(shape), None)


@pytest.mark.parametrize("shape", [(2 * 3 ** 17,), (3 ** 17,), (3 ** 18,)])
def test_noalloc_rejects_too_many_stages_without_gpu(shape):
    from dfft import _lib
    import dfft
    assert _noalloc_status(shape) == _lib.ERROR_UNSUPPORTED_SIZE
    assert b"radix stages" in dfft.lib().dfft_last_error()


@pytest.mark.parametrize("shape", [(16, 17, 2), (16, 4, 34), (2 * 17,)])
def test_noalloc_checks_every_axis_before_launch(shape):
    # a prime factor above 13 on any axis (dims 2 and 3 run first) is
    # rejected before the first pass is queued
    from dfft import _lib
    import dfft
    assert _noalloc_status(shape) == _lib.ERROR_UNSUPPORTED_SIZE
    assert b"prime factor above 13" in dfft.lib().dfft_last_error()
