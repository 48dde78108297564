"""ctypes binding of libdfft (include/dfft.h).

The shared library is built in-tree (``daggerfft.jl_b200/lib/libdfft.so``).
There is no fallback: if it cannot be loaded, every entry point raises.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.normpath(os.path.join(_HERE, "..", "lib", "libdfft.so"))

# status codes (dfft_status)
SUCCESS = 0
ERROR_INVALID_VALUE = 1
ERROR_UNKNOWN_TRANSFORM = 2
ERROR_UNSUPPORTED_SIZE = 3
ERROR_CUDA = 4
ERROR_OUT_OF_MEMORY = 5
ERROR_NOT_READY = 6
ERROR_TIMEOUT = 7
ERROR_CANCELLED = 8

# transform tags (dfft_transform)
T_FFT, T_IFFT, T_RFFT, T_IRFFT = 0, 1, 2, 3
T_FFT_INPLACE, T_IFFT_INPLACE, T_RFFT_INPLACE, T_IRFFT_INPLACE = 4, 5, 6, 7
T_R2R = 8

F32, F64 = 0, 1
PENCIL, SLAB = 0, 1
PLAIN, MIXED = 0, 1

FLAG_DESTROY_INPUT = 1 << 0
FLAG_TUNE = 1 << 1
FLAG_NO_WISDOM = 1 << 2
FLAG_NO_FUSE = 1 << 3
FLAG_FUSE = 1 << 4


class DFFTError(RuntimeError):
    """A libdfft call failed; ``status`` is the dfft_status code."""

    def __init__(self, status, msg):
        super().__init__(msg)
        self.status = status


class ArgumentError(DFFTError, ValueError):
    """Mirrors Julia's ArgumentError raised by the reference's plan layer."""


_lib = None
_load_error = None


def lib():
    """The loaded library; raises if it is missing (no CPU fallback)."""
    global _lib, _load_error
    if _lib is not None:
        return _lib
    if _load_error is not None:
        raise _load_error
    try:
        L = ctypes.CDLL(LIB_PATH)
    except OSError as e:
        _load_error = DFFTError(ERROR_CUDA, f"libdfft is not built or cannot be loaded ({LIB_PATH}): {e}")
        raise _load_error
    c_int, c_void_p, c_char_p = ctypes.c_int, ctypes.c_void_p, ctypes.c_char_p
    i64p = ctypes.POINTER(ctypes.c_int64)
    i32p = ctypes.POINTER(ctypes.c_int32)
    L.dfft_plan_create.argtypes = [ctypes.POINTER(c_void_p), c_int, i64p, c_int, c_int, c_int, i32p,
                                   i32p, ctypes.c_int64, c_int, c_int, ctypes.c_uint]
    L.dfft_plan_create.restype = c_int
    L.dfft_plan_output_shape.argtypes = [c_void_p, i64p]
    L.dfft_plan_output_shape.restype = c_int
    L.dfft_plan_workspace_bytes.argtypes = [c_void_p, ctypes.POINTER(ctypes.c_size_t)]
    L.dfft_plan_workspace_bytes.restype = c_int
    L.dfft_plan_launches.argtypes = [c_void_p, ctypes.POINTER(c_int)]
    L.dfft_plan_launches.restype = c_int
    L.dfft_plan_describe.argtypes = [c_void_p, ctypes.c_char_p, ctypes.c_size_t]
    L.dfft_plan_describe.restype = c_int
    L.dfft_execute.argtypes = [c_void_p, c_void_p, c_void_p, c_void_p]
    L.dfft_execute.restype = c_int
    L.dfft_plan_destroy.argtypes = [c_void_p]
    L.dfft_plan_destroy.restype = c_int
    L.dfft_device_error.argtypes = [ctypes.POINTER(c_int)]
    L.dfft_device_error.restype = c_int
    for nm in ("dfft_wisdom_export", "dfft_wisdom_import"):
        getattr(L, nm).argtypes = [c_char_p]
        getattr(L, nm).restype = c_int
    L.dfft_wisdom_forget.argtypes = []
    L.dfft_wisdom_forget.restype = c_int
    L.dfft_wisdom_size.argtypes = [ctypes.POINTER(c_int)]
    L.dfft_wisdom_size.restype = c_int
    L.dfft_last_error.argtypes = []
    L.dfft_last_error.restype = c_char_p
    L.dfft_status_string.argtypes = [c_int]
    L.dfft_status_string.restype = c_char_p
    L.dfft_version.argtypes = []
    L.dfft_version.restype = c_char_p
    _lib = L
    return L


def check(status):
    if status == SUCCESS:
        return
    L = lib()
    msg = L.dfft_last_error().decode() or L.dfft_status_string(status).decode()
    if status == ERROR_UNKNOWN_TRANSFORM:
        raise ArgumentError(status, msg)
    if status in (ERROR_INVALID_VALUE, ERROR_UNSUPPORTED_SIZE):
        raise ArgumentError(status, msg)
    raise DFFTError(status, msg)


def i64_array(vals):
    return (ctypes.c_int64 * len(vals))(*[int(v) for v in vals])


def i32_array(vals):
    return (ctypes.c_int32 * max(1, len(vals)))(*[int(v) for v in vals])


def device_error():
    """Reads and clears the device error word (0 = no kernel gave up a wait)."""
    v = ctypes.c_int()
    check(lib().dfft_device_error(ctypes.byref(v)))
    return v.value


def wisdom_export(path):
    """Writes the tuning cache (FFTW-wisdom analogue) to ``path``."""
    check(lib().dfft_wisdom_export(str(path).encode()))


def wisdom_import(path):
    """Merges a tuning cache written by ``wisdom_export``."""
    check(lib().dfft_wisdom_import(str(path).encode()))


def wisdom_forget():
    check(lib().dfft_wisdom_forget())


def wisdom_size():
    v = ctypes.c_int()
    check(lib().dfft_wisdom_size(ctypes.byref(v)))
    return v.value
