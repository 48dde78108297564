"""Python client of libdfft's serving runtime (``dfft_server_*``).

The server runs inside libdfft (a C++ dispatcher thread): requests are
admitted in arrival order while an execution slot is free and their staging
memory fits the HBM arena, run concurrently on their own streams, and are
timestamped on completion (p50/p99 latency in ``stats()``).

Arrays follow the same conventions as ``dfft.fft``: torch tensors indexed
like the Julia arrays they stand for, C- or Fortran-ordered; CUDA tensors are
read in place, pinned CPU tensors are copied in by the server.
"""
from __future__ import annotations

import ctypes
from typing import Optional

import torch

from . import _lib
from ._lib import ArgumentError, check
from .api import R2R, Pencil, Transform, _norm_dims, _order, _precision

MEM_DEVICE, MEM_HOST, MEM_SERVER = 0, 1, 2


class _Request(ctypes.Structure):
    _fields_ = [("transform", ctypes.c_int), ("precision", ctypes.c_int), ("decomp", ctypes.c_int),
                ("ndim", ctypes.c_int), ("shape", ctypes.c_int64 * 3), ("ndims", ctypes.c_int),
                ("dims", ctypes.c_int32 * 3), ("r2r_kinds", ctypes.c_int32 * 3),
                ("irfft_len", ctypes.c_int64), ("in_", ctypes.c_void_p), ("in_location", ctypes.c_int),
                ("out", ctypes.c_void_p), ("out_location", ctypes.c_int)]


class _Stats(ctypes.Structure):
    _fields_ = [("completed", ctypes.c_uint64), ("rejected", ctypes.c_uint64),
                ("cancelled", ctypes.c_uint64), ("failed", ctypes.c_uint64), ("queued", ctypes.c_uint64),
                ("p50_ms", ctypes.c_double), ("p99_ms", ctypes.c_double), ("max_ms", ctypes.c_double),
                ("bytes_moved", ctypes.c_double), ("elapsed_s", ctypes.c_double),
                ("arena_bytes", ctypes.c_size_t), ("arena_peak_bytes", ctypes.c_size_t),
                ("peak_running", ctypes.c_int), ("resident_plans", ctypes.c_int)]


_BOUND = False


def _bind(L):
    global _BOUND
    if _BOUND:
        return
    vp, ci = ctypes.c_void_p, ctypes.c_int
    L.dfft_server_create.argtypes = [ctypes.POINTER(vp), ctypes.c_size_t, ci, ctypes.c_uint]
    L.dfft_server_submit.argtypes = [vp, ctypes.POINTER(_Request), ctypes.POINTER(ctypes.c_uint64)]
    L.dfft_server_poll.argtypes = [vp, ctypes.POINTER(ctypes.c_uint64), ci, ctypes.POINTER(ci)]
    L.dfft_server_wait.argtypes = [vp, ctypes.c_uint64, ci, ctypes.POINTER(ci)]
    L.dfft_server_fetch.argtypes = [vp, ctypes.c_uint64, vp, ci, vp]
    L.dfft_server_result_pointer.argtypes = [vp, ctypes.c_uint64, ctypes.POINTER(vp)]
    L.dfft_server_release.argtypes = [vp, ctypes.c_uint64]
    L.dfft_server_cancel.argtypes = [vp, ctypes.c_uint64]
    L.dfft_server_get_stats.argtypes = [vp, ctypes.POINTER(_Stats)]
    L.dfft_server_reset_stats.argtypes = [vp]
    L.dfft_server_destroy.argtypes = [vp]
    for nm in ("dfft_server_create", "dfft_server_submit", "dfft_server_poll", "dfft_server_wait",
               "dfft_server_fetch", "dfft_server_result_pointer", "dfft_server_release",
               "dfft_server_cancel", "dfft_server_get_stats", "dfft_server_reset_stats",
               "dfft_server_destroy"):
        getattr(L, nm).restype = ci
    _BOUND = True


class Server:
    """A serving instance on the current device with an HBM arena of
    ``hbm_budget_bytes`` and ``slots`` concurrently running requests."""

    def __init__(self, hbm_budget_bytes: int, slots: int = 8, tune: bool = False):
        L = _lib.lib()
        _bind(L)
        self._L = L
        h = ctypes.c_void_p()
        check(L.dfft_server_create(ctypes.byref(h), int(hbm_budget_bytes), int(slots),
                                   _lib.FLAG_TUNE if tune else 0))
        self._h = h
        self._keep = {}

    def submit(self, transform: Transform, A: torch.Tensor, dims=(1, 2, 3), n=None, decomp=None,
               out: Optional[torch.Tensor] = None) -> int:
        """Queues ``transform`` of ``A`` over ``dims``; with ``out`` None the
        result stays in the server's arena (``fetch`` it, then ``release``)."""
        if not isinstance(transform, Transform):
            raise ArgumentError(_lib.ERROR_UNKNOWN_TRANSFORM, "Unknown transform type")
        o = _order(A)
        if o == "X":
            raise ArgumentError(_lib.ERROR_INVALID_VALUE, "array must be contiguous")
        nd = A.dim()
        dims = _norm_dims(dims, nd)
        shape = tuple(A.shape)
        if o == "C":
            shape = tuple(reversed(shape))
            dims = tuple(nd + 1 - d for d in dims)
        r = _Request()
        r.transform = transform.code
        r.precision = _precision(A.dtype)
        r.decomp = (decomp or Pencil()).code
        r.ndim = nd
        for i in range(3):
            r.shape[i] = shape[i] if i < nd else 1
        r.ndims = len(dims)
        kinds = transform.kinds if isinstance(transform, R2R) else ()
        if isinstance(transform, R2R) and len(kinds) == 1:
            kinds = kinds * len(dims)
        for i in range(3):
            r.dims[i] = dims[i] if i < len(dims) else 0
            r.r2r_kinds[i] = kinds[i] if i < len(kinds) else 0
        r.irfft_len = int(n) if n is not None else 0
        r.in_ = A.data_ptr()
        r.in_location = MEM_DEVICE if A.is_cuda else MEM_HOST
        if out is None:
            r.out = None
            r.out_location = MEM_SERVER
        else:
            if out.dim() > 1 and _order(out) != o:
                raise ArgumentError(_lib.ERROR_INVALID_VALUE, "output must have the input's memory order")
            r.out = out.data_ptr()
            r.out_location = MEM_DEVICE if out.is_cuda else MEM_HOST
        rid = ctypes.c_uint64()
        check(self._L.dfft_server_submit(self._h, ctypes.byref(r), ctypes.byref(rid)))
        self._keep[rid.value] = (A, out)  # inputs/outputs must stay alive until done
        return rid.value

    def poll(self, max_ids: int = 4096):
        """Ids of finished requests (completed, failed or cancelled)."""
        buf = (ctypes.c_uint64 * max_ids)()
        n = ctypes.c_int()
        check(self._L.dfft_server_poll(self._h, buf, max_ids, ctypes.byref(n)))
        return [buf[i] for i in range(n.value)]

    def wait(self, rid: int, timeout_ms: int = 10000) -> int:
        """Bounded wait; returns the request's status (0 = success)."""
        st = ctypes.c_int()
        check(self._L.dfft_server_wait(self._h, rid, int(timeout_ms), ctypes.byref(st)))
        return st.value

    def fetch(self, rid: int, dst: torch.Tensor, stream=None):
        s = stream or torch.cuda.current_stream()
        check(self._L.dfft_server_fetch(self._h, rid, ctypes.c_void_p(dst.data_ptr()),
                                        MEM_DEVICE if dst.is_cuda else MEM_HOST,
                                        ctypes.c_void_p(s.cuda_stream)))
        return dst

    def release(self, rid: int):
        check(self._L.dfft_server_release(self._h, rid))
        self._keep.pop(rid, None)

    def cancel(self, rid: int):
        check(self._L.dfft_server_cancel(self._h, rid))

    def stats(self) -> dict:
        s = _Stats()
        check(self._L.dfft_server_get_stats(self._h, ctypes.byref(s)))
        return {f: getattr(s, f) for f, _ in _Stats._fields_}

    def reset_stats(self):
        check(self._L.dfft_server_reset_stats(self._h))

    def close(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            self._L.dfft_server_destroy(h)
            self._h = None
            self._keep.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
