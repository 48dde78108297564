"""Host-side mirror of DaggerFFT's transform API over libdfft.

Reference interface mirrored here (paths relative to DaggerFFT.jl):
  * tags ``Pencil``/``Slab`` and ``FFT``/``IFFT``/``RFFT``/``IRFFT`` plus the
    in-place ``FFT!`` family (here ``FFT_`` ...)          src/fft.jl:13-24
  * ``R2R((kind, ...))`` and the FFTW kind constants     README.md:58-67,
                                                         src/fft.jl:1-11
  * ``gpu_plan_transform`` / ``get_or_create_gpu_plan``  src/fftgpu.jl:83-116
    (same cache key: eltype, size, tag type, dims)
  * ``apply_gpu_fft!`` = plan + ``mul!``                src/fftgpu.jl:118-124
  * README-level ``fft/ifft/rfft/irfft(A; decomp, transforms, dims)``
                                                         README.md:27-67

Arrays are torch CUDA tensors indexed like the Julia arrays they stand for:
``A[i, j, k]`` is Julia's ``A[i+1, j+1, k+1]`` and ``dims`` are 1-based.
Both Fortran-ordered (Julia's own layout) and C-ordered tensors are accepted
without a copy: a C-ordered tensor is the column-major array with reversed
dims, so the dims are renumbered instead of the data moved.  Outputs take
the memory order of the input.  All work is enqueued on torch's current
stream.
"""
from __future__ import annotations

import ctypes
import threading
from typing import Dict, Sequence, Tuple

import torch

from . import _lib
from ._lib import ArgumentError, DFFTError, check

# ---------------------------------------------------------------------------
# tags (src/fft.jl:13-24)
# ---------------------------------------------------------------------------


class Decomposition:
    code = -1

    def __repr__(self):
        return type(self).__name__ + "()"

    def __eq__(self, other):
        return type(self) is type(other)

    def __hash__(self):
        return hash(type(self).__name__)


class Pencil(Decomposition):
    """2-D domain decomposition: one stage per transformed dim."""
    code = _lib.PENCIL


class Slab(Decomposition):
    """1-D decomposition: a 2-D stage on (dims[1], dims[2]) then dims[3]."""
    code = _lib.SLAB


class Transform:
    code = -1
    name = "?"

    def __repr__(self):
        return self.name + "()"

    def __eq__(self, other):
        return type(self) is type(other)

    def __hash__(self):
        return hash(self.name)


def _tag(name, code):
    return type(name.replace("!", "_"), (Transform,), {"code": code, "name": name})


FFT = _tag("FFT", _lib.T_FFT)
IFFT = _tag("IFFT", _lib.T_IFFT)
RFFT = _tag("RFFT", _lib.T_RFFT)
IRFFT = _tag("IRFFT", _lib.T_IRFFT)
FFT_ = _tag("FFT!", _lib.T_FFT_INPLACE)
IFFT_ = _tag("IFFT!", _lib.T_IFFT_INPLACE)
RFFT_ = _tag("RFFT!", _lib.T_RFFT_INPLACE)
IRFFT_ = _tag("IRFFT!", _lib.T_IRFFT_INPLACE)

# FFTW r2r kinds (fftw_r2r_kind values)
R2HC, HC2R, DHT = 0, 1, 2
REDFT00, REDFT01, REDFT10, REDFT11 = 3, 4, 5, 6
RODFT00, RODFT01, RODFT10, RODFT11 = 7, 8, 9, 10
R2R_SUPPORTED_KINDS = (DHT, REDFT00, REDFT01, REDFT10, REDFT11,
                       RODFT00, RODFT01, RODFT10, RODFT11)


class R2R(Transform):
    """``R2R((kind1, kind2, ...))``: one FFTW r2r kind per transformed dim."""
    code = _lib.T_R2R
    name = "R2R"

    def __init__(self, kinds):
        kinds = tuple(int(k) for k in (kinds if isinstance(kinds, (tuple, list)) else (kinds,)))
        for k in kinds:
            if k not in R2R_SUPPORTED_KINDS:
                raise ArgumentError(_lib.ERROR_UNKNOWN_TRANSFORM, "Unknown transform type")
        self.kinds = kinds

    def __repr__(self):
        return f"R2R({self.kinds})"

    def __eq__(self, other):
        return isinstance(other, R2R) and other.kinds == self.kinds

    def __hash__(self):
        return hash(("R2R", self.kinds))


_METHODS = {"plain": _lib.PLAIN, "mixed": _lib.MIXED}

# ---------------------------------------------------------------------------
# layout helpers
# ---------------------------------------------------------------------------


def _order(t: torch.Tensor) -> str:
    """'F' if ``t`` is column-major contiguous, 'C' if row-major contiguous."""
    if t.dim() <= 1:
        return "F"
    if t.is_contiguous():
        return "C"
    if t.permute(*reversed(range(t.dim()))).is_contiguous():
        return "F"
    return "X"


def _empty(shape, dtype, device, order):
    if order == "F" and len(shape) > 1:
        return torch.empty(tuple(reversed(shape)), dtype=dtype, device=device).permute(
            *reversed(range(len(shape))))
    return torch.empty(tuple(shape), dtype=dtype, device=device)


def empty_like_layout(shape, dtype, like: torch.Tensor):
    """A new tensor of ``shape``/``dtype`` in the memory order of ``like``."""
    o = _order(like)
    return _empty(shape, dtype, like.device, "F" if o == "F" else "C")


def _norm_dims(dims, ndim) -> Tuple[int, ...]:
    if isinstance(dims, int):
        dims = (dims,)
    dims = tuple(int(d) for d in dims)
    for d in dims:
        if d < 1 or d > ndim:
            raise ArgumentError(_lib.ERROR_INVALID_VALUE, f"dims entry {d} out of range 1..{ndim}")
    return dims


def _precision(dtype) -> int:
    if dtype in (torch.complex64, torch.float32):
        return _lib.F32
    if dtype in (torch.complex128, torch.float64):
        return _lib.F64
    raise ArgumentError(_lib.ERROR_INVALID_VALUE, f"unsupported element type {dtype}")


# ---------------------------------------------------------------------------
# plans (src/fftgpu.jl:83-124)
# ---------------------------------------------------------------------------


class Plan:
    """A libdfft plan for one (shape, layout, eltype, tag, dims) combination."""

    def __init__(self, transform: Transform, shape, dtype, dims, order="F", n=None,
                 decomp: Decomposition = None, method="plain", flags=0, device=None):
        if not isinstance(transform, Transform):
            raise ArgumentError(_lib.ERROR_UNKNOWN_TRANSFORM, "Unknown transform type")
        decomp = decomp or Pencil()
        L = _lib.lib()
        self._L = L
        self.transform = transform
        self.shape = tuple(int(s) for s in shape)
        self.dtype = dtype
        self.order = order
        nd = len(self.shape)
        self.dims = _norm_dims(dims, nd)
        if order == "C":
            cm_shape = tuple(reversed(self.shape))
            cm_dims = tuple(nd + 1 - d for d in self.dims)
        else:
            cm_shape = self.shape
            cm_dims = self.dims
        kinds = transform.kinds if isinstance(transform, R2R) else ()
        if isinstance(transform, R2R):
            if len(kinds) == 1 and len(self.dims) > 1:
                kinds = kinds * len(self.dims)
            if len(kinds) != len(self.dims):
                raise ArgumentError(_lib.ERROR_INVALID_VALUE, "R2R needs one kind per dim")
        self.kinds = kinds
        self.n = n
        self.device = device if device is not None else torch.cuda.current_device()
        h = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            check(L.dfft_plan_create(
                ctypes.byref(h), nd, _lib.i64_array(cm_shape), _precision(dtype), transform.code,
                len(cm_dims), _lib.i32_array(cm_dims), _lib.i32_array(kinds),
                int(n) if n is not None else 0, decomp.code, _METHODS[method], int(flags)))
        self._h = h
        out = (ctypes.c_int64 * nd)()
        check(L.dfft_plan_output_shape(h, out))
        cm_out = tuple(out[i] for i in range(nd))
        self.out_shape = tuple(reversed(cm_out)) if order == "C" else cm_out
        nl = ctypes.c_int()
        check(L.dfft_plan_launches(h, ctypes.byref(nl)))
        self.launches = nl.value
        wb = ctypes.c_size_t()
        check(L.dfft_plan_workspace_bytes(h, ctypes.byref(wb)))
        self.workspace_bytes = wb.value

    def describe(self) -> str:
        """One line per kernel launch (kernel kind, length, columns, launch
        shape): ``dfft_plan_describe``."""
        buf = ctypes.create_string_buffer(8192)
        check(self._L.dfft_plan_describe(self._h, buf, ctypes.c_size_t(len(buf))))
        return buf.value.decode()

    def execute(self, inp: torch.Tensor, out: torch.Tensor, stream=None):
        if stream is None:
            stream = torch.cuda.current_stream(inp.device)
        s = stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream or 0)
        check(self._L.dfft_execute(self._h, ctypes.c_void_p(inp.data_ptr()),
                                   ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(s)))
        return out

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                self._L.dfft_plan_destroy(h)
            except Exception:
                pass
            self._h = None


GPU_PLAN_CACHE: Dict[tuple, Plan] = {}
_CACHE_LOCK = threading.Lock()


def gpu_plan_transform(transform, A: torch.Tensor, dims, n=None, decomp=None, method="plain",
                       flags=0) -> Plan:
    """src/fftgpu.jl:85-105: a fresh plan for tag ``transform`` on ``A``."""
    o = _order(A)
    if o == "X":
        raise ArgumentError(_lib.ERROR_INVALID_VALUE, "array must be contiguous (C or Fortran order)")
    return Plan(transform, tuple(A.shape), A.dtype, dims, order=o, n=n, decomp=decomp,
                method=method, flags=flags, device=A.device.index)


def get_or_create_gpu_plan(transform, A: torch.Tensor, dims, n=None, decomp=None,
                           method="plain", flags=0) -> Plan:
    """src/fftgpu.jl:107-116; key (eltype, size, tag, dims) plus the layout,
    device, real length, decomposition and arithmetic form."""
    if not isinstance(transform, Transform):
        raise ArgumentError(_lib.ERROR_UNKNOWN_TRANSFORM, "Unknown transform type")
    dims_t = tuple(dims) if isinstance(dims, (tuple, list)) else (int(dims),)
    key = (A.dtype, tuple(A.shape), _order(A), transform, dims_t, n, type(decomp or Pencil()),
           method, flags, A.device.index)
    with _CACHE_LOCK:
        p = GPU_PLAN_CACHE.get(key)
    if p is None:
        p = gpu_plan_transform(transform, A, dims_t, n, decomp, method, flags)
        with _CACHE_LOCK:
            GPU_PLAN_CACHE.setdefault(key, p)
            p = GPU_PLAN_CACHE[key]
    return p


def gpu_cleanup_plans():
    """``gpu_cleanup_workspace!``'s plan-cache part (src/fftgpu.jl:630-634)."""
    with _CACHE_LOCK:
        GPU_PLAN_CACHE.clear()


def _check_tensor(A):
    if not isinstance(A, torch.Tensor) or not A.is_cuda:
        raise ArgumentError(_lib.ERROR_INVALID_VALUE, "expected a CUDA tensor (the CuArray path)")


def apply_gpu_fft_(out: torch.Tensor, inp: torch.Tensor, transform, dim, n=None, decomp=None,
                   method="plain"):
    """``apply_gpu_fft!(out, in, transform, dim)``: plan lookup + ``mul!``."""
    _check_tensor(inp)
    p = get_or_create_gpu_plan(transform, inp, dim, n, decomp, method)
    if tuple(out.shape) != p.out_shape:
        raise ArgumentError(_lib.ERROR_INVALID_VALUE, f"output shape {tuple(out.shape)} != {p.out_shape}")
    if _order(out) != _order(inp) and out.dim() > 1:
        raise ArgumentError(_lib.ERROR_INVALID_VALUE, "output must have the input's memory order")
    return p.execute(inp, out)


# ---------------------------------------------------------------------------
# README-level API (README.md:27-67)
# ---------------------------------------------------------------------------


def _prep(A):
    _check_tensor(A)
    if _order(A) == "X":
        A = A.contiguous()
    return A


def _run(transform, A, dims, n=None, decomp=None, method="plain", flags=0, out_dtype=None):
    A = _prep(A)
    p = get_or_create_gpu_plan(transform, A, dims, n, decomp, method, flags)
    out = empty_like_layout(p.out_shape, out_dtype or A.dtype, A)
    return p.execute(A, out)


def _complex_dtype(dt):
    return {torch.float32: torch.complex64, torch.float64: torch.complex128}.get(dt, dt)


def _real_dtype(dt):
    return {torch.complex64: torch.float32, torch.complex128: torch.float64}.get(dt, dt)


def _r2r_of(transforms):
    if transforms is None:
        return None
    ts = transforms if isinstance(transforms, (tuple, list)) else (transforms,)
    if ts and isinstance(ts[0], R2R):
        return ts[0]
    for t in ts:
        if not isinstance(t, Transform):
            raise ArgumentError(_lib.ERROR_UNKNOWN_TRANSFORM, "Unknown transform type")
    return None


def fft(A, decomp=None, dims=(1, 2, 3), transforms=None, method="plain"):
    """Forward transform of ``A`` over ``dims``: C2C, or the r2r kinds of
    ``transforms=(R2R((k1, k2, ...)),)``."""
    dims = _norm_dims(dims, A.dim())
    r = _r2r_of(transforms)
    if r is not None:
        if A.is_complex():
            raise ArgumentError(_lib.ERROR_INVALID_VALUE, "R2R transforms take real arrays")
        return _run(r, A, dims, decomp=decomp)
    if not A.is_complex():
        A = A.to(_complex_dtype(A.dtype))
    return _run(FFT(), A, dims, decomp=decomp, method=method)


def ifft(A, decomp=None, dims=(1, 2, 3), transforms=None, method="plain"):
    """Inverse C2C scaled by 1/prod(n_i); with R2R transforms, the given
    (unnormalised) kinds, e.g. REDFT01 to undo REDFT10 up to 2N per dim."""
    dims = _norm_dims(dims, A.dim())
    r = _r2r_of(transforms)
    if r is not None:
        if A.is_complex():
            raise ArgumentError(_lib.ERROR_INVALID_VALUE, "R2R transforms take real arrays")
        return _run(r, A, dims, decomp=decomp)
    if not A.is_complex():
        A = A.to(_complex_dtype(A.dtype))
    return _run(IFFT(), A, dims, decomp=decomp, method=method)


def rfft(A, decomp=None, dims=(1, 2, 3)):
    """Real-to-complex: dims[1] is halved to n//2+1."""
    dims = _norm_dims(dims, A.dim())
    if A.is_complex():
        raise ArgumentError(_lib.ERROR_INVALID_VALUE, "rfft takes a real array")
    return _run(RFFT(), A, dims, decomp=decomp, out_dtype=_complex_dtype(A.dtype))


def irfft(F, d, decomp=None, dims=(1, 2, 3), destroy_input=False):
    """Complex-to-real with real length ``d`` along dims[1]."""
    dims = _norm_dims(dims, F.dim())
    if not F.is_complex():
        raise ArgumentError(_lib.ERROR_INVALID_VALUE, "irfft takes a complex array")
    flags = _lib.FLAG_DESTROY_INPUT if destroy_input else 0
    return _run(IRFFT(), F, dims, n=int(d), decomp=decomp, flags=flags,
                out_dtype=_real_dtype(F.dtype))


def fft_(A, decomp=None, dims=(1, 2, 3), method="plain"):
    """``fft!``: in-place forward C2C."""
    A_ = _prep(A)
    if A_.data_ptr() != A.data_ptr():
        raise ArgumentError(_lib.ERROR_INVALID_VALUE, "fft! needs a contiguous array")
    p = get_or_create_gpu_plan(FFT_(), A, _norm_dims(dims, A.dim()), decomp=decomp, method=method)
    return p.execute(A, A)


def ifft_(A, decomp=None, dims=(1, 2, 3), method="plain"):
    """``ifft!``: in-place inverse C2C."""
    A_ = _prep(A)
    if A_.data_ptr() != A.data_ptr():
        raise ArgumentError(_lib.ERROR_INVALID_VALUE, "ifft! needs a contiguous array")
    p = get_or_create_gpu_plan(IFFT_(), A, _norm_dims(dims, A.dim()), decomp=decomp, method=method)
    return p.execute(A, A)


# ---------------------------------------------------------------------------
# batches of uneven transforms (one CUDA graph launch)
# ---------------------------------------------------------------------------


class Batch:
    """Independent plans executed together (``dfft_batch_*``): one CUDA
    graph of the plans' passes, or, with ``persistent=True``, one launch of
    the persistent batch kernel when every plan is a complex transform of
    the lengths it runs (``launches == 1``; ``lag`` staggers a pass behind
    its predecessor in the work list, 0 = automatic).  ``execute(ins,
    outs)`` takes one input and one output tensor per plan; a graph is
    captured on the first call and replayed while the same buffers are
    passed."""

    def __init__(self, plans: Sequence[Plan], persistent: bool = False, lag: int = 0):
        L = _lib.lib()
        self._L = L
        self.plans = list(plans)  # keeps the plans alive
        L.dfft_batch_create_ex.argtypes = [ctypes.POINTER(ctypes.c_void_p), ctypes.c_int,
                                           ctypes.POINTER(ctypes.c_void_p), ctypes.c_uint]
        L.dfft_batch_create_ex.restype = ctypes.c_int
        L.dfft_batch_execute.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p),
                                         ctypes.POINTER(ctypes.c_void_p), ctypes.c_void_p]
        L.dfft_batch_execute.restype = ctypes.c_int
        L.dfft_batch_launches.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int)]
        L.dfft_batch_launches.restype = ctypes.c_int
        L.dfft_batch_destroy.argtypes = [ctypes.c_void_p]
        L.dfft_batch_destroy.restype = ctypes.c_int
        arr = (ctypes.c_void_p * len(self.plans))(*[p._h.value for p in self.plans])
        h = ctypes.c_void_p()
        if not 0 <= lag <= 255:
            raise ArgumentError(_lib.ERROR_INVALID_VALUE, "lag must be in 0..255")
        flags = (2 if persistent else 0) | (lag << 8)
        check(L.dfft_batch_create_ex(ctypes.byref(h), len(self.plans), arr, flags))
        self._h = h
        n = ctypes.c_int()
        check(L.dfft_batch_launches(h, ctypes.byref(n)))
        self.launches = n.value

    def execute(self, ins, outs, stream=None):
        if len(ins) != len(self.plans) or len(outs) != len(self.plans):
            raise ArgumentError(_lib.ERROR_INVALID_VALUE, "one input and one output per plan")
        if stream is None:
            stream = torch.cuda.current_stream()
        ia = (ctypes.c_void_p * len(ins))(*[t.data_ptr() for t in ins])
        oa = (ctypes.c_void_p * len(outs))(*[t.data_ptr() for t in outs])
        check(self._L.dfft_batch_execute(self._h, ia, oa, ctypes.c_void_p(stream.cuda_stream)))
        return outs

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                self._L.dfft_batch_destroy(h)
            except Exception:
                pass
            self._h = None
