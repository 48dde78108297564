"""CPU oracle for the DaggerFFT transform hot path -- TEST INFRASTRUCTURE ONLY.

This module is the checker that the CUDA library is compared against.  Only
``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import it; the product path (``libdfft`` and the ``dfft``
Python package) never calls into it and has no CPU fallback.

What it restates (file:line cites are relative to the DaggerFFT.jl tree):

* the transform tags and decomposition tags           src/fft.jl:1-24
* plan selection per tag, incl. the error message      src/fft.jl:126-154,
                                                       src/fftgpu.jl:85-105
* ``apply_fft!`` = plan + ``mul!`` on one chunk         src/fft.jl:168-174,
                                                       src/fftgpu.jl:118-124
* ``compute_overlap`` and the copy-pattern builder      src/fft.jl:176-178,
  ``create_workspace`` (dst-outer / src-inner walk,    src/fft.jl:233-407
  local / send / recv classification, per-peer buffer
  offsets in walk order)
* ``pack_data!`` / ``unpack_data!`` / ``local_copy!``  src/fft.jl:180-231
* ``flat_redistribute!`` (pack -> exchange -> local     src/fft.jl:413-495
  copies -> unpack)
* Pencil ``fft!``/``ifft!`` and Slab ``fft!``/``ifft!`` src/fft.jl:650-776,
  stage order and axes                                 src/fftgpu.jl:497-619
* ``Blocks`` layouts used by the benchmarks             benchmarks/fftmpi.jl:18-52
* the README-level ``fft/ifft/rfft/irfft`` and R2R       README.md:27-67
  (REDFT10/REDFT01) entry points.

The per-axis arithmetic in the reference is FFTW (CPU) / cuFFT (GPU), both
third-party and not present in the reference tree (FFTW.jl, CUDA.jl CUFFT and
AbstractFFTs are unpinned in Project.toml:4-26; no Manifest is shipped).  The
oracle restates their *published definitions*:

* forward DFT  X_k = sum_n x_n exp(-2 pi i n k / n), unnormalised;
* inverse      x_n = (1/n) sum_k X_k exp(+2 pi i n k / n)  (AbstractFFTs
  ``ScaledPlan``; across several dims the scale is 1/prod(n_i));
* rfft halves the FIRST transformed dim to n//2+1 (AbstractFFTs);
  irfft(F, d) needs the real length d of that dim;
* FFTW's r2r kinds (FFTW manual, "What FFTW Really Computes"), all
  unnormalised: REDFT00/01/10/11, RODFT00/01/10/11, DHT.

Per-axis DFTs are evaluated with numpy's pocketfft in float64 or extended
(long double) precision; ``dft_direct`` and ``r2r_direct`` are O(n^2) direct
sums in long double used to pin those evaluations on small sizes.

PARITY STATUS: the reference itself cannot run here (no Julia, no FFTW C
library), and its own correctness checks are commented out
(benchmarks/fftmpi.jl:80-100, benchmarks/fftmpigpu.jl:106-120), so no
golden vector from the reference exists.  Parity is therefore pinned to the
published transform definitions (direct sums and analytic known answers in
tests/golden/), not to reference output: "parity unpinned" with respect to
the reference binary.
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

# pi to long-double precision (np.pi is only the float64 value)
PI_LD = 4 * np.arctan(np.longdouble(1))

# --------------------------------------------------------------------------
# Tags (src/fft.jl:1-24)
# --------------------------------------------------------------------------

# FFTW's fftw_r2r_kind enumeration values (shared by FFTW.jl).
R2HC, HC2R, DHT = 0, 1, 2
REDFT00, REDFT01, REDFT10, REDFT11 = 3, 4, 5, 6
RODFT00, RODFT01, RODFT10, RODFT11 = 7, 8, 9, 10

# src/fft.jl:1-11
R2R_SUPPORTED_KINDS = (DHT, REDFT00, REDFT01, REDFT10, REDFT11,
                       RODFT00, RODFT01, RODFT10, RODFT11)


class Decomposition:
    pass


class Pencil(Decomposition):      # src/fft.jl:14
    pass


class Slab(Decomposition):        # src/fft.jl:15
    pass


class _Tag:
    name = "?"

    def __repr__(self):
        return self.name + "()"


def _mk(name):
    return type(name, (_Tag,), {"name": name})


FFT = _mk("FFT")          # src/fft.jl:17-24
RFFT = _mk("RFFT")
IRFFT = _mk("IRFFT")
IFFT = _mk("IFFT")
FFT_ = _mk("FFT!")
RFFT_ = _mk("RFFT!")
IRFFT_ = _mk("IRFFT!")
IFFT_ = _mk("IFFT!")


class R2R:
    """README.md:58-67 ``R2R((kind1, kind2, ...))``: one FFTW kind per dim."""

    def __init__(self, kinds):
        self.kinds = tuple(int(k) for k in kinds)


# --------------------------------------------------------------------------
# Direct definitions (pins for the evaluations below)
# --------------------------------------------------------------------------

def dft_direct(x, axis=0, sign=-1):
    """Unnormalised DFT along ``axis`` by an O(n^2) long-double sum."""
    x = np.moveaxis(np.asarray(x, dtype=np.clongdouble), axis, 0)
    n = x.shape[0]
    k = np.arange(n, dtype=np.longdouble)
    # exact reduction of the phase index modulo n keeps the angle small
    idx = np.outer(np.arange(n), np.arange(n)) % n
    ang = (sign * 2 * PI_LD / np.longdouble(n)) * idx.astype(np.longdouble)
    w = np.cos(ang) + 1j * np.sin(ang)
    y = np.tensordot(w.astype(np.clongdouble), x, axes=([1], [0]))
    del k
    return np.moveaxis(y, 0, axis)


def r2r_direct(x, kind, axis=0):
    """FFTW r2r kinds by their defining sums, in long double."""
    x = np.moveaxis(np.asarray(x, dtype=np.longdouble), axis, 0)
    n = x.shape[0]
    j = np.arange(n, dtype=np.longdouble)[None, :]
    k = np.arange(n, dtype=np.longdouble)[:, None]
    pi = PI_LD
    if kind == REDFT00:
        assert n >= 2
        m = (np.cos(pi * j[:, 1:-1] * k / (n - 1)) * 2)
        M = np.zeros((n, n), dtype=np.longdouble)
        M[:, 0] = 1
        M[:, -1] = ((-1.0) ** np.arange(n)).astype(np.longdouble)
        M[:, 1:-1] = m
        y = np.tensordot(M, x, axes=([1], [0]))
    elif kind == REDFT10:
        M = 2 * np.cos(pi * (j + 0.5) * k / n)
        y = np.tensordot(M, x, axes=([1], [0]))
    elif kind == REDFT01:
        M = 2 * np.cos(pi * j * (k + 0.5) / n)
        M[:, 0] = 1
        y = np.tensordot(M, x, axes=([1], [0]))
    elif kind == REDFT11:
        M = 2 * np.cos(pi * (j + 0.5) * (k + 0.5) / n)
        y = np.tensordot(M, x, axes=([1], [0]))
    elif kind == RODFT00:
        M = 2 * np.sin(pi * (j + 1) * (k + 1) / (n + 1))
        y = np.tensordot(M, x, axes=([1], [0]))
    elif kind == RODFT10:
        M = 2 * np.sin(pi * (j + 0.5) * (k + 1) / n)
        y = np.tensordot(M, x, axes=([1], [0]))
    elif kind == RODFT01:
        M = 2 * np.sin(pi * (j + 1) * (k + 0.5) / n)
        M[:, -1] = ((-1.0) ** np.arange(n)).astype(np.longdouble)
        y = np.tensordot(M, x, axes=([1], [0]))
    elif kind == RODFT11:
        M = 2 * np.sin(pi * (j + 0.5) * (k + 0.5) / n)
        y = np.tensordot(M, x, axes=([1], [0]))
    elif kind == DHT:
        a = 2 * pi * j * k / n
        M = np.cos(a) + np.sin(a)
        y = np.tensordot(M, x, axes=([1], [0]))
    else:
        raise ValueError("Unknown transform type")
    return np.moveaxis(y, 0, axis)


# --------------------------------------------------------------------------
# Fast evaluations of the same definitions (pocketfft, f64 or long double)
# --------------------------------------------------------------------------

def _work_dtype(x, precision):
    if precision == "native":
        return x
    if precision == "extended":
        return x.astype(np.clongdouble if np.iscomplexobj(x) else np.longdouble)
    return x.astype(np.complex128 if np.iscomplexobj(x) else np.float64)


# Host threads used by the per-chunk transforms (the CPU-baseline timing sets
# this to the core count; parity checks leave it at 1).
WORKERS = 1


def _c2c(x, axes, inverse):
    y = x
    if WORKERS > 1 and x.dtype in (np.complex64, np.complex128) and axes:
        import scipy.fft as sfft
        f = sfft.ifftn if inverse else sfft.fftn
        return f(y, axes=tuple(axes), workers=WORKERS)
    for a in axes:
        y = np.fft.ifft(y, axis=a) if inverse else np.fft.fft(y, axis=a)
    return y


def r2r_1d(x, kind, axis):
    """One FFTW r2r kind along ``axis`` evaluated through complex FFTs of the
    symmetric extension that defines it (FFTW manual, r2r kinds)."""
    x = np.moveaxis(x, axis, -1)
    n = x.shape[-1]
    cdt = np.clongdouble if x.dtype == np.longdouble else np.complex128
    pi = PI_LD if x.dtype == np.longdouble else np.pi
    k = np.arange(n, dtype=x.dtype)
    if kind == REDFT10:
        # even extension around n=-1/2 and n=N-1/2, period 2N
        ext = np.concatenate([x, x[..., ::-1]], axis=-1)
        X = np.fft.fft(ext.astype(cdt), axis=-1)[..., :n]
        y = (X * np.exp(-1j * pi * k / (2 * n))).real
    elif kind == REDFT01:
        # inverse of REDFT10 up to 2N: y_k = Re sum_n c_n x_n e^{i pi n (2k+1)/2N}
        w = np.exp(1j * pi * k / (2 * n)).astype(cdt)
        v = x.astype(cdt) * w
        v[..., 0] *= 0.5
        big = np.zeros(x.shape[:-1] + (2 * n,), dtype=cdt)
        big[..., :n] = v
        Y = np.fft.ifft(big, axis=-1) * (2 * n)
        y = 2 * Y[..., :n].real
    elif kind == REDFT00:
        ext = np.concatenate([x, x[..., -2:0:-1]], axis=-1)
        y = np.fft.fft(ext.astype(cdt), axis=-1)[..., :n].real
    elif kind == RODFT00:
        z = np.zeros(x.shape[:-1] + (1,), dtype=x.dtype)
        ext = np.concatenate([z, x, z, -x[..., ::-1]], axis=-1)
        y = -np.fft.fft(ext.astype(cdt), axis=-1)[..., 1:n + 1].imag
    elif kind == REDFT11:
        ext = np.concatenate([x, -x[..., ::-1], -x, x[..., ::-1]], axis=-1)
        m = 4 * n
        X = np.fft.fft(ext.astype(cdt), axis=-1)
        kk = np.arange(n, dtype=x.dtype)
        # Y_k = (1/2) Re( e^{-i pi (k+1/2) / (2N)} X_{2k+1} ) for the
        # 4N-periodic extension defined above
        y = 0.5 * (X[..., 2 * np.arange(n) + 1] *
                   np.exp(-1j * pi * (kk + 0.5) / (2 * n))).real
        del m
    elif kind == RODFT10:
        y = r2r_1d((x * ((-1.0) ** np.arange(n)).astype(x.dtype)), REDFT10, -1)[..., ::-1]
    elif kind == RODFT01:
        y = r2r_1d(x[..., ::-1], REDFT01, -1) * ((-1.0) ** np.arange(n)).astype(x.dtype)
    elif kind == RODFT11:
        y = r2r_1d(x[..., ::-1], REDFT11, -1) * ((-1.0) ** np.arange(n)).astype(x.dtype)
    elif kind == DHT:
        X = np.fft.fft(x.astype(cdt), axis=-1)
        y = X.real - X.imag
    else:
        raise ValueError("Unknown transform type")
    return np.moveaxis(np.ascontiguousarray(y), -1, axis)


# --------------------------------------------------------------------------
# Plans and apply_fft!  (src/fft.jl:113-174, src/fftgpu.jl:83-124)
# --------------------------------------------------------------------------

@dataclass
class OraclePlan:
    transform: type
    dims: Tuple[int, ...]     # 1-based, Julia convention
    n: Optional[int] = None   # real length for IRFFT


PLAN_CACHE: Dict[tuple, OraclePlan] = {}


def plan_transform(transform, A, dims, n=None):
    """src/fft.jl:126-154: tag -> plan.  RFFT/IRFFT need ``n`` (4-arg
    method); any other object is rejected with the reference's message."""
    dims = tuple(dims) if isinstance(dims, (tuple, list)) else (int(dims),)
    t = transform if isinstance(transform, type) else type(transform)
    if t in (FFT, IFFT, FFT_, IFFT_, RFFT_, IRFFT_, RFFT, IRFFT) or isinstance(transform, R2R):
        if t is IRFFT_ and n is None:
            n = A.shape[dims[0] - 1]     # src/fft.jl:138 size(A, first(dims))
        return OraclePlan(t if not isinstance(transform, R2R) else R2R, dims, n)
    raise ValueError("Unknown transform type")


def get_or_create_plan(transform, A, dims, n=None):
    """src/fft.jl:156-166, key (eltype, size, typeof(transform), dims)."""
    dims_t = tuple(dims) if isinstance(dims, (tuple, list)) else (int(dims),)
    t = transform if isinstance(transform, type) else type(transform)
    key = (A.dtype.str, A.shape, t, dims_t, n)
    if key not in PLAN_CACHE:
        PLAN_CACHE[key] = plan_transform(transform, A, dims_t, n)
    return PLAN_CACHE[key]


def apply_plan(plan, A, precision="f64", r2r_kinds=None):
    """``mul!(out, plan, in)`` for one chunk (src/fft.jl:168-174)."""
    axes = [d - 1 for d in plan.dims]
    x = _work_dtype(np.asarray(A), precision)
    t = plan.transform
    if t in (FFT, FFT_):
        return _c2c(x, axes, False)
    if t in (IFFT, IFFT_):
        return _c2c(x, axes, True)
    if t in (RFFT, RFFT_):
        y = np.fft.rfft(x, axis=axes[0])
        return _c2c(y, axes[1:], False)
    if t in (IRFFT, IRFFT_):
        y = _c2c(x, axes[1:], True)
        return np.fft.irfft(y, n=plan.n, axis=axes[0])
    if t is R2R:
        y = x
        kinds = list(r2r_kinds)
        if len(kinds) == 1 and len(axes) > 1:
            kinds = kinds * len(axes)
        for a, kd in zip(axes, kinds):
            y = r2r_1d(y, kd, a)
        return y
    raise ValueError("Unknown transform type")


def apply_fft(chunk, transform, dim, precision="f64", n=None):
    """``apply_fft!(chunk, transform, dim)``: returns the transformed chunk."""
    plan = get_or_create_plan(transform, chunk, dim, n)
    kinds = transform.kinds if isinstance(transform, R2R) else None
    return apply_plan(plan, chunk, precision, kinds)


# --------------------------------------------------------------------------
# Blocks / DArray model and the redistribution (src/fft.jl:176-495)
# --------------------------------------------------------------------------

@dataclass
class DArrayModel:
    """A logical column-major N1 x N2 x N3 array cut into ``Blocks`` chunks.

    ``subdomains[i]`` are 0-based half-open ranges per dim; chunks are
    enumerated in Julia's column-major order over the block grid, the order
    ``DArray.chunks`` uses.  ``owner[i]`` is the rank holding chunk i."""
    shape: Tuple[int, int, int]
    blocksize: Tuple[int, int, int]
    subdomains: List[Tuple[range, range, range]] = field(default_factory=list)
    owner: List[int] = field(default_factory=list)
    chunks: List[np.ndarray] = field(default_factory=list)


def blocks(shape, blocksize, nranks=1):
    """``distribute(A, Blocks(b1,b2,b3))`` layout (benchmarks/fftmpi.jl:18-52).
    Chunks are assigned round-robin over ranks in chunk order."""
    shape = tuple(int(s) for s in shape)
    bs = tuple(int(b) for b in blocksize)
    nb = [(s + b - 1) // b for s, b in zip(shape, bs)]
    dm = DArrayModel(shape, bs)
    i = 0
    for kz in range(nb[2]):
        for ky in range(nb[1]):
            for kx in range(nb[0]):
                sd = tuple(range(k * b, min((k + 1) * b, s))
                           for k, b, s in zip((kx, ky, kz), bs, shape))
                dm.subdomains.append(sd)
                dm.owner.append(i % nranks)
                i += 1
    return dm


def distribute(A, layout: DArrayModel):
    A = np.asarray(A)
    layout.chunks = [np.array(A[sd[0].start:sd[0].stop, sd[1].start:sd[1].stop,
                               sd[2].start:sd[2].stop]) for sd in layout.subdomains]
    return layout


def collect(layout: DArrayModel):
    out = np.empty(layout.shape, dtype=layout.chunks[0].dtype)
    for sd, c in zip(layout.subdomains, layout.chunks):
        out[sd[0].start:sd[0].stop, sd[1].start:sd[1].stop, sd[2].start:sd[2].stop] = c
    return out


def compute_overlap(src_domain, dst_domain):
    """src/fft.jl:176-178: per-dim intersection of index ranges."""
    return tuple(range(max(a.start, b.start), min(a.stop, b.stop))
                 for a, b in zip(src_domain, dst_domain))


@dataclass
class Pattern:
    """``CoalescedPattern`` (src/fft.jl:66-75), 0-based local index ranges."""
    src_idx: int
    dst_idx: int
    overlap: tuple
    src_indices: tuple
    dst_indices: tuple
    buffer_offset: int
    buffer_size: int


@dataclass
class Workspace:
    rank: int
    local_patterns: List[Pattern]
    send_peers: Dict[int, List[Pattern]]
    recv_peers: Dict[int, List[Pattern]]
    send_sizes: Dict[int, int]
    recv_sizes: Dict[int, int]


def create_workspace(src: DArrayModel, dst: DArrayModel, rank=0):
    """src/fft.jl:233-407 (flat path): walk dst chunks (outer) x src chunks
    (inner); classify each non-empty overlap as a local copy, a send to the
    dst owner, or a receive from the src owner; per-peer buffers are packed
    in walk order (offsets accumulate, src/fft.jl:313-343)."""
    local, sendp, recvp = [], {}, {}
    for di, dd in enumerate(dst.subdomains):
        drank = dst.owner[di]
        for si, sd in enumerate(src.subdomains):
            srank = src.owner[si]
            ov = compute_overlap(sd, dd)
            if any(len(r) == 0 for r in ov):
                continue
            size = int(np.prod([len(r) for r in ov]))
            s_ix = tuple(range(o.start - s.start, o.stop - s.start) for o, s in zip(ov, sd))
            d_ix = tuple(range(o.start - d.start, o.stop - d.start) for o, d in zip(ov, dd))
            if srank == rank and drank != rank:
                sendp.setdefault(drank, []).append((si, di, ov, s_ix, d_ix, size))
            elif drank == rank and srank != rank:
                recvp.setdefault(srank, []).append((si, di, ov, s_ix, d_ix, size))
            elif srank == rank and drank == rank:
                local.append(Pattern(si, di, ov, s_ix, d_ix, 0, size))

    def coalesce(d):
        out, sizes = {}, {}
        for peer, lst in d.items():
            off = 0
            pats = []
            for (si, di, ov, s_ix, d_ix, size) in lst:
                pats.append(Pattern(si, di, ov, s_ix, d_ix, off, size))
                off += size
            out[peer] = pats
            sizes[peer] = off
        return out, sizes

    sp, ss = coalesce(sendp)
    rp, rs = coalesce(recvp)
    return Workspace(rank, local, sp, rp, ss, rs)


def pack_data(buffer, src, indices, offset=0):
    """src/fft.jl:180-196: x-fastest gather of a sub-block into ``buffer``."""
    blk = src[indices[0].start:indices[0].stop, indices[1].start:indices[1].stop,
              indices[2].start:indices[2].stop]
    n = blk.size
    buffer[offset:offset + n] = blk.reshape(-1, order="F")


def unpack_data(dst, buffer, indices, offset=0):
    """src/fft.jl:198-214: inverse of ``pack_data``."""
    shp = tuple(len(r) for r in indices)
    n = int(np.prod(shp))
    dst[indices[0].start:indices[0].stop, indices[1].start:indices[1].stop,
        indices[2].start:indices[2].stop] = buffer[offset:offset + n].reshape(shp, order="F")


def local_copy(dst, src, dst_indices, src_indices):
    """src/fft.jl:216-231."""
    dst[dst_indices[0].start:dst_indices[0].stop, dst_indices[1].start:dst_indices[1].stop,
        dst_indices[2].start:dst_indices[2].stop] = \
        src[src_indices[0].start:src_indices[0].stop, src_indices[1].start:src_indices[1].stop,
            src_indices[2].start:src_indices[2].stop]


def flat_redistribute(dst: DArrayModel, src: DArrayModel, workspaces: Sequence[Workspace]):
    """src/fft.jl:413-495 for every rank of a world in one process: each rank
    packs its send buffers, the buffers are delivered, local copies run, and
    the receivers unpack (the MPI exchange becomes a dict hand-off)."""
    if not dst.chunks:
        dst.chunks = [np.empty(tuple(len(r) for r in sd), dtype=src.chunks[0].dtype)
                      for sd in dst.subdomains]
    mailbox = {}
    for ws in workspaces:
        for peer, pats in ws.send_peers.items():
            buf = np.empty(ws.send_sizes[peer], dtype=src.chunks[0].dtype)
            for p in pats:
                pack_data(buf, src.chunks[p.src_idx], p.src_indices, p.buffer_offset)
            mailbox[(ws.rank, peer)] = buf
    for ws in workspaces:
        for p in ws.local_patterns:
            local_copy(dst.chunks[p.dst_idx], src.chunks[p.src_idx], p.dst_indices, p.src_indices)
    for ws in workspaces:
        for peer, pats in ws.recv_peers.items():
            buf = mailbox[(peer, ws.rank)]
            for p in pats:
                unpack_data(dst.chunks[p.dst_idx], buf, p.dst_indices, p.buffer_offset)
    return dst


def _stage(layout: DArrayModel, transform, dims, precision):
    layout.chunks = [np.asarray(apply_fft(c, transform, dims, precision)) for c in layout.chunks]


def fft_pencil(C, A, B, wsAB, wsBC, transforms, dims, precision="f64"):
    """Pencil ``fft!`` (src/fft.jl:651-688, src/fftgpu.jl:498-531)."""
    _stage(A, transforms[0], dims[0], precision)
    flat_redistribute(B, A, wsAB)
    _stage(B, transforms[1], dims[1], precision)
    flat_redistribute(C, B, wsBC)
    _stage(C, transforms[2], dims[2], precision)
    return C


def ifft_pencil(C, A, B, wsAB, wsBC, transforms, dims, precision="f64"):
    """Pencil ``ifft!`` (src/fft.jl:691-724): transforms[3] on dims[3] first."""
    _stage(A, transforms[2], dims[2], precision)
    flat_redistribute(B, A, wsAB)
    _stage(B, transforms[1], dims[1], precision)
    flat_redistribute(C, B, wsBC)
    _stage(C, transforms[0], dims[0], precision)
    return C


def fft_slab(B, A, wsAB, transforms, dims, precision="f64"):
    """Slab ``fft!`` (src/fft.jl:727-750): 2-D on (dims[1],dims[2]) then dims[3]."""
    _stage(A, transforms[0], (dims[0], dims[1]), precision)
    flat_redistribute(B, A, wsAB)
    _stage(B, transforms[2], dims[2], precision)
    return B


def ifft_slab(A, B, wsBA, transforms, dims, precision="f64"):
    """Slab ``ifft!`` (src/fft.jl:753-776)."""
    _stage(B, transforms[2], dims[2], precision)
    flat_redistribute(A, B, wsBA)
    _stage(A, transforms[0], (dims[0], dims[1]), precision)
    return A


def pencil_layouts(n, chunk, nranks=1):
    """benchmarks/fftmpi.jl:35-41: DA Blocks(N,c,c), DB Blocks(c,N,c), DC Blocks(c,c,N)."""
    N1, N2, N3 = n
    return (blocks(n, (N1, chunk, chunk), nranks), blocks(n, (chunk, N2, chunk), nranks),
            blocks(n, (chunk, chunk, N3), nranks))


def slab_layouts(n, chunk, nranks=1):
    """benchmarks/fftmpi.jl:18-25: DA Blocks(N,N,c), DB Blocks(c,N,N)."""
    N1, N2, N3 = n
    return blocks(n, (N1, N2, chunk), nranks), blocks(n, (chunk, N2, N3), nranks)


# --------------------------------------------------------------------------
# README-level API (README.md:27-67)
# --------------------------------------------------------------------------

def _dims(dims):
    return tuple(int(d) for d in (dims if isinstance(dims, (tuple, list)) else (dims,)))


def fft(A, decomp=None, dims=(1, 2, 3), transforms=None, precision="f64"):
    A = np.asarray(A)
    dims = _dims(dims)
    if transforms is not None:
        t = transforms[0]
        if isinstance(t, R2R):
            return apply_plan(OraclePlan(R2R, dims), A, precision, t.kinds)
    return apply_plan(OraclePlan(FFT, dims), A, precision)


def ifft(A, decomp=None, dims=(1, 2, 3), transforms=None, precision="f64"):
    A = np.asarray(A)
    dims = _dims(dims)
    if transforms is not None:
        t = transforms[0]
        if isinstance(t, R2R):
            return apply_plan(OraclePlan(R2R, dims), A, precision, t.kinds)
    return apply_plan(OraclePlan(IFFT, dims), A, precision)


def rfft(A, decomp=None, dims=(1, 2, 3), precision="f64"):
    return apply_plan(OraclePlan(RFFT, _dims(dims)), np.asarray(A), precision)


def irfft(F, d, decomp=None, dims=(1, 2, 3), precision="f64"):
    return apply_plan(OraclePlan(IRFFT, _dims(dims), int(d)), np.asarray(F), precision)


# --------------------------------------------------------------------------
# Seeded inputs for the benchmark configurations
# --------------------------------------------------------------------------

def make_input(kind, shape, seed, dtype):
    """Synthetic inputs with the distributions the configurations name:
    ``uniform01`` (Julia ``rand``), ``normal`` (``randn``), ``uniform11``."""
    rng = np.random.default_rng(seed)
    cplx = np.dtype(dtype).kind == "c"
    real_t = np.float32 if np.dtype(dtype) in (np.complex64, np.float32) else np.float64

    def draw():
        if kind == "uniform01":
            return rng.random(shape, dtype=np.float64)
        if kind == "uniform11":
            return rng.random(shape, dtype=np.float64) * 2 - 1
        if kind == "normal":
            return rng.standard_normal(shape)
        raise ValueError(kind)

    re = draw().astype(real_t)
    if not cplx:
        return np.asfortranarray(re)
    im = draw().astype(real_t)
    return np.asfortranarray(re + 1j * im).astype(dtype)


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.clongdouble if np.iscomplexobj(a) or np.iscomplexobj(b) else np.longdouble)
    b = np.asarray(b, dtype=a.dtype)
    num = np.sqrt(np.sum(np.abs(a - b) ** 2))
    den = np.sqrt(np.sum(np.abs(b) ** 2))
    return float(num / den) if den != 0 else float(num)


def cpu_threads():
    return os.cpu_count() or 1
