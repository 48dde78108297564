"""Distributed Slab FFT with the exchange's pack and unpack folded into the
slab pass (the multi-GPU Slab path).

The reference's Slab ``gpu_fft!`` (src/fftgpu.jl:534-557) runs the 2-D
stage on each z-slab chunk, then ``gpu_flat_redistribute!``
(src/fftgpu.jl:324-415): a pack kernel into a flat send buffer, MPI
point-to-point, an unpack kernel (src/fftgpu.jl:417-480), then the
last-axis stage.  Here, for an L x L x N3 complex array with L divisible by
the number of ranks P:

* rank r holds the z-slabs Z_r (contiguous, ``zsplit``) as an F-ordered
  (L, L, |Z_r|) array A_r, and receives either the x-columns X_r = [r R,
  (r+1) R), R = L / P, of every slab as an F-ordered (R, L, N3) array B_r
  (split "x": the reference's Blocks(L, L, c) -> Blocks(c, L, N3)) or the
  y-rows Y_r as an (L, R, N3) array (split "y");
* the fused slab pass writes its output in a rank-split layout
  (``dfft_slab_split_create``): the columns (rows) rank s owns, of every
  local slab, form one contiguous block -- exactly what rank s receives
  from r, and exactly the slab range Z_r of B_s.  No pack or unpack kernel
  runs (for split "x" the slab pass runs its y-phase first and writes the
  x-phase's pencils in per-rank pieces);
* the local slabs run in ``ngroups`` groups; group g's blocks go out
  (NCCL grouped send/recv through ``torch.distributed``) while group g+1
  is still transforming, and the last-axis pass runs on B_r in place once
  every block has arrived.

The inverse mirrors it: the last-axis IFFT on B_r, group g's z-range of
B_r (contiguous) sent to its owner while the receiver transforms the
groups that have arrived, from the split layout back to A_r.

The compute steps go through a ``kernels`` object (default
``CudaSlabKernels``: libdfft plans) so that the exchange schedule runs on
CPU ranks too.
"""
from __future__ import annotations

import ctypes
from typing import List, Optional, Sequence, Tuple

import torch

from . import _lib
from ._lib import ArgumentError, check
from .api import FFT_, IFFT_, _precision, get_or_create_gpu_plan


def zsplit(n3: int, world: int) -> List[Tuple[int, int]]:
    """Slab ranges (start, count) per rank: blocks of ceil(n3 / world), the
    reference's Blocks(N1, N2, ceil(N3 / P)) chunking with one chunk per
    rank (the last ranks may hold fewer slabs, or none)."""
    b = -(-n3 // world)
    out = []
    for r in range(world):
        z0 = min(r * b, n3)
        out.append((z0, min(b, n3 - z0)))
    return out


def groups_of(count: int, ngroups: int) -> List[Tuple[int, int]]:
    """Slab groups (offset, count) of a rank's ``count`` local slabs: the
    same rule on every rank, so a receiver knows each sender's groups."""
    if count == 0:
        return [(0, 0)] * ngroups
    g = max(1, min(ngroups, count))
    base, extra = divmod(count, g)
    out, z = [], 0
    for i in range(ngroups):
        n = base + (1 if i < extra else 0) if i < g else 0
        out.append((z, n))
        z += n
    return out


def split_row(R: int, zr: int, z: int, y: int) -> int:
    """Row (units of L elements) of row y of local slab z in the row-split
    layout with R rows per rank and zr slabs between rank blocks."""
    return (y % R) + R * (z + zr * (y // R))


def split_col(R: int, L: int, zr: int, z: int, y: int, x: int) -> int:
    """Element offset of (x, y, local slab z) in the column-split layout
    with R columns per rank and zr slabs between rank blocks."""
    return (x % R) + R * (y + L * (z + zr * (x // R)))


def _flat(t: torch.Tensor) -> torch.Tensor:
    """The memory of an F-ordered (column-major, dense) array as a flat view."""
    shape = tuple(t.shape)
    want, acc = [], 1
    for s in shape:
        want.append(acc)
        acc *= s
    if t.numel() > 1 and tuple(st for st, s in zip(t.stride(), shape) if s > 1) != \
            tuple(w for w, s in zip(want, shape) if s > 1):
        raise ArgumentError(_lib.ERROR_INVALID_VALUE, "slab exchange needs dense column-major chunks")
    return t.as_strided((t.numel(),), (1,))


class SlabSplitPlan:
    """``dfft_slab_split_create``: the fused dims-(1, 2) pass over ``nslab``
    L x L slabs with the output (forward) or input (inverse) in the
    rank-split layout of ``nranks`` ranks, ``zr`` slabs between rank
    blocks.  ``execute`` takes flat tensors and element offsets."""

    def __init__(self, L, nslab, zr, nranks, dtype, inverse, device=None, split_dim=2):
        lib = _lib.lib()
        self._L = lib
        lib.dfft_slab_split_create.argtypes = [ctypes.POINTER(ctypes.c_void_p), ctypes.c_int, ctypes.c_int,
                                               ctypes.c_int64, ctypes.c_int64, ctypes.c_int64, ctypes.c_int,
                                               ctypes.c_int, ctypes.c_uint]
        lib.dfft_slab_split_create.restype = ctypes.c_int
        self.key = (L, nslab, zr, nranks, dtype, bool(inverse), split_dim)
        self.esz = torch.empty((), dtype=dtype).element_size()
        h = ctypes.c_void_p()
        dev = device if device is not None else torch.cuda.current_device()
        with torch.cuda.device(dev):
            check(lib.dfft_slab_split_create(ctypes.byref(h), _precision(dtype), 1 if inverse else 0,
                                             L, nslab, zr, nranks, split_dim, 0))
        self._h = h

    def execute(self, src: torch.Tensor, src_off: int, dst: torch.Tensor, dst_off: int, stream=None):
        if stream is None:
            stream = torch.cuda.current_stream(src.device)
        s = stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream or 0)
        a = src.data_ptr() + src_off * self.esz
        b = dst.data_ptr() + dst_off * self.esz
        check(self._L.dfft_execute(self._h, ctypes.c_void_p(a), ctypes.c_void_p(b), ctypes.c_void_p(s)))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                self._L.dfft_plan_destroy(h)
            except Exception:
                pass
            self._h = None


class CudaSlabKernels:
    """The compute steps of ``FusedSlabFFT`` on the GPU: the split slab
    plans (one per group size and direction, cached) and the last-axis
    plan on the received array, in place."""

    def __init__(self):
        self._plans = {}

    def slab(self, inverse, src, src_off, dst, dst_off, L, nslab, zr, nranks, split_dim=2):
        key = (L, nslab, zr, nranks, src.dtype, bool(inverse), src.device, split_dim)
        p = self._plans.get(key)
        if p is None:
            p = self._plans[key] = SlabSplitPlan(L, nslab, zr, nranks, src.dtype, inverse, src.device,
                                                 split_dim)
        p.execute(src, src_off, dst, dst_off)

    def zpass(self, B: torch.Tensor, inverse: bool):
        t = IFFT_() if inverse else FFT_()
        p = get_or_create_gpu_plan(t, B, (3,))
        p.execute(B, B)

    def copy(self, dst: torch.Tensor, src: torch.Tensor):
        dst.copy_(src)

    def empty(self, n, dtype, device):
        return torch.empty(n, dtype=dtype, device=device)


def _nccl_exchange(ops, group):
    """Issue one grouped batch of sends / receives; the works to wait on."""
    import torch.distributed as dist
    if not ops:
        return []
    p2p = [dist.P2POp(dist.isend if kind == "send" else dist.irecv, t, peer, group=group)
           for kind, t, peer in ops]
    return dist.batch_isend_irecv(p2p)


class FusedSlabFFT:
    """3-D C2C FFT of an L x L x N3 ComplexF32/F64 array distributed in
    z-slabs over ``world`` ranks (L % world == 0), with the pack and unpack
    of the exchange folded into the slab pass (module docstring).

    ``split``: "x" -- B is split along dim 1, this rank's result chunk is
    (L / world, L, N3) (the reference's Slab layouts, Blocks(L, L, c) to
    Blocks(c, L, N3)); "y" -- split along dim 2, chunk (L, L / world, N3).
    ``forward(A, B)``: A = this rank's (L, L, |Z_r|) slab chunk (F-ordered;
    with split "x" it is overwritten, as the reference's in-place slab
    stage overwrites it), B = its chunk of the result, written.
    ``inverse(B, A)``: the reverse (B is transformed in place along dim 3
    first).  Every rank calls the same methods in the same order.
    ``exchange(ops, group)`` issues one batch of ("send" | "recv", tensor,
    peer) operations and returns works to wait on (default: NCCL through
    torch.distributed)."""

    def __init__(self, L: int, n3: int, dtype, rank: int, world: int, group=None, ngroups: int = 2,
                 kernels=None, exchange=None, device=None, split: str = "x"):
        if world < 1 or L % world != 0:
            raise ArgumentError(_lib.ERROR_INVALID_VALUE, "fused Slab exchange needs L % ranks == 0")
        if ngroups < 1:
            raise ArgumentError(_lib.ERROR_INVALID_VALUE, "ngroups must be >= 1")
        if split not in ("x", "y"):
            raise ArgumentError(_lib.ERROR_INVALID_VALUE, 'split must be "x" or "y"')
        self.split_dim = 1 if split == "x" else 2
        self.L, self.n3, self.dtype = int(L), int(n3), dtype
        self.rank, self.world, self.group = rank, world, group
        self.R = self.L // world
        self.zs = zsplit(self.n3, world)
        self.Zr = self.zs[rank][1]
        self.groups = [groups_of(self.zs[s][1], ngroups) for s in range(world)]
        self.kernels = kernels or CudaSlabKernels()
        self.exchange = exchange or _nccl_exchange
        if exchange is None and world > 1:
            # a collective first, so that every rank has joined the
            # communicator before the point-to-point batches (a rank's first
            # batch may be empty)
            import torch.distributed as dist
            dist.barrier(group=group)
        self.device = device
        # the split side of this rank's slab passes: every rank block of
        # every local slab (the send buffer forward, the receive buffer inverse)
        n = self.L * self.R * self.Zr * world
        self.buf = self.kernels.empty(n, dtype, device) if n else None

    def _blk(self, s: int, z0: int, n: int):
        """Rank s's block of local slabs [z0, z0 + n) in the split buffer."""
        LR = self.L * self.R
        a = (s * self.Zr + z0) * LR
        return self.buf[a:a + n * LR]

    def _col(self, Bf, s: int, z0: int, n: int):
        """Slabs [z0, z0 + n) of rank s's z-range in a flat (L, R, N3) chunk."""
        LR = self.L * self.R
        a = (self.zs[s][0] + z0) * LR
        return Bf[a:a + n * LR]

    def forward(self, A: torch.Tensor, B: torch.Tensor) -> torch.Tensor:
        L, R, r, P = self.L, self.R, self.rank, self.world
        Af = _flat(A) if self.Zr else None
        Bf = _flat(B)
        works = []
        for g in range(len(self.groups[r])):
            z0, n = self.groups[r][g]
            if n:
                self.kernels.slab(False, Af, z0 * L * L, self.buf, z0 * L * R, L, n, self.Zr, P,
                                  self.split_dim)
                self.kernels.copy(self._col(Bf, r, z0, n), self._blk(r, z0, n))
            ops = []
            for s in range(P):
                if s == r:
                    continue
                zs0, ns = self.groups[s][g]
                if ns:
                    ops.append(("recv", self._col(Bf, s, zs0, ns), s))
                if n:
                    ops.append(("send", self._blk(s, z0, n), s))
            works += self.exchange(ops, self.group)
        for w in works:
            w.wait()
        self.kernels.zpass(B, False)
        return B

    def inverse(self, B: torch.Tensor, A: torch.Tensor) -> torch.Tensor:
        L, R, r, P = self.L, self.R, self.rank, self.world
        Af = _flat(A) if self.Zr else None
        Bf = _flat(B)
        self.kernels.zpass(B, True)
        batches = []
        for g in range(len(self.groups[r])):
            z0, n = self.groups[r][g]
            ops = []
            for s in range(P):
                if s == r:
                    continue
                zs0, ns = self.groups[s][g]
                if n:
                    ops.append(("recv", self._blk(s, z0, n), s))
                if ns:
                    ops.append(("send", self._col(Bf, s, zs0, ns), s))
            if n:
                self.kernels.copy(self._blk(r, z0, n), self._col(Bf, r, z0, n))
            batches.append(self.exchange(ops, self.group))
        for g, works in enumerate(batches):
            for w in works:
                w.wait()
            z0, n = self.groups[r][g]
            if n:
                self.kernels.slab(True, self.buf, z0 * L * R, Af, z0 * L * L, L, n, self.Zr, P,
                                  self.split_dim)
        return A
