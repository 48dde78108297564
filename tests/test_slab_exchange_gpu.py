"""The fused multi-rank Slab exchange with libdfft's kernels: P ranks run
as host threads on one GPU, exchanging through an in-process mailbox (a
receive waits on the host for its matching send, then copies on the
device), so the split-layout slab pass, the groups and the last-axis pass
all run as they would across GPUs.  No kernel waits on another.  Results
against the oracle's FP64 fftn, forward and inverse."""
import collections
import threading

import numpy as np
import pytest
import torch

import dfft
import dfft_oracle as oracle
from dfft.slab_dist import FusedSlabFFT, zsplit
from helpers import rand, tol_for

pytestmark = pytest.mark.gpu


class LoopbackFabric:
    """Point-to-point messages between threads of one process, matched in
    order per (sender, receiver) pair as NCCL matches them."""

    def __init__(self):
        self.mail = collections.defaultdict(collections.deque)
        self.cv = threading.Condition()

    def exchange_for(self, rank):
        fabric = self

        class _Recv:
            def __init__(self, src, t):
                self.src, self.t = src, t

            def wait(self):
                with fabric.cv:
                    ok = fabric.cv.wait_for(lambda: fabric.mail[(self.src, rank)], timeout=120)
                    assert ok, f"rank {rank}: no message from {self.src}"
                    t = fabric.mail[(self.src, rank)].popleft()
                self.t.copy_(t)

        def ex(ops, group):
            works = []
            for kind, t, peer in ops:
                if kind == "send":
                    with fabric.cv:
                        fabric.mail[(rank, peer)].append(t)
                        fabric.cv.notify_all()
                else:
                    works.append(_Recv(peer, t))
            return works
        return ex


def _fcol_cuda(a):
    return torch.from_numpy(np.ascontiguousarray(a.T)).cuda().permute(2, 1, 0)


def _run_ranks(world, fn):
    errs = []

    def body(r):
        try:
            torch.cuda.set_device(0)
            fn(r)
        except BaseException as e:  # reported below
            errs.append((r, repr(e)))

    ts = [threading.Thread(target=body, args=(r,)) for r in range(world)]
    for t in ts:
        t.start()
    for t in ts:
        t.join(timeout=300)
    assert not errs, errs


@pytest.mark.parametrize("split", ["x", "y"])
@pytest.mark.parametrize("L,n3,world,ngroups,dtype", [
    (512, 64, 2, 2, np.complex64),
    (512, 48, 4, 3, np.complex64),     # R = 128 rows / columns per rank
    (256, 30, 4, 2, np.complex64),     # uneven z-ranges (8, 8, 8, 6)
    (256, 20, 2, 2, np.complex128),
    (512, 3, 4, 2, np.complex64),      # a rank with no slabs
    (512, 12, 2, 3, np.complex128),    # ComplexF64 L = 512 (16-byte elements, 8 x 8 x 8 slab kernel)
])
def test_fused_slab_exchange_loopback(L, n3, world, ngroups, dtype, split):
    a = rand((L, L, n3), dtype, seed=L + n3 + world)
    ref = oracle.fft(a, dims=(1, 2, 3))
    fabric = LoopbackFabric()
    R = L // world
    tdt = torch.complex64 if dtype == np.complex64 else torch.complex128
    outs, backs = {}, {}

    def rank_body(r):
        fs = FusedSlabFFT(L, n3, tdt, r, world, ngroups=ngroups, exchange=fabric.exchange_for(r),
                          device=torch.device("cuda", 0), split=split)
        z0, nz = zsplit(n3, world)[r]
        Ar = _fcol_cuda(a[:, :, z0:z0 + nz])
        Br = _fcol_cuda(np.zeros((R, L, n3) if split == "x" else (L, R, n3), dtype))
        fs.forward(Ar, Br)
        torch.cuda.synchronize()
        outs[r] = Br.cpu().numpy()
        A2 = _fcol_cuda(np.zeros((L, L, nz), dtype))
        fs.inverse(Br, A2)
        torch.cuda.synchronize()
        backs[r] = A2.cpu().numpy()

    _run_ranks(world, rank_body)
    tol = tol_for(dtype)
    got = np.concatenate([outs[r] for r in range(world)], axis=0 if split == "x" else 1)
    assert oracle.rel_l2(got, ref) <= tol
    back = np.concatenate([backs[r] for r in range(world) if backs[r].size], axis=2)
    assert oracle.rel_l2(back, a) <= tol
    assert dfft.device_error() == 0


def test_darray_slab_takes_fused_path():
    # the reference's Slab layouts on one rank: Blocks(L, L, N3) ->
    # Blocks(L, L, N3) goes through the fused slab pass (columns split,
    # y-phase first), forward and inverse, against the oracle
    L, n3 = 256, 24
    a = rand((L, L, n3), np.complex64, seed=77)
    A = torch.from_numpy(a)
    DA = dfft.distribute(A.cuda(), dfft.Blocks(L, L, n3))
    DB = dfft.empty_darray((L, L, n3), dfft.Blocks(L, L, n3), A.dtype)
    ws = dfft.create_gpu_workspace(DA, DB)
    dfft.gpu_fft_(DB, DA, ws, (dfft.FFT_(),) * 3, (1, 2, 3), dfft.Slab())
    torch.cuda.synchronize()
    assert getattr(ws, "_fused", None) is not None
    out = DB.chunks[DB.local_indices[0]].cpu().numpy()
    assert oracle.rel_l2(out, oracle.fft(a, dims=(1, 2, 3))) <= 1e-5
    wsBA = dfft.create_gpu_workspace(DB, DA)
    dfft.gpu_ifft_(DA, DB, wsBA, (dfft.IFFT_(),) * 3, (1, 2, 3), dfft.Slab())
    torch.cuda.synchronize()
    assert getattr(wsBA, "_fused", None) is not None
    back = DA.chunks[DA.local_indices[0]].cpu().numpy()
    assert oracle.rel_l2(back, a) <= 1e-5


def test_split_plan_rejects_bad_splits():
    g = torch.zeros(1, dtype=torch.complex64, device="cuda")
    from dfft.slab_dist import SlabSplitPlan
    with pytest.raises(dfft.ArgumentError):
        SlabSplitPlan(512, 4, 4, 3, torch.complex64, False)     # 512 % 3 != 0
    with pytest.raises(dfft.ArgumentError):
        SlabSplitPlan(512, 8, 4, 2, torch.complex64, False)     # zr < nslab
    with pytest.raises(dfft.ArgumentError):
        SlabSplitPlan(512, 4, 4, 256, torch.complex64, False)   # 2 rows per rank < one tile
    with pytest.raises(dfft.ArgumentError):
        SlabSplitPlan(512, 4, 4, 256, torch.complex64, False, split_dim=1)  # 2 columns per rank
    with pytest.raises(dfft.ArgumentError):
        SlabSplitPlan(512, 4, 4, 2, torch.complex64, False, split_dim=3)
    del g
