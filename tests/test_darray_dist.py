"""Multi-rank logic on CPU ranks (gloo, world sizes 2 and 3): the pattern
walk, flat per-peer buffers in walk order, the batched isend/irecv exchange
and unpacking, and the Pencil / Slab gpu_fft_ / gpu_ifft_ drivers end to end,
with a CPU copier and a CPU stage standing in for the CUDA copy kernels and
the per-chunk plans (the GPU path runs them through libdfft)."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


class CpuCopier:
    """Test double for dfft.CudaCopier: the same copies with torch slicing."""

    def prepare(self, ws, src, dst):
        pass

    def run(self, ws, phase, src, dst):
        from dfft.darray import _peer_base
        if phase == "local":
            for p in ws.local_patterns:
                s, d = p.src_indices, p.dst_indices
                dst.chunks[p.dst_idx][d[0].start:d[0].stop, d[1].start:d[1].stop, d[2].start:d[2].stop] = \
                    src.chunks[p.src_idx][s[0].start:s[0].stop, s[1].start:s[1].stop, s[2].start:s[2].stop]
        elif phase == "pack":
            base = _peer_base(ws.send_sizes, ws.send_ranks)
            for peer in ws.send_ranks:
                for p in ws.send_peers[peer]:
                    s = p.src_indices
                    blk = src.chunks[p.src_idx][s[0].start:s[0].stop, s[1].start:s[1].stop, s[2].start:s[2].stop]
                    o = base[peer] + p.buffer_offset
                    ws.send_buffer[o:o + p.buffer_size] = blk.permute(2, 1, 0).reshape(-1)
        elif phase == "unpack":
            base = _peer_base(ws.recv_sizes, ws.recv_ranks)
            for peer in ws.recv_ranks:
                for p in ws.recv_peers[peer]:
                    d = p.dst_indices
                    cnt = tuple(len(r) for r in d)
                    o = base[peer] + p.buffer_offset
                    blk = ws.recv_buffer[o:o + p.buffer_size].reshape(cnt[2], cnt[1], cnt[0]).permute(2, 1, 0)
                    dst.chunks[p.dst_idx][d[0].start:d[0].stop, d[1].start:d[1].stop, d[2].start:d[2].stop] = blk


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, cases, q):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, os.path.join(root, "daggerfft.jl_b200"))
    sys.path.insert(0, os.path.join(root, "oracle"))
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import dfft
        import dfft_oracle as oracle
        cpu = torch.device("cpu")
        for (shape, bsrc, bdst) in cases:
            g = torch.Generator().manual_seed(7)
            A = torch.randn(shape, dtype=torch.complex64, generator=g)
            DA = dfft.distribute(A, dfft.Blocks(*bsrc), rank=rank, world=world, device=cpu)
            DB = dfft.empty_darray(shape, dfft.Blocks(*bdst), A.dtype, device=cpu, rank=rank, world=world)
            cop = CpuCopier()
            ws = dfft.create_gpu_workspace(DA, DB, copier=cop)
            # same walk as the oracle's restatement of create_workspace
            ows = oracle.create_workspace(oracle.blocks(shape, bsrc, world), oracle.blocks(shape, bdst, world), rank)
            assert ws.send_sizes == ows.send_sizes and ws.recv_sizes == ows.recv_sizes
            dfft.gpu_coalesced_redistribute_(DB, DA, ws, copier=cop)
            for i in DB.local_indices:
                d = DB.subdomains[i]
                exp = A[d[0].start:d[0].stop, d[1].start:d[1].stop, d[2].start:d[2].stop]
                assert torch.equal(DB.chunks[i], exp), (shape, bsrc, bdst, i)
        q.put((rank, "ok"))
    except Exception as e:  # report to the parent instead of hanging it
        q.put((rank, repr(e)))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_redistribute_across_ranks(world):
    cases = [((8, 6, 4), (8, 6, 1), (2, 6, 4)),      # slab -> slab
             ((8, 8, 8), (8, 4, 4), (4, 8, 4)),      # pencil x -> pencil y
             ((10, 9, 7), (10, 3, 2), (3, 9, 3))]    # ragged blocks
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, cases, q)) for r in range(world)]
    for p in procs:
        p.start()
    results = {}
    for _ in range(world):
        r, msg = q.get(timeout=120)
        results[r] = msg
    for p in procs:
        p.join(timeout=60)
    assert all(v == "ok" for v in results.values()), results


def cpu_stage(D, transform, dims):
    """Test double for the per-chunk plans: torch.fft on CPU chunks, in place
    (forward unnormalised, inverse 1/n, as the GPU plans)."""
    import dfft
    axes = tuple(d - 1 for d in dims)
    inverse = isinstance(transform, (dfft.IFFT, dfft.IFFT_))
    for i in D.local_indices:
        c = D.chunks[i]
        c.copy_(torch.fft.ifftn(c, dim=axes) if inverse else torch.fft.fftn(c, dim=axes))


def _driver_worker(rank, world, port, cases, q):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, os.path.join(root, "daggerfft.jl_b200"))
    sys.path.insert(0, os.path.join(root, "oracle"))
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import dfft
        import dfft_oracle as oracle
        cpu = torch.device("cpu")
        for (decomp, shape, c) in cases:
            g = torch.Generator().manual_seed(11)
            A = torch.complex(torch.rand(shape, dtype=torch.float64, generator=g),
                              torch.rand(shape, dtype=torch.float64, generator=g))
            ref = oracle.fft(A.numpy(), dims=(1, 2, 3))
            cop = CpuCopier()
            n1, n2, n3 = shape
            if decomp == "pencil":
                DA = dfft.distribute(A, dfft.Blocks(n1, c, c), rank=rank, world=world, device=cpu)
                DB = dfft.empty_darray(shape, dfft.Blocks(c, n2, c), A.dtype, device=cpu, rank=rank, world=world)
                DC = dfft.empty_darray(shape, dfft.Blocks(c, c, n3), A.dtype, device=cpu, rank=rank, world=world)
                wsAB = dfft.create_gpu_workspace(DA, DB, copier=cop)
                wsBC = dfft.create_gpu_workspace(DB, DC, copier=cop)
                dfft.gpu_fft_(DC, DA, DB, wsAB, wsBC, (dfft.FFT_(),) * 3, (1, 2, 3), dfft.Pencil(),
                              stage=cpu_stage, copier=cop)
                out = DC
            else:
                DA = dfft.distribute(A, dfft.Blocks(n1, n2, c), rank=rank, world=world, device=cpu)
                DB = dfft.empty_darray(shape, dfft.Blocks(c, n2, n3), A.dtype, device=cpu, rank=rank, world=world)
                wsAB = dfft.create_gpu_workspace(DA, DB, copier=cop)
                dfft.gpu_fft_(DB, DA, wsAB, (dfft.FFT_(),) * 3, (1, 2, 3), dfft.Slab(), stage=cpu_stage,
                              copier=cop)
                out = DB
            for i in out.local_indices:
                d = out.subdomains[i]
                exp = ref[d[0].start:d[0].stop, d[1].start:d[1].stop, d[2].start:d[2].stop]
                err = oracle.rel_l2(out.chunks[i].numpy(), exp)
                assert err <= 1e-12, (decomp, shape, i, err)
            # and back: the inverse drivers (reverse stage order) restore A
            if decomp == "pencil":
                wsCB = dfft.create_gpu_workspace(DC, DB, copier=cop)
                wsBA = dfft.create_gpu_workspace(DB, DA, copier=cop)
                # gpu_ifft!(C=DA, A=DC, B=DB, wsAB=wsCB, wsBC=wsBA, ...): stages on DC, DB, DA
                dfft.gpu_ifft_(DA, DC, DB, wsCB, wsBA, (dfft.IFFT_(),) * 3, (1, 2, 3), dfft.Pencil(),
                               stage=cpu_stage, copier=cop)
            else:
                wsBA = dfft.create_gpu_workspace(DB, DA, copier=cop)
                dfft.gpu_ifft_(DA, DB, wsBA, (dfft.IFFT_(),) * 3, (1, 2, 3), dfft.Slab(), stage=cpu_stage,
                               copier=cop)
            for i in DA.local_indices:
                d = DA.subdomains[i]
                exp = A[d[0].start:d[0].stop, d[1].start:d[1].stop, d[2].start:d[2].stop]
                err = oracle.rel_l2(DA.chunks[i].numpy(), exp.numpy())
                assert err <= 1e-12, (decomp, shape, "inverse", i, err)
        q.put((rank, "ok"))
    except Exception as e:  # report to the parent instead of hanging it
        import traceback
        q.put((rank, repr(e) + traceback.format_exc()[-800:]))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_fft_drivers_across_ranks(world):
    """gpu_fft_ / gpu_ifft_ (Pencil and Slab stage order, src/fftgpu.jl:498-619)
    end to end across gloo ranks: every stage, every exchange, against the
    oracle's fftn of the whole array."""
    cases = [("pencil", (12, 10, 8), 4), ("slab", (12, 10, 8), 3), ("pencil", (9, 7, 5), 3)]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_driver_worker, args=(r, world, port, cases, q)) for r in range(world)]
    for p in procs:
        p.start()
    results = {}
    for _ in range(world):
        r, msg = q.get(timeout=120)
        results[r] = msg
    for p in procs:
        p.join(timeout=60)
    assert all(v == "ok" for v in results.values()), results
