"""The fused multi-rank Slab exchange (dfft.slab_dist) on CPU ranks (gloo,
world sizes 2 and 3): slab groups, rank blocks of the split layout, the
grouped sends / receives in both directions, uneven and empty z-ranges,
end to end against the oracle's fftn, with a CPU double of the split slab
pass and the last-axis pass (the GPU path runs libdfft's kernels; the
split layout itself is checked on the GPU in test_slab_exchange_gpu.py)."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


class CpuSlabKernels:
    """Test double for dfft.slab_dist.CudaSlabKernels: torch.fft on CPU,
    writing / reading the rank-split layout row by row."""

    def slab(self, inverse, src, src_off, dst, dst_off, L, nslab, zr, nranks, split_dim=2):
        from dfft.slab_dist import split_col, split_row
        R = L // nranks

        def spans(z, y):
            # (destination start, source columns) of row y of slab z, per piece
            if split_dim == 2:
                r = split_row(R, zr, z, y)
                return [(r * L, slice(0, L))]
            return [(split_col(R, L, zr, z, y, s * R), slice(s * R, (s + 1) * R)) for s in range(nranks)]

        if not inverse:
            x = src[src_off:src_off + L * L * nslab].reshape(nslab, L, L).permute(2, 1, 0)
            F = torch.fft.fftn(x, dim=(0, 1))
            for z in range(nslab):
                for y in range(L):
                    for o, cols in spans(z, y):
                        n = cols.stop - cols.start
                        dst[dst_off + o:dst_off + o + n] = F[cols, y, z]
        else:
            x = torch.empty((L, L, nslab), dtype=src.dtype)
            for z in range(nslab):
                for y in range(L):
                    for o, cols in spans(z, y):
                        n = cols.stop - cols.start
                        x[cols, y, z] = src[src_off + o:src_off + o + n]
            F = torch.fft.ifftn(x, dim=(0, 1))
            dst[dst_off:dst_off + L * L * nslab] = F.permute(2, 1, 0).reshape(-1)

    def zpass(self, B, inverse):
        B.copy_(torch.fft.ifft(B, dim=2) if inverse else torch.fft.fft(B, dim=2))

    def copy(self, dst, src):
        dst.copy_(src)

    def empty(self, n, dtype, device):
        return torch.empty(n, dtype=dtype)


def _fcol(t):
    """A column-major (F-ordered) copy of t."""
    return t.permute(2, 1, 0).contiguous().permute(2, 1, 0)


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
        import dfft_oracle as oracle
        from dfft.slab_dist import FusedSlabFFT, zsplit
        for (L, n3, ngroups, split) in cases:
            g = torch.Generator().manual_seed(L * 100 + n3)
            A = torch.complex(torch.rand((L, L, n3), dtype=torch.float64, generator=g),
                              torch.rand((L, L, n3), dtype=torch.float64, generator=g))
            ref = torch.from_numpy(oracle.fft(A.numpy(), dims=(1, 2, 3)))
            fs = FusedSlabFFT(L, n3, A.dtype, rank, world, ngroups=ngroups, kernels=CpuSlabKernels(),
                              device=torch.device("cpu"), split=split)
            z0, nz = zsplit(n3, world)[rank]
            R = L // world
            Ar = _fcol(A[:, :, z0:z0 + nz])
            Br = _fcol(torch.zeros((R, L, n3) if split == "x" else (L, R, n3), dtype=A.dtype))
            fs.forward(Ar, Br)
            exp = ref[rank * R:(rank + 1) * R] if split == "x" else ref[:, rank * R:(rank + 1) * R, :]
            err = oracle.rel_l2(Br.numpy(), exp.numpy())
            assert err <= 1e-12, (L, n3, ngroups, "forward", err)
            A2 = _fcol(torch.zeros((L, L, nz), dtype=A.dtype))
            fs.inverse(Br, A2)
            if nz:
                err = oracle.rel_l2(A2.numpy(), A[:, :, z0:z0 + nz].numpy())
                assert err <= 1e-12, (L, n3, ngroups, "inverse", err)
        q.put((rank, "ok"))
    except Exception as e:  # report to the parent instead of hanging it
        import traceback
        q.put((rank, repr(e) + traceback.format_exc()[-800:]))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_fused_slab_exchange_across_ranks(world):
    # (L, N3, slab groups, split): even and uneven z-ranges, a rank with no
    # slabs (N3 < world), more groups than some ranks have slabs, columns
    # (the reference's layouts) or rows split by rank
    cases = [(12, 8, 2, "y"), (12, 7, 2, "x"), (12, 5, 3, "y"), (12, 2, 1, "x"), (6, 9, 4, "x"),
             (12, 8, 2, "x")]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, cases, q)) for r in range(world)]
    for p in procs:
        p.start()
    results = {}
    for _ in range(world):
        r, msg = q.get(timeout=180)
        results[r] = msg
    for p in procs:
        p.join(timeout=60)
    assert all(v == "ok" for v in results.values()), results


def test_groups_and_split_rows():
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, os.path.join(root, "daggerfft.jl_b200"))
    from dfft.slab_dist import groups_of, split_col, split_row, zsplit
    assert zsplit(7, 3) == [(0, 3), (3, 3), (6, 1)]
    assert zsplit(2, 3) == [(0, 1), (1, 1), (2, 0)]
    assert groups_of(5, 2) == [(0, 3), (3, 2)]
    assert groups_of(1, 3) == [(0, 1), (1, 0), (1, 0)]
    assert groups_of(0, 2) == [(0, 0), (0, 0)]
    # every (slab, row) lands in its own row, rank s's rows of every slab form
    # one block [s*zr*R, (s+1)*zr*R)
    L, P, zr = 12, 3, 4
    R = L // P
    rows = sorted(split_row(R, zr, z, y) for z in range(zr) for y in range(L))
    assert rows == list(range(L * zr))
    for z in range(zr):
        for y in range(L):
            s = y // R
            assert s * zr * R <= split_row(R, zr, z, y) < (s + 1) * zr * R
    # column split: rank s's block is [s * zr * R * L, (s + 1) * zr * R * L)
    offs = sorted(split_col(R, L, zr, z, y, x) for z in range(zr) for y in range(L) for x in range(L))
    assert offs == list(range(L * L * zr))
    for z in range(zr):
        for y in range(L):
            for x in range(L):
                s = x // R
                assert s * zr * R * L <= split_col(R, L, zr, z, y, x) < (s + 1) * zr * R * L
