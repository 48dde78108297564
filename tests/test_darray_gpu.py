"""DArray front end on one GPU: Blocks layouts, create_gpu_workspace, the
one-launch redistribution and the Pencil/Slab gpu_fft!/gpu_ifft! drivers
(src/fftgpu.jl:126-619) against the oracle's restatement of the same
pipeline and against fftn."""
import numpy as np
import pytest
import torch

import dfft
import dfft_oracle as oracle
from helpers import rand, rel, to_gpu, to_np

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,c", [((32, 32, 32), 8), ((48, 40, 24), 16), ((64, 64, 64), 32)])
@pytest.mark.parametrize("dtype", [np.complex64, np.complex128])
def test_pencil_pipeline(n, c, dtype):
    a = rand(n, dtype, seed=c)
    A = to_gpu(a)
    N1, N2, N3 = n
    DA = dfft.distribute(A, dfft.Blocks(N1, c, c))
    DB = dfft.empty_darray(n, dfft.Blocks(c, N2, c), A.dtype)
    DC = dfft.empty_darray(n, dfft.Blocks(c, c, N3), A.dtype)
    wsAB = dfft.create_gpu_workspace(DA, DB)
    wsBC = dfft.create_gpu_workspace(DB, DC)
    wsCB = dfft.create_gpu_workspace(DC, DB)
    wsBA = dfft.create_gpu_workspace(DB, DA)
    # one rank: every overlap is a local copy, c^3-sized blocks
    assert not wsAB.send_peers and not wsAB.recv_peers
    cd = lambda n: -(-n // c)
    assert len(wsAB.local_patterns) == cd(N2) * cd(N3) * cd(N1)
    dfft.gpu_fft_(DC, DA, DB, wsAB, wsBC, (dfft.FFT_(),) * 3, (1, 2, 3), dfft.Pencil())
    tol = 1e-5 if dtype == np.complex64 else 1e-12
    assert rel(to_np(dfft.collect(DC)), oracle.fft(a, dims=(1, 2, 3))) <= tol
    dfft.gpu_ifft_(DA, DC, DB, wsCB, wsBA, (dfft.IFFT_(),) * 3, (1, 2, 3), dfft.Pencil())
    assert rel(to_np(dfft.collect(DA)), a) <= tol


@pytest.mark.parametrize("n,c", [((32, 24, 16), 4), ((64, 64, 64), 16)])
def test_slab_pipeline(n, c):
    a = rand(n, np.complex64, seed=2)
    A = to_gpu(a)
    N1, N2, N3 = n
    DA = dfft.distribute(A, dfft.Blocks(N1, N2, c))
    DB = dfft.empty_darray(n, dfft.Blocks(c, N2, N3), A.dtype)
    wsAB = dfft.create_gpu_workspace(DA, DB)
    wsBA = dfft.create_gpu_workspace(DB, DA)
    dfft.gpu_fft_(DB, DA, wsAB, (dfft.FFT_(),) * 3, (1, 2, 3), dfft.Slab())
    assert rel(to_np(dfft.collect(DB)), oracle.fft(a, dims=(1, 2, 3))) <= 1e-5
    dfft.gpu_ifft_(DA, DB, wsBA, (dfft.IFFT_(),) * 3, (1, 2, 3), dfft.Slab())
    assert rel(to_np(dfft.collect(DA)), a) <= 1e-5


def test_redistribute_is_exact_copy():
    # the redistribution itself is a byte-exact copy (ragged blocks too)
    n = (30, 22, 14)
    a = rand(n, np.complex128, seed=3)
    A = to_gpu(a)
    DA = dfft.distribute(A, dfft.Blocks(30, 7, 5))
    DB = dfft.empty_darray(n, dfft.Blocks(4, 22, 6), A.dtype)
    ws = dfft.create_gpu_workspace(DA, DB)
    dfft.gpu_coalesced_redistribute_(DB, DA, ws)
    assert np.array_equal(to_np(dfft.collect(DB)), a)
    assert ws.plans["local"].bytes() == a.size * 16


def test_patterns_match_oracle():
    n = (24, 18, 12)
    A = torch.zeros(n, dtype=torch.complex64, device="cuda")
    DA = dfft.distribute(A, dfft.Blocks(24, 6, 4))
    DB = dfft.empty_darray(n, dfft.Blocks(8, 18, 4), A.dtype)
    ws = dfft.create_gpu_workspace(DA, DB)
    oA = oracle.blocks(n, (24, 6, 4))
    oB = oracle.blocks(n, (8, 18, 4))
    ows = oracle.create_workspace(oA, oB, 0)
    got = [(p.src_idx, p.dst_idx, p.src_indices, p.dst_indices, p.buffer_size) for p in ws.local_patterns]
    exp = [(p.src_idx, p.dst_idx, p.src_indices, p.dst_indices, p.buffer_size) for p in ows.local_patterns]
    assert got == exp
