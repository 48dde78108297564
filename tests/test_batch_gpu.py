"""Batches of uneven transforms in one graph launch (or one persistent-kernel
launch on request) (configuration: 64
independent 3-D C2C ComplexF32 grids with edges from
{48,64,80,96,120,128,160,192}, plus a 2-D DCT-II/III Float64 stack), each
result checked against the oracle and against the same plan run alone."""
import numpy as np
import pytest
import torch

import dfft
import dfft_oracle as oracle
from helpers import rand, rel, to_gpu, to_np

pytestmark = pytest.mark.gpu

EDGES = [48, 64, 80, 96, 120, 128, 160, 192]


def _grids(n, seed=0):
    rng = np.random.default_rng(seed)
    return [tuple(int(e) for e in rng.choice(EDGES, 3)) for _ in range(n)]


@pytest.mark.parametrize("persistent", [False, True])
def test_batch_uneven_grids_match_oracle_and_alone(persistent):
    # default: the graph of the plans' own passes, bit-identical to each plan
    # run alone; persistent=True: one launch of the persistent batch kernel
    # (these lengths are all in its set), equal to rounding
    shapes = _grids(12, seed=1)
    arrays = [rand(s, np.complex64, seed=i, kind="uniform11") for i, s in enumerate(shapes)]
    ins = [to_gpu(a) for a in arrays]
    plans = [dfft.gpu_plan_transform(dfft.FFT(), g, (1, 2, 3), flags=dfft.FLAG_TUNE) for g in ins]
    outs = [dfft.empty_like_layout(p.out_shape, g.dtype, g) for p, g in zip(plans, ins)]
    b = dfft.Batch(plans, persistent=persistent)
    assert b.launches == (1 if persistent else sum(p.launches for p in plans))
    for rep in range(3):  # capture, then replays of the same graph
        b.execute(ins, outs)
        torch.cuda.synchronize()
        for a, o, p, g in zip(arrays, outs, plans, ins):
            assert rel(to_np(o), oracle.fft(a, dims=(1, 2, 3))) <= 1e-5
            alone = dfft.empty_like_layout(p.out_shape, g.dtype, g)
            p.execute(g, alone)
            if not persistent:
                assert torch.equal(alone, o), "batched result differs from the plan run alone"
            else:  # other kernels than the plan's: equal to rounding
                assert rel(to_np(o), to_np(alone)) <= 1e-6
    # new buffers: the graph is updated, results follow the new inputs
    ins2 = [to_gpu(rand(s, np.complex64, seed=100 + i)) for i, s in enumerate(shapes)]
    b.execute(ins2, outs)
    torch.cuda.synchronize()
    for g, o in zip(ins2, outs):
        assert rel(to_np(o), oracle.fft(to_np(g), dims=(1, 2, 3))) <= 1e-5


def test_batch_mixes_kinds_and_precisions():
    a = rand((64, 48, 32), np.complex64, seed=3)
    r = rand((256, 256, 8), np.float64, seed=4)
    d = rand((128, 96), np.float64, seed=5)
    ga, gr, gd = to_gpu(a), to_gpu(r), to_gpu(d)
    pa = dfft.gpu_plan_transform(dfft.IFFT(), ga, (1, 2, 3))
    pr = dfft.gpu_plan_transform(dfft.RFFT(), gr, (1, 2))
    pd = dfft.gpu_plan_transform(dfft.R2R((dfft.REDFT10, dfft.REDFT10)), gd, (1, 2))
    outs = [dfft.empty_like_layout(p.out_shape, dt, g) for p, dt, g in
            ((pa, torch.complex64, ga), (pr, torch.complex128, gr), (pd, torch.float64, gd))]
    dfft.Batch([pa, pr, pd]).execute([ga, gr, gd], outs)
    torch.cuda.synchronize()
    assert rel(to_np(outs[0]), oracle.ifft(a, dims=(1, 2, 3))) <= 1e-5
    assert rel(to_np(outs[1]), oracle.rfft(r, dims=(1, 2))) <= 1e-12
    assert rel(to_np(outs[2]), oracle.fft(d, dims=(1, 2), transforms=(oracle.R2R((oracle.REDFT10, oracle.REDFT10)),))) <= 1e-12


@pytest.mark.parametrize("lag", [0, 1, 3])
def test_persistent_batch_inverse_and_float64(lag):
    # inverse transforms (reverse stage order, 1/N) and ComplexF64, 2-D and 3-D
    shapes = [(48, 64, 40), (96, 24), (160, 120, 16), (32, 256, 16)]
    for dt, tol in ((np.complex64, 1e-5), (np.complex128, 1e-12)):
        arrays = [rand(s, dt, seed=7 + i) for i, s in enumerate(shapes)]
        ins = [to_gpu(a) for a in arrays]
        plans = [dfft.gpu_plan_transform(dfft.IFFT(), g, tuple(range(1, g.dim() + 1))) for g in ins]
        outs = [dfft.empty_like_layout(p.out_shape, g.dtype, g) for p, g in zip(plans, ins)]
        b = dfft.Batch(plans, persistent=True, lag=lag)
        assert b.launches == 1
        for _ in range(2):
            b.execute(ins, outs)
            torch.cuda.synchronize()
            for a, o in zip(arrays, outs):
                assert rel(to_np(o), oracle.ifft(a, dims=tuple(range(1, a.ndim + 1)))) <= tol
    assert dfft.device_error() == 0


def test_persistent_batch_falls_back_to_graph():
    # a length outside the persistent kernel's set (7 * 11): the graph form
    a = rand((77, 32, 8), np.complex64, seed=1)
    g = to_gpu(a)
    p = dfft.gpu_plan_transform(dfft.FFT(), g, (1, 2, 3))
    b = dfft.Batch([p], persistent=True)
    assert b.launches == p.launches
    o = dfft.empty_like_layout(p.out_shape, g.dtype, g)
    b.execute([g], [o])
    torch.cuda.synchronize()
    assert rel(to_np(o), oracle.fft(a, dims=(1, 2, 3))) <= 1e-5
