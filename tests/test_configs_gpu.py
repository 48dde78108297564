"""The configured workloads at their full sizes, each checked against the
FP64 host oracle (pocketfft in float64 on all host cores) on the same
seeded input, plus the round trip:

  * 128^3 ComplexF64 fft + ifft, Pencil, real and imaginary parts U[0,1)
  * 256^3 Float64 and Float32 rfft + irfft, Pencil, U[0,1)
  * 512^3 ComplexF32 fft + ifft, Slab, real and imaginary parts N(0,1)
    (the fused dims-(1,2) slab pass and the dim-3 pass)
  * 64 independent ComplexF32 grids with edges from
    {48,64,80,96,120,128,160,192}, U[-1,1), as one batch launch, and the
    2-D DCT-II / DCT-III Float64 256 x 256 x 32 stack

Bounds: relative L2 <= 1e-5 (ComplexF32 / Float32) and <= 1e-12
(ComplexF64 / Float64) against the oracle; the inverse is checked on the
GPU's own forward output against the oracle's inverse of that same data.
The reference stage order is src/fftgpu.jl:534-557,596-619 (Slab) and
src/fftgpu.jl:498-531,560-593 (Pencil)."""
import os

import numpy as np
import pytest
import torch

import dfft
import dfft_oracle as oracle
from helpers import to_gpu, to_np

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _all_host_threads():
    old = oracle.WORKERS
    oracle.WORKERS = os.cpu_count() or 1
    yield
    oracle.WORKERS = old


def rel64(a, b, chunk_elems=1 << 24):
    """Relative L2 of a against b (same logical shape, any memory order),
    accumulated in float64 over slabs of the last axis (the oracle's
    long-double rel_l2 is too slow and too large at 512^3)."""
    a = np.asarray(a)
    b = np.asarray(b)
    assert a.shape == b.shape, (a.shape, b.shape)
    per = max(1, a.size // a.shape[-1])
    step = max(1, chunk_elems // per)
    wide = np.complex128 if (np.iscomplexobj(a) or np.iscomplexobj(b)) else np.float64
    num = den = 0.0
    for k in range(0, a.shape[-1], step):
        x = a[..., k:k + step].astype(wide)
        y = b[..., k:k + step].astype(wide)
        num += float(np.sum(np.abs(x - y) ** 2))
        den += float(np.sum(np.abs(y) ** 2))
    return float(np.sqrt(num / den))


def test_c2c_f64_128cube_pencil():
    n = 128
    a = oracle.make_input("uniform01", (n, n, n), 1, np.complex128)
    g = to_gpu(a)
    F = dfft.fft(g, decomp=dfft.Pencil(), dims=(1, 2, 3))
    Fh = to_np(F)
    assert rel64(Fh, oracle.fft(a, dims=(1, 2, 3))) <= 1e-12
    B = dfft.ifft(F, decomp=dfft.Pencil(), dims=(1, 2, 3))
    assert rel64(to_np(B), oracle.ifft(Fh, dims=(1, 2, 3))) <= 1e-12
    assert rel64(to_np(B), a) <= 1e-12


@pytest.mark.parametrize("dt,tol", [(np.float64, 1e-12), (np.float32, 1e-5)])
def test_rfft_irfft_256cube_pencil(dt, tol):
    n = 256
    a = oracle.make_input("uniform01", (n, n, n), 2, dt)
    g = to_gpu(a)
    R = dfft.rfft(g, decomp=dfft.Pencil(), dims=(1, 2, 3))
    Rh = to_np(R)
    assert Rh.shape == (n // 2 + 1, n, n)
    assert rel64(Rh, oracle.rfft(a, dims=(1, 2, 3))) <= tol
    X = dfft.irfft(R, n, decomp=dfft.Pencil(), dims=(1, 2, 3))
    assert rel64(to_np(X), oracle.irfft(Rh, n, dims=(1, 2, 3))) <= tol
    assert rel64(to_np(X), a) <= tol


def test_c2c_f32_512cube_slab():
    n = 512
    a = oracle.make_input("normal", (n, n, n), 3, np.complex64)
    g = to_gpu(a)
    del a
    p = dfft.gpu_plan_transform(dfft.FFT(), g, (1, 2, 3), decomp=dfft.Slab())
    F = dfft.empty_like_layout(p.out_shape, g.dtype, g)
    p.execute(g, F)
    ah = to_np(g)
    Fh = to_np(F)
    ref = oracle.fft(ah, dims=(1, 2, 3))
    e_fwd = rel64(Fh, ref)
    del ref
    pi = dfft.gpu_plan_transform(dfft.IFFT(), F, (1, 2, 3), decomp=dfft.Slab())
    B = dfft.empty_like_layout(pi.out_shape, F.dtype, F)
    pi.execute(F, B)
    Bh = to_np(B)
    e_rt = rel64(Bh, ah)
    ref_inv = oracle.ifft(Fh, dims=(1, 2, 3))
    e_inv = rel64(Bh, ref_inv)
    del ref_inv
    print(f"512^3 ComplexF32 Slab: fwd {e_fwd:.3e} inv {e_inv:.3e} roundtrip {e_rt:.3e} "
          f"({p.launches}+{pi.launches} launches)")
    assert e_fwd <= 1e-5 and e_inv <= 1e-5 and e_rt <= 1e-5
    assert dfft.device_error() == 0


def test_batch_64_uneven_grids_and_dct_stack():
    edges = [48, 64, 80, 96, 120, 128, 160, 192]
    rng = np.random.default_rng(4)
    shapes = [tuple(int(e) for e in rng.choice(edges, 3)) for _ in range(64)]
    arrays = [oracle.make_input("uniform11", s, 100 + i, np.complex64) for i, s in enumerate(shapes)]
    ins = [to_gpu(x) for x in arrays]
    plans = [dfft.gpu_plan_transform(dfft.FFT(), x, (1, 2, 3)) for x in ins]
    outs = [dfft.empty_like_layout(p.out_shape, x.dtype, x) for p, x in zip(plans, ins)]
    b = dfft.Batch(plans)
    b.execute(ins, outs)
    torch.cuda.synchronize()
    worst = max(rel64(to_np(o), oracle.fft(x, dims=(1, 2, 3))) for o, x in zip(outs, arrays))
    assert worst <= 1e-5
    d = oracle.make_input("uniform01", (256, 256, 32), 5, np.float64)
    gd = to_gpu(d)
    E = dfft.fft(gd, transforms=(dfft.R2R((dfft.REDFT10, dfft.REDFT10)),), dims=(1, 2))
    Eh = to_np(E)
    R2 = oracle.R2R((oracle.REDFT10, oracle.REDFT10))
    R3 = oracle.R2R((oracle.REDFT01, oracle.REDFT01))
    assert rel64(Eh, oracle.fft(d, dims=(1, 2), transforms=(R2,))) <= 1e-12
    R = dfft.fft(E, transforms=(dfft.R2R((dfft.REDFT01, dfft.REDFT01)),), dims=(1, 2))
    Rh = to_np(R)
    assert rel64(Rh, oracle.fft(Eh, dims=(1, 2), transforms=(R3,))) <= 1e-12
    assert rel64(Rh / (2 * 256) ** 2, d) <= 1e-12
