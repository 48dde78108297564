"""Tile-staged R2R passes (tiled_pass): every FFTW kind the reference lists
(src/fft.jl:1-11) along the contiguous axis (whole pencils) and a strided
axis (column tiles), at extents whose FFT length is 128, 256 or 512, checked
against the oracle's direct sums / FFTW definitions."""
import numpy as np
import pytest

import dfft
import dfft_oracle as oracle
from helpers import rand, rel, to_gpu, to_np, tol_for

pytestmark = pytest.mark.gpu

# kind -> data extents N whose FFT length (N, 2N, 2(N-1), 2(N+1)) is 128 / 256 / 512
EXTENTS = {dfft.REDFT10: [128, 256, 512], dfft.REDFT01: [128, 256, 512], dfft.RODFT10: [128, 256],
           dfft.RODFT01: [128, 256], dfft.DHT: [128, 512], dfft.REDFT11: [64, 128, 256],
           dfft.RODFT11: [64, 128], dfft.REDFT00: [65, 129], dfft.RODFT00: [63, 127]}
CASES = [(k, n) for k, ns in EXTENTS.items() for n in ns]


@pytest.mark.parametrize("kind,n", CASES)
@pytest.mark.parametrize("axis", [1, 2])
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_tiled_kinds(kind, n, axis, dtype):
    shape = (n, 16, 4) if axis == 1 else (16, n, 4)
    a = rand(shape, dtype, seed=kind * 997 + n + axis)
    g = to_gpu(a)
    tr = (dfft.R2R((kind,)),)
    p = dfft.gpu_plan_transform(dfft.R2R((kind,)), g, (axis,))
    y = dfft.fft(g, dims=(axis,), transforms=tr)
    ref = oracle.fft(a, dims=(axis,), transforms=(oracle.R2R((kind,)),))
    assert rel(to_np(y), ref) <= tol_for(dtype), p.describe()
    assert dfft.device_error() == 0


@pytest.mark.parametrize("order", ["F", "C"])
def test_dct_stack_uses_tiles(order):
    # the DCT-II / DCT-III stack of the batched configuration, 256 x 256 x 32
    a = rand((256, 256, 32), np.float64, seed=3, kind="uniform01")
    g = to_gpu(a, order)
    for kind in (dfft.REDFT10, dfft.REDFT01):
        p = dfft.gpu_plan_transform(dfft.R2R((kind, kind)), g, (1, 2))
        kinds = [ln.split()[0] for ln in p.describe().strip().splitlines()]
        assert kinds and all(k.startswith("tiled") for k in kinds), p.describe()
    F = dfft.fft(g, dims=(1, 2), transforms=(dfft.R2R((dfft.REDFT10, dfft.REDFT10)),))
    ref = oracle.fft(a, dims=(1, 2), transforms=(oracle.R2R((oracle.REDFT10, oracle.REDFT10)),))
    assert rel(to_np(F), ref) <= 1e-12
    B = dfft.fft(F, dims=(1, 2), transforms=(dfft.R2R((dfft.REDFT01, dfft.REDFT01)),))
    assert rel(to_np(B), a * (2 * 256) ** 2) <= 1e-12
