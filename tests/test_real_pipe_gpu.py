"""Pipelined R2C / C2R passes (real_pass): the first pass of rfft and the
last pass of irfft along the contiguous axis (apply_fft! with the RFFT /
IRFFT tags, src/fft.jl:146-174), for every half length the kernel is built
for, checked against the oracle (rfft halves dims[1] to n//2+1; irfft
needs the real length)."""
import numpy as np
import pytest

import dfft
import dfft_oracle as oracle
from helpers import rand, rel, to_gpu, to_np, tol_for

pytestmark = pytest.mark.gpu

HALF = [32, 48, 64, 96, 128, 192, 256]


@pytest.mark.parametrize("m", HALF)
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_every_half_length(m, dtype):
    n = 2 * m
    a = rand((n, 8, 8), dtype, seed=m, kind="uniform01")  # 64 pencils: whole tiles
    g = to_gpu(a)
    p = dfft.gpu_plan_transform(dfft.RFFT(), g, (1,))
    assert "real-pipe" in p.describe(), p.describe()
    F = dfft.rfft(g, dims=(1,))
    ref = oracle.rfft(a, dims=(1,))
    assert rel(to_np(F), ref) <= tol_for(dtype)
    q = dfft.gpu_plan_transform(dfft.IRFFT(), F, (1,), n=n)
    assert "real-pipe" in q.describe(), q.describe()
    x = dfft.irfft(F, n, dims=(1,))
    assert rel(to_np(x), a) <= tol_for(dtype)
    assert rel(to_np(x), oracle.irfft(ref, n, dims=(1,))) <= tol_for(dtype)
    assert dfft.device_error() == 0


@pytest.mark.parametrize("order", ["F", "C"])
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_3d_round_trip(order, dtype):
    a = rand((256, 64, 32), dtype, seed=9)
    g = to_gpu(a, order)
    F = dfft.rfft(g, dims=(1, 2, 3))
    ref = oracle.rfft(a, dims=(1, 2, 3))
    assert rel(to_np(F), ref) <= tol_for(dtype)
    x = dfft.irfft(F, 256, dims=(1, 2, 3))
    assert rel(to_np(x), a) <= tol_for(dtype)
    y = dfft.irfft(F.clone(), 256, dims=(1, 2, 3), destroy_input=True)
    assert rel(to_np(y), to_np(x)) <= tol_for(dtype)


def test_known_answers():
    # a cosine of frequency 3 -> two spikes; irfft brings it back
    n = 128
    t = np.arange(n)
    a = np.repeat(np.cos(2 * np.pi * 3 * t / n)[:, None], 32, axis=1).astype(np.float64)
    F = to_np(dfft.rfft(to_gpu(a), dims=(1,)))
    e = np.zeros((n // 2 + 1, 32), np.complex128)
    e[3] = n / 2
    assert np.abs(F - e).max() <= 1e-11
    x = to_np(dfft.irfft(to_gpu(e), n, dims=(1,)))
    assert np.abs(x - a).max() <= 1e-14
