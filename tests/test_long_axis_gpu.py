"""Complex axes longer than one CTA holds run as a four-step pair of passes
(L = L1 * L2: L2-point transforms, the twiddle W_L^(n1 k2) on the way out,
then L1-point transforms written to k2 + L2 k1) instead of Bluestein's
passes of length >= 2L; prime axes whose Bluestein length M exceeds one CTA
run that convolution as two four-step pairs.  Checked against the FP64
oracle at the precision's stated tolerance, forward and inverse, on
contiguous and strided axes, for static and dynamic factors."""
import numpy as np
import pytest
import torch

import dfft
import dfft_oracle as oracle
from helpers import rand, rel, to_gpu, to_np, tol_for

pytestmark = pytest.mark.gpu


def _run(transform, g, dims):
    p = dfft.gpu_plan_transform(transform, g, dims)
    out = dfft.empty_like_layout(p.out_shape, g.dtype, g)
    p.execute(g, out)
    torch.cuda.synchronize()
    return p, out


def _four_step_lines(p):
    return [ln for ln in p.describe().splitlines() if "four-step" in ln]


@pytest.mark.parametrize("dtype,shape,dims", [
    (np.complex64, (65536,), (1,)),            # 256 x 256
    (np.complex64, (1 << 20,), (1,)),          # 1024 x 1024
    (np.complex64, (196608, 2), (1,)),         # 384 x 512, two pencils
    (np.complex64, (1000000,), (1,)),          # 1000 x 1000
    (np.complex64, (4, 32768, 3), (2,)),       # strided long axis, I = 4
    (np.complex64, (8, 65536, 5), (1, 2, 3)),  # long axis among short ones
    (np.complex64, (64064,), (1,)),            # 7 * 11 * 13 * 64: dynamic factors
    (np.complex128, (1 << 20,), (1,)),         # 1024 x 1024
    (np.complex128, (3, 40000, 2), (2,)),      # strided, 200 x 200
    (np.complex128, (200704,), (1,)),          # 392 (dynamic) x 512 (static)
])
def test_long_axis_matches_oracle(dtype, shape, dims):
    a = rand(shape, dtype, seed=len(shape) + shape[0] % 97)
    g = to_gpu(a)
    p, F = _run(dfft.FFT(), g, dims)
    assert len(_four_step_lines(p)) >= 2, p.describe()
    tol = tol_for(dtype)
    assert rel(to_np(F), oracle.fft(a, dims=dims)) <= tol
    _, B = _run(dfft.IFFT(), F, dims)
    assert rel(to_np(B), oracle.ifft(to_np(F), dims=dims)) <= tol
    assert rel(to_np(B), a) <= tol
    assert dfft.device_error() == 0


def test_long_axis_impulse_and_constant():
    # exact spectra: an impulse at n0 gives W^(n0 k), a constant gives L at k = 0
    L = 1 << 16
    a = np.zeros(L, np.complex128)
    a[12345] = 1
    _, F = _run(dfft.FFT(), to_gpu(a), (1,))
    k = np.arange(L)
    # the phase reduced exactly modulo L (2 pi * 12345 * k / L itself would
    # carry ~1e-11 of FP64 rounding)
    assert np.max(np.abs(to_np(F) - np.exp(-2j * np.pi * ((12345 * k) % L) / L))) <= 1e-12
    c = np.ones(L, np.complex128)
    _, F = _run(dfft.FFT(), to_gpu(c), (1,))
    Fh = to_np(F)
    assert abs(Fh[0] - L) <= 1e-9 and np.max(np.abs(Fh[1:])) <= 1e-9


def test_long_axis_in_place():
    a = rand((1 << 18,), np.complex64, seed=3)
    g = to_gpu(a)
    p = dfft.gpu_plan_transform(dfft.FFT(), g, (1,))
    p.execute(g, g)
    torch.cuda.synchronize()
    assert rel(to_np(g), oracle.fft(a, dims=(1,))) <= 1e-5


@pytest.mark.parametrize("dtype,shape,dims", [
    (np.complex64, (32771,), (1,)),        # M = 65610 = 243 x 270
    (np.complex64, (65537, 2), (1,)),      # M = 131220, two pencils
    (np.complex128, (3, 100003), (2,)),    # strided, M = 202500
    (np.complex64, (1000003,), (1,)),      # M = 2025000
    (np.complex128, (1000003,), (1,)),     # M = 2025000, ComplexF64 factors <= 2048
])
def test_prime_long_axis_bluestein_over_four_step(dtype, shape, dims):
    # a long prime axis: Bluestein's length-M convolution runs as two
    # four-step pairs (chirp on the first load, the filter on the third
    # pass's load, chirp and truncation on the last store)
    a = rand(shape, dtype, seed=shape[0] % 101)
    p, F = _run(dfft.FFT(), to_gpu(a), dims)
    assert len(_four_step_lines(p)) == 4, p.describe()
    tol = tol_for(dtype)
    assert rel(to_np(F), oracle.fft(a, dims=dims)) <= tol
    _, B = _run(dfft.IFFT(), F, dims)
    assert rel(to_np(B), a) <= tol
    assert dfft.device_error() == 0


@pytest.mark.parametrize("dtype,shape,dims", [
    (np.float32, (1 << 20,), (1,)),          # full-length form over a 1024 x 1024 pair
    (np.float64, (3, 131072), (2,)),         # strided, 256 x 512
    (np.float32, (65536, 4, 3), (1, 2, 3)),  # long first axis, then the half spectrum
    (np.float64, (100003,), (1,)),           # prime: Bluestein over four-step pairs
    (np.float32, (99999,), (1,)),            # odd, 3^2 x 41 x 271: Bluestein, real sides
    (np.float64, (1 << 20, 2), (1,)),        # Float64 full-length form, two columns
    (np.float32, (5, 262144), (2,)),         # strided long real axis
])
def test_long_real_axis_rfft_irfft(dtype, shape, dims):
    # real transforms whose half length no single pass handles take the
    # full-length form (real in, first n/2+1 outputs kept; Hermitian half
    # in, real out), split into a four-step pair like a complex axis
    a = rand(shape, dtype, seed=shape[0] % 89)
    F = dfft.rfft(to_gpu(a), dims=dims)
    ref = oracle.rfft(a, dims=dims)
    tol = tol_for(dtype)
    assert tuple(F.shape) == ref.shape
    assert rel(to_np(F), ref) <= tol
    d = shape[dims[0] - 1]
    x = dfft.irfft(F, d, dims=dims)
    assert rel(to_np(x), oracle.irfft(ref, d, dims=dims)) <= tol
    assert rel(to_np(x), a) <= tol
    assert dfft.device_error() == 0


@pytest.mark.parametrize("kind,n,dtype,cols", [
    (dfft.REDFT10, 65536, np.float64, 1),    # FFT length 65536: 256 x 256
    (dfft.REDFT01, 40000, np.float32, 2),    # 200 x 200
    (dfft.REDFT00, 20001, np.float64, 1),    # FFT length 40000
    (dfft.RODFT00, 32767, np.float64, 1),    # FFT length 65536
    (dfft.REDFT11, 30000, np.float32, 1),    # FFT length 60000
    (dfft.RODFT11, 25000, np.float64, 1),    # FFT length 50000
    (dfft.DHT, 50000, np.float64, 2),        # 5-smooth, 200 x 250
    (dfft.RODFT10, 100003, np.float64, 1),   # prime: Bluestein over four-step pairs
    (dfft.REDFT10, 65536, np.float32, 3),
    (dfft.RODFT01, 36000, np.float32, 1),
    (dfft.REDFT11, 70001, np.float64, 1),    # FFT length 140002 = 2 x 70001: Bluestein
])
def test_long_r2r_axis(kind, n, dtype, cols):
    # r2r kinds on axes whose FFT no single pass handles: the loads and
    # stores of the four-step sub-axes index the whole axis
    a = rand((n, cols), dtype, seed=n % 97 + kind)
    y = dfft.fft(to_gpu(a), dims=(1,), transforms=(dfft.R2R((kind,)),))
    ref = oracle.r2r_1d(a.astype(np.float64), kind, 0)
    assert rel(to_np(y), ref) <= tol_for(dtype)
    assert dfft.device_error() == 0


def test_long_r2r_strided_axis():
    a = rand((3, 65536), np.float32, seed=11)
    y = dfft.fft(to_gpu(a), dims=(2,), transforms=(dfft.R2R((dfft.REDFT10,)),))
    ref = oracle.r2r_1d(a.astype(np.float64), dfft.REDFT10, 1)
    assert rel(to_np(y), ref) <= 1e-5


@pytest.mark.parametrize("dtype,shape,dims", [
    (np.complex64, (1 << 20,), (1,)),
    (np.complex64, (6, 65536), (2,)),        # strided: the swap moves rows of 6
    (np.complex128, (1 << 18, 3), (1,)),
])
def test_long_axis_fast_form(dtype, shape, dims):
    # plain complex long axes take the three-pass form: the strided pass
    # (pipelined, twiddle on its tile), the contiguous pass, the axis swap
    a = rand(shape, dtype, seed=len(shape))
    p, F = _run(dfft.FFT(), to_gpu(a), dims)
    desc = p.describe()
    assert "axis-swap" in desc and "strided-pipe" in desc, desc
    tol = tol_for(dtype)
    assert rel(to_np(F), oracle.fft(a, dims=dims)) <= tol
    _, B = _run(dfft.IFFT(), F, dims)
    assert rel(to_np(B), a) <= tol
