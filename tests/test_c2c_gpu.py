"""C2C parity of libdfft against the oracle (per-axis FFT semantics of
src/fft.jl:168-174 / src/fftgpu.jl:118-124 and the stage drivers
src/fft.jl:650-776 / src/fftgpu.jl:497-619)."""
import numpy as np
import pytest
import torch

import dfft
import dfft_oracle as oracle
from helpers import rand, rel, to_gpu, to_np, tol_for

pytestmark = pytest.mark.gpu

# every length up to 64 (primes above 13 go through Bluestein), the
# configuration edges, large powers of two, lengths only the dynamic kernel
# covers (7/11/13 factors), and large primes
LENGTHS_1D = sorted(set(list(range(1, 65)) + [
    80, 96, 100, 120, 125, 128, 160, 192, 243, 256, 384, 500, 512, 625, 729, 1000, 1024,
    1536, 2048, 3072, 4096, 8192, 77, 91, 98, 143, 169, 343, 1001, 2002, 4914,
    127, 251, 509, 1009, 2039, 4093]))


@pytest.mark.parametrize("n", LENGTHS_1D)
@pytest.mark.parametrize("dtype", [np.complex64, np.complex128])
def test_1d_batched_forward(n, dtype):
    if n > 4096 and dtype == np.complex128 and n % 2:
        pytest.skip("long odd double transform exceeds one CTA")
    batch = 3
    a = rand((n, batch), dtype, seed=n)
    y = dfft.fft(to_gpu(a), dims=(1,))
    ref = oracle.fft(a, dims=(1,))
    assert rel(to_np(y), ref) <= tol_for(dtype)


@pytest.mark.parametrize("n", [1, 2, 3, 5, 8, 12, 16, 48, 64, 96, 120, 128, 192, 243, 256, 512, 1000])
@pytest.mark.parametrize("dtype", [np.complex64, np.complex128])
def test_1d_inverse(n, dtype):
    a = rand((n, 5), dtype, seed=100 + n)
    y = dfft.ifft(to_gpu(a), dims=(1,))
    ref = oracle.ifft(a, dims=(1,))
    assert rel(to_np(y), ref) <= tol_for(dtype)


SHAPES_3D = [(8, 8, 8), (16, 12, 10), (5, 7, 9), (1, 16, 4), (32, 1, 24), (48, 64, 80),
             (3, 128, 2), (64, 64, 64), (96, 40, 30), (13, 11, 7), (17, 19, 23), (34, 31, 8)]


@pytest.mark.parametrize("shape", SHAPES_3D)
@pytest.mark.parametrize("order", ["F", "C"])
@pytest.mark.parametrize("dtype", [np.complex64, np.complex128])
def test_3d_fft_ifft(shape, order, dtype):
    a = rand(shape, dtype, seed=sum(shape))
    g = to_gpu(a, order)
    y = dfft.fft(g, decomp=dfft.Pencil(), dims=(1, 2, 3))
    ref = oracle.fft(a, dims=(1, 2, 3))
    assert rel(to_np(y), ref) <= tol_for(dtype)
    z = dfft.ifft(y, decomp=dfft.Pencil(), dims=(1, 2, 3))
    assert rel(to_np(z), a) <= tol_for(dtype)
    assert rel(to_np(z), oracle.ifft(ref, dims=(1, 2, 3))) <= tol_for(dtype)


@pytest.mark.parametrize("dims", [(1,), (2,), (3,), (1, 2), (2, 3), (1, 3), (3, 1), (2, 1, 3)])
@pytest.mark.parametrize("order", ["F", "C"])
def test_dims_subsets(dims, order):
    a = rand((12, 20, 9), np.complex128, seed=7)
    y = dfft.fft(to_gpu(a, order), dims=dims)
    assert rel(to_np(y), oracle.fft(a, dims=dims)) <= 1e-12
    z = dfft.ifft(to_gpu(a, order), dims=dims)
    assert rel(to_np(z), oracle.ifft(a, dims=dims)) <= 1e-12


@pytest.mark.parametrize("decomp", [dfft.Pencil(), dfft.Slab()])
def test_slab_equals_pencil(decomp):
    a = rand((32, 24, 16), np.complex64, seed=3)
    y = dfft.fft(to_gpu(a), decomp=decomp, dims=(1, 2, 3))
    assert rel(to_np(y), oracle.fft(a, dims=(1, 2, 3))) <= 1e-5


def test_2d_and_1d_arrays():
    a = rand((64, 48), np.complex64, seed=1)
    assert rel(to_np(dfft.fft(to_gpu(a), dims=(1, 2))), oracle.fft(a, dims=(1, 2))) <= 1e-5
    b = rand((1000,), np.complex128, seed=2)
    assert rel(to_np(dfft.fft(to_gpu(b), dims=(1,))), oracle.fft(b, dims=(1,))) <= 1e-12


def test_inplace_fft_bang():
    a = rand((16, 16, 16), np.complex64, seed=4)
    g = to_gpu(a)
    ptr = g.data_ptr()
    dfft.fft_(g, dims=(1, 2, 3))
    assert g.data_ptr() == ptr
    assert rel(to_np(g), oracle.fft(a, dims=(1, 2, 3))) <= 1e-5
    dfft.ifft_(g, dims=(1, 2, 3))
    assert rel(to_np(g), a) <= 1e-5


def test_known_answers():
    # impulse -> constant, constant -> scaled impulse, single tone -> delta
    n = 64
    x = np.zeros((n, 1), np.complex128)
    x[0] = 1
    assert np.allclose(to_np(dfft.fft(to_gpu(x), dims=(1,))), 1.0, atol=1e-14)
    c = np.ones((n, 1), np.complex128)
    y = to_np(dfft.fft(to_gpu(c), dims=(1,)))
    e = np.zeros((n, 1)); e[0] = n
    assert np.allclose(y, e, atol=1e-12)
    k0 = 5
    tone = np.exp(2j * np.pi * k0 * np.arange(n) / n).reshape(n, 1)
    y = to_np(dfft.fft(to_gpu(tone), dims=(1,)))
    e = np.zeros((n, 1)); e[k0] = n
    assert np.allclose(y, e, atol=1e-11)


def test_parseval_and_linearity():
    a = rand((40, 30, 20), np.complex128, seed=11)
    b = rand((40, 30, 20), np.complex128, seed=12)
    A = to_np(dfft.fft(to_gpu(a)))
    B = to_np(dfft.fft(to_gpu(b)))
    AB = to_np(dfft.fft(to_gpu(2.5 * a - 1j * b)))
    assert rel(AB, 2.5 * A - 1j * B) <= 1e-13
    assert abs(np.sum(np.abs(A) ** 2) / a.size - np.sum(np.abs(a) ** 2)) / np.sum(np.abs(a) ** 2) < 1e-13


def test_unknown_transform_and_bad_args():
    g = torch.zeros((4, 4), dtype=torch.complex64, device="cuda")
    with pytest.raises(dfft.ArgumentError, match="Unknown transform type"):
        dfft.get_or_create_gpu_plan("not a tag", g, (1,))
    with pytest.raises(dfft.ArgumentError):
        dfft.fft(g, dims=(3,))
    # a prime length beyond the longest Bluestein convolution (2^23) is
    # rejected, not faked
    with pytest.raises(dfft.ArgumentError):
        dfft.fft(torch.zeros((8388617,), dtype=torch.complex64, device="cuda"), dims=(1,))


@pytest.mark.parametrize("shape", [(512, 64, 48), (64, 512, 8), (96, 96, 96), (256, 8, 512)])
def test_tuned_plans_match(shape):
    # DFFT_FLAG_TUNE times every launch candidate (pipelined / one-tile
    # kernels, tile widths); whichever wins must give the same answer
    a = rand(shape, np.complex64, seed=sum(shape))
    g = to_gpu(a)
    p = dfft.gpu_plan_transform(dfft.FFT(), g, (1, 2, 3), flags=dfft.FLAG_TUNE)
    out = dfft.empty_like_layout(p.out_shape, g.dtype, g)
    p.execute(g, out)
    assert rel(to_np(out), oracle.fft(a, dims=(1, 2, 3))) <= 1e-5
    assert dfft.wisdom_size() > 0
    assert dfft.device_error() == 0


def test_wisdom_roundtrip(tmp_path):
    a = rand((64, 64, 64), np.complex64, seed=1)
    dfft.gpu_plan_transform(dfft.FFT(), to_gpu(a), (1, 2, 3), flags=dfft.FLAG_TUNE)
    n = dfft.wisdom_size()
    f = tmp_path / "wisdom.txt"
    dfft.wisdom_export(f)
    dfft.wisdom_forget()
    assert dfft.wisdom_size() == 0
    dfft.wisdom_import(f)
    assert dfft.wisdom_size() == n
