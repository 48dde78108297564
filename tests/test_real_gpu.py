"""rfft / irfft parity (README.md:36-45; AbstractFFTs conventions: dims[1]
halved to n//2+1, irfft needs the real length d)."""
import numpy as np
import pytest

import dfft
import dfft_oracle as oracle
from helpers import rand, rel, to_gpu, to_np, tol_for

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [1, 2, 3, 4, 5, 6, 7, 8, 9, 15, 16, 30, 31, 34, 64, 96, 100, 127, 128,
                               255, 256, 500, 512, 1024, 1018, 2048])
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_rfft_irfft_1d(n, dtype):
    a = rand((n, 4), dtype, seed=n)
    F = dfft.rfft(to_gpu(a), dims=(1,))
    ref = oracle.rfft(a, dims=(1,))
    assert F.shape == (n // 2 + 1, 4)
    assert rel(to_np(F), ref) <= tol_for(dtype)
    x = dfft.irfft(F, n, dims=(1,))
    assert x.shape == (n, 4)
    assert rel(to_np(x), a) <= tol_for(dtype)
    assert rel(to_np(x), oracle.irfft(ref, n, dims=(1,))) <= tol_for(dtype)


@pytest.mark.parametrize("shape", [(16, 8, 4), (15, 6, 5), (64, 32, 48), (9, 10, 11), (256, 16, 8),
                                   (34, 17, 6)])
@pytest.mark.parametrize("dims", [(1, 2, 3), (2, 3), (3, 1, 2), (1,), (2,)])
@pytest.mark.parametrize("order", ["F", "C"])
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_rfft_irfft_nd(shape, dims, order, dtype):
    a = rand(shape, dtype, seed=sum(shape) + len(dims))
    F = dfft.rfft(to_gpu(a, order), decomp=dfft.Pencil(), dims=dims)
    ref = oracle.rfft(a, dims=dims)
    assert tuple(F.shape) == ref.shape
    assert rel(to_np(F), ref) <= tol_for(dtype)
    d = shape[dims[0] - 1]
    Fin = F.clone()
    x = dfft.irfft(F, d, decomp=dfft.Pencil(), dims=dims)
    assert rel(to_np(F), to_np(Fin)) == 0.0, "irfft must not modify its input"
    assert rel(to_np(x), oracle.irfft(ref, d, dims=dims)) <= tol_for(dtype)
    assert rel(to_np(x), a) <= tol_for(dtype)


def test_irfft_destroy_input_matches():
    a = rand((32, 20, 12), np.float64, seed=5)
    F = dfft.rfft(to_gpu(a))
    x1 = dfft.irfft(F.clone(), 32)
    x2 = dfft.irfft(F.clone(), 32, destroy_input=True)
    assert rel(to_np(x1), to_np(x2)) <= 1e-15
    assert rel(to_np(x1), a) <= 1e-12


def test_irfft_length_mismatch():
    F = dfft.rfft(to_gpu(rand((16, 4), np.float32)), dims=(1,))
    with pytest.raises(dfft.ArgumentError):
        dfft.irfft(F, 20, dims=(1,))
    # d = 17 also has 17//2+1 == 9 entries: both 16 and 17 are accepted
    x = dfft.irfft(F, 17, dims=(1,))
    assert x.shape[0] == 17
