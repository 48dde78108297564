"""R2R parity for every FFTW kind the reference lists (src/fft.jl:1-11) and
the README's 2-D REDFT10/REDFT01 round trip (README.md:58-67)."""
import numpy as np
import pytest

import dfft
import dfft_oracle as oracle
from helpers import rand, rel, to_gpu, to_np, tol_for

pytestmark = pytest.mark.gpu

KINDS = [dfft.REDFT10, dfft.REDFT01, dfft.REDFT11, dfft.RODFT10, dfft.RODFT01, dfft.RODFT11,
         dfft.REDFT00, dfft.RODFT00, dfft.DHT]


@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("n", [2, 3, 4, 5, 8, 9, 16, 31, 64, 100, 256, 257])
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_r2r_1d(kind, n, dtype):
    a = rand((n, 3), dtype, seed=kind * 1000 + n)
    y = dfft.fft(to_gpu(a), dims=(1,), transforms=(dfft.R2R((kind,)),))
    ref = oracle.r2r_direct(a.astype(np.longdouble), kind, 0)
    assert rel(to_np(y), ref) <= tol_for(dtype)


def _smooth(m):
    for p in (2, 3, 5, 7, 11, 13):
        while m % p == 0:
            m //= p
    return m == 1


@pytest.mark.parametrize("order", ["F", "C"])
def test_readme_dct_2d_roundtrip(order):
    # README.md:58-67: F = REDFT10 x REDFT10, A_recon = REDFT01 x REDFT01 (= (2*256)^2 A)
    a = rand((256, 256), np.float64, seed=42, kind="uniform01")
    F = dfft.fft(to_gpu(a, order), decomp=dfft.Slab(),
                 transforms=(dfft.R2R((dfft.REDFT10, dfft.REDFT10)),), dims=(1, 2))
    ref = oracle.fft(a, dims=(1, 2), transforms=(oracle.R2R((oracle.REDFT10, oracle.REDFT10)),))
    assert rel(to_np(F), ref) <= 1e-12
    A = dfft.ifft(F, decomp=dfft.Slab(), transforms=(dfft.R2R((dfft.REDFT01, dfft.REDFT01)),),
                  dims=(1, 2))
    assert rel(to_np(A) / (2 * 256) ** 2, a) <= 1e-12


def test_batched_dct_3d_stack():
    # 2-D DCT-II/III over a stack of 32 planes (dims (1,2) of 256x256x32)
    a = rand((64, 48, 32), np.float64, seed=9)
    F = dfft.fft(to_gpu(a), transforms=(dfft.R2R((dfft.REDFT10, dfft.REDFT10)),), dims=(1, 2))
    ref = oracle.fft(a, dims=(1, 2), transforms=(oracle.R2R((oracle.REDFT10, oracle.REDFT10)),))
    assert rel(to_np(F), ref) <= 1e-12
    B = dfft.ifft(F, transforms=(dfft.R2R((dfft.REDFT01, dfft.REDFT01)),), dims=(1, 2))
    assert rel(to_np(B) / (4 * 64 * 48), a) <= 1e-12


def test_unknown_kind():
    with pytest.raises(dfft.ArgumentError, match="Unknown transform type"):
        dfft.R2R((42,))
