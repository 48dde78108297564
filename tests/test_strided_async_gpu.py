"""cp.async strided axis pass (axis_pass_async): strided ComplexF32 passes
whose row stride is not a multiple of 16 bytes, which TMA cannot address
(the half-spectrum rows of a Float32 rfft: n/2+1 elements).  Every launch
shape is forced through an edited wisdom file (the FFTW-wisdom analogue,
src/fft.jl:113-124,162) and checked against the oracle on the per-axis
semantics of src/fft.jl:168-174; the untuned planner's choice and whole
rfft / irfft transforms are checked too."""
import numpy as np
import pytest

import dfft
import dfft_oracle as oracle
from helpers import rand, rel, to_gpu, to_np

pytestmark = pytest.mark.gpu

# (shape, dim, launch shapes of that length); I * 8 bytes is never a
# multiple of 16 (odd I)
CASES = [((129, 256, 24), 2, 2), ((65, 128, 40), 2, 1), ((257, 512, 4), 2, 2),
         ((33, 64, 64), 2, 1), ((49, 96, 32), 2, 1), ((97, 192, 8), 2, 1),
         ((193, 384, 2), 2, 1), ((13, 15, 128), 3, 1), ((7, 3, 512), 3, 2)]


def _forced_plan(tag, g, dim, idx, tmp_path):
    dfft.wisdom_forget()
    dfft.gpu_plan_transform(tag, g, (dim,), flags=dfft.FLAG_TUNE)
    f = tmp_path / "w.txt"
    dfft.wisdom_export(f)
    lines = [ln for ln in f.read_text().splitlines() if ln and not ln.startswith("#")]
    assert len(lines) == 1
    key = lines[0].split()[0]
    f.write_text(f"{key} 5 {idx} 0\n")  # variant 5 = cp.async strided, C = launch shape
    dfft.wisdom_forget()
    dfft.wisdom_import(f)
    p = dfft.gpu_plan_transform(tag, g, (dim,))
    dfft.wisdom_forget()
    return p


@pytest.mark.parametrize("shape,dim,nshapes", CASES)
@pytest.mark.parametrize("inverse", [False, True])
def test_every_launch_shape(shape, dim, nshapes, inverse, tmp_path):
    a = rand(shape, np.complex64, seed=sum(shape) + dim)
    g = to_gpu(a)
    tag = dfft.IFFT() if inverse else dfft.FFT()
    ref = (oracle.ifft if inverse else oracle.fft)(a, dims=(dim,))
    for idx in range(nshapes):
        p = _forced_plan(tag, g, dim, idx, tmp_path)
        assert "strided-async" in p.describe(), p.describe()
        out = dfft.empty_like_layout(p.out_shape, g.dtype, g)
        p.execute(g, out)
        assert rel(to_np(out), ref) <= 1e-5, idx
        assert dfft.device_error() == 0


def test_in_place_and_c_order(tmp_path):
    a = rand((129, 256, 6), np.complex64, seed=9)
    for order in ["F", "C"]:
        g = to_gpu(a, order)
        # C order: the dim-2 columns are the 6 elements of dim 3 (48-byte rows)
        p = _forced_plan(dfft.FFT(), g, 2, 1, tmp_path)
        assert "strided-async" in p.describe(), p.describe()
        p.execute(g, g)
        assert rel(to_np(g), oracle.fft(a, dims=(2,))) <= 1e-5


def test_untuned_plan_uses_it():
    # untuned plans take it for L = 512 (the other lengths are tuner candidates)
    a = rand((257, 512, 40), np.complex64, seed=3)  # 42 MB pass
    g = to_gpu(a)
    p = dfft.gpu_plan_transform(dfft.FFT(), g, (2,))
    assert "strided-async" in p.describe(), p.describe()
    out = dfft.empty_like_layout(p.out_shape, g.dtype, g)
    p.execute(g, out)
    assert rel(to_np(out), oracle.fft(a, dims=(2,))) <= 1e-5


def test_rfft_irfft_float32():
    # the dim-2 pass of a Float32 rfft over 512 x 512 x 24 runs on 257-element rows
    x = rand((512, 512, 24), np.float32, seed=4)
    g = to_gpu(x)
    p = dfft.gpu_plan_transform(dfft.RFFT(), g, (1, 2, 3))
    assert "strided-async" in p.describe(), p.describe()
    Y = dfft.rfft(g, dims=(1, 2, 3))
    assert rel(to_np(Y), oracle.rfft(x, dims=(1, 2, 3))) <= 1e-5
    z = dfft.irfft(Y, 512, dims=(1, 2, 3))
    assert rel(to_np(z), x) <= 1e-5
    assert dfft.device_error() == 0
