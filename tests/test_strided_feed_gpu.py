"""Producer-fed strided axis pass (axis_pass_strided): every launch shape,
forced through an edited wisdom file (the FFTW-wisdom analogue, which the
reference writes after planning, src/fft.jl:113-124,162), checked against
the oracle on the per-axis semantics of src/fft.jl:168-174."""
import numpy as np
import pytest

import dfft
import dfft_oracle as oracle
from helpers import rand, rel, to_gpu, to_np, tol_for

pytestmark = pytest.mark.gpu

# (shape, dim, dtype, launch shapes of that length)
CASES = [((64, 512, 12), 2, np.complex64, 7), ((72, 512, 6), 2, np.complex64, 7),
         ((16, 8, 512), 3, np.complex64, 7), ((40, 256, 20), 2, np.complex64, 3),
         ((128, 128, 30), 2, np.complex64, 2), ((24, 512, 6), 2, np.complex128, 2),
         ((32, 256, 18), 2, np.complex128, 2),
         # lengths of the batched / serving configurations (plain row layout
         # unless a power of two)
         ((32, 48, 6), 2, np.complex64, 1), ((16, 64, 8), 2, np.complex64, 1),
         ((32, 80, 6), 2, np.complex64, 1), ((16, 8, 96), 3, np.complex64, 1),
         ((48, 120, 4), 2, np.complex64, 1), ((16, 160, 4), 2, np.complex64, 1),
         ((32, 192, 4), 2, np.complex64, 1), ((16, 384, 2), 2, np.complex64, 1),
         ((16, 64, 8), 2, np.complex128, 1), ((8, 96, 8), 2, np.complex128, 1),
         ((8, 128, 4), 2, np.complex128, 1), ((8, 192, 4), 2, np.complex128, 1),
         ((8, 384, 2), 2, np.complex128, 1)]


def _forced_plan(tag, g, dim, idx, tmp_path):
    dfft.wisdom_forget()
    dfft.gpu_plan_transform(tag, g, (dim,), flags=dfft.FLAG_TUNE)
    f = tmp_path / "w.txt"
    dfft.wisdom_export(f)
    lines = [ln for ln in f.read_text().splitlines() if ln and not ln.startswith("#")]
    assert len(lines) == 1
    key = lines[0].split()[0]
    f.write_text(f"{key} 4 {idx} 0\n")  # variant 4 = producer-fed strided, C = launch shape
    dfft.wisdom_forget()
    dfft.wisdom_import(f)
    p = dfft.gpu_plan_transform(tag, g, (dim,))
    dfft.wisdom_forget()
    return p


@pytest.mark.parametrize("shape,dim,dtype,nshapes", CASES)
@pytest.mark.parametrize("inverse", [False, True])
def test_every_launch_shape(shape, dim, dtype, nshapes, inverse, tmp_path):
    a = rand(shape, dtype, seed=sum(shape) + dim)
    g = to_gpu(a)
    tag = dfft.IFFT() if inverse else dfft.FFT()
    ref = (oracle.ifft if inverse else oracle.fft)(a, dims=(dim,))
    for idx in range(nshapes):
        p = _forced_plan(tag, g, dim, idx, tmp_path)
        assert "strided-feed" in p.describe(), p.describe()
        out = dfft.empty_like_layout(p.out_shape, g.dtype, g)
        p.execute(g, out)
        assert rel(to_np(out), ref) <= tol_for(dtype), idx
        assert dfft.device_error() == 0


def test_in_place_and_c_order(tmp_path):
    a = rand((48, 512, 8), np.complex64, seed=5)
    for order in ["F", "C"]:
        g = to_gpu(a, order)
        # launch shape 1 (8-column tiles) fits both layouts: I = 48 (F), 8 (C)
        p = _forced_plan(dfft.FFT(), g, 2, 1, tmp_path)
        assert "strided-feed" in p.describe()
        p.execute(g, g)
        assert rel(to_np(g), oracle.fft(a, dims=(2,))) <= 1e-5


def test_describe_lists_every_launch():
    g = to_gpu(rand((256, 256, 64), np.complex64, seed=1))
    p = dfft.gpu_plan_transform(dfft.FFT(), g, (1, 2, 3))
    d = p.describe().strip().splitlines()
    assert len(d) == p.launches
    assert d[0].startswith("slab-xy L=256")


def test_untuned_shape_fits_the_columns():
    # untuned plans take the first launch shape whose tile is not wider than
    # the columns along the contiguous axes (16-column tiles need I >= 16)
    for shape in [(8, 512, 1100), (64, 512, 140)]:
        a = rand(shape, np.complex64, seed=shape[0])
        g = to_gpu(a)
        p = dfft.gpu_plan_transform(dfft.FFT(), g, (2,))
        assert "strided-feed" in p.describe(), p.describe()
        out = dfft.empty_like_layout(p.out_shape, g.dtype, g)
        p.execute(g, out)
        assert rel(to_np(out), oracle.fft(a, dims=(2,))) <= 1e-5
