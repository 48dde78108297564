"""The mixed (tensor-core) form: ComplexF32 axes of length 512 run as
radix-32 x radix-16 complex matrix products on tcgen05 with FP16 hi+lo split
operands, FP32 accumulation and per-pencil power-of-two scaling; other axes
keep the plain form.  Every result is checked against the FP64 oracle at
relative L2 <= 1e-6 (the mixed form's stated bound), plus round trips."""
import os

import numpy as np
import pytest
import torch

import dfft
import dfft_oracle as oracle
from helpers import rand, rel, to_gpu, to_np

pytestmark = pytest.mark.gpu

MIXED_TOL = 1e-6


def _mixed(transform, g, dims, decomp=None):
    p = dfft.gpu_plan_transform(transform, g, dims, decomp=decomp, method="mixed")
    out = dfft.empty_like_layout(p.out_shape, g.dtype, g)
    p.execute(g, out)
    torch.cuda.synchronize()
    return p, out


@pytest.mark.parametrize("shape,dims", [
    ((512, 48, 8), (1,)),          # contiguous pencils, 384 of them (24 tiles)
    ((512, 40, 3), (1,)),          # 120 pencils: a partial last tile
    ((64, 512, 4), (2,)),          # strided, I = 64
    ((18, 512, 3), (2,)),          # strided, I = 18: a partial column tile
    ((16, 8, 512), (3,)),          # strided, I = 128
    ((512, 512, 4), (1, 2)),       # both variants
    ((512, 24, 512), (1, 2, 3)),   # dim 2 (length 24) runs the plain form
])
def test_mixed_axes_match_oracle(shape, dims):
    a = rand(shape, np.complex64, seed=sum(shape))
    g = to_gpu(a)
    p, F = _mixed(dfft.FFT(), g, dims)
    desc = p.describe()
    assert "mixed" in desc, desc
    assert rel(to_np(F), oracle.fft(a, dims=dims)) <= MIXED_TOL
    pi, B = _mixed(dfft.IFFT(), F, dims)
    assert rel(to_np(B), oracle.ifft(to_np(F), dims=dims)) <= MIXED_TOL
    assert rel(to_np(B), a) <= MIXED_TOL
    assert dfft.device_error() == 0


def test_mixed_single_pass_error_and_bias():
    # one pass over 4096 pencils: the relative error, and its projection on
    # the exact result (a systematic shrink would show up there; the product
    # chains are kept short so that it stays near 2.5 * 0.36 * 2^-23)
    a = rand((512, 4096), np.complex64, seed=21)
    _, F = _mixed(dfft.FFT(), to_gpu(a), (1,))
    ref = oracle.fft(a, dims=(1,))
    Fh = to_np(F).astype(np.complex128)
    err = rel(Fh, ref)
    bias = float(np.vdot(ref, Fh).real / np.vdot(ref, ref).real) - 1.0
    print(f"mixed single pass: rel {err:.3e}, projected bias {bias:+.3e}")
    assert err <= 4e-7
    assert abs(bias) <= 2e-7


def test_mixed_row_major_input():
    a = rand((4, 512, 512), np.complex64, seed=5)   # logical (4, 512, 512), C order
    g = to_gpu(a, order="C")
    _, F = _mixed(dfft.FFT(), g, (2, 3))
    assert rel(to_np(F), oracle.fft(a, dims=(2, 3))) <= MIXED_TOL


def test_mixed_per_pencil_scaling():
    # pencils 40 orders of magnitude apart, zero pencils and an impulse: each
    # pencil is scaled on its own, so each keeps its own relative accuracy
    a = rand((512, 64), np.complex64, seed=9)
    a[:, 1::4] *= np.float32(1e-20)
    a[:, 2::4] *= np.float32(1e18)
    a[:, 3::8] = 0
    a[:, 7] = 0
    a[3, 7] = 1 + 1j
    g = to_gpu(a)
    _, F = _mixed(dfft.FFT(), g, (1,))
    Fh = to_np(F)
    ref = oracle.fft(a, dims=(1,))
    for j in range(a.shape[1]):
        n = np.linalg.norm(ref[:, j])
        if n == 0:
            assert np.all(Fh[:, j] == 0), j
        else:
            assert np.linalg.norm(Fh[:, j] - ref[:, j]) / n <= MIXED_TOL, j


def test_mixed_complex128_keeps_plain_form():
    a = rand((512, 16, 4), np.complex128, seed=2)
    g = to_gpu(a)
    p, F = _mixed(dfft.FFT(), g, (1, 2, 3))
    assert "mixed" not in p.describe()
    assert rel(to_np(F), oracle.fft(a, dims=(1, 2, 3))) <= 1e-12


def test_mixed_rejects_real_transforms():
    g = torch.zeros((512, 8), dtype=torch.float32, device="cuda")
    with pytest.raises(dfft.ArgumentError, match="mixed form"):
        dfft.gpu_plan_transform(dfft.RFFT(), g, (1,), method="mixed")


def test_mixed_512cube_slab_against_fp64_oracle():
    n = 512
    old = oracle.WORKERS
    oracle.WORKERS = os.cpu_count() or 1
    try:
        a = oracle.make_input("normal", (n, n, n), 3, np.complex64)
        g = to_gpu(a)
        del a
        p, F = _mixed(dfft.FFT(), g, (1, 2, 3), decomp=dfft.Slab())
        assert p.launches == 3
        ah = to_np(g)
        Fh = to_np(F)
        ref = oracle.fft(ah, dims=(1, 2, 3))
        e_fwd = _rel64(Fh, ref)
        del ref
        pi, B = _mixed(dfft.IFFT(), F, (1, 2, 3), decomp=dfft.Slab())
        Bh = to_np(B)
        e_rt = _rel64(Bh, ah)
        ref_inv = oracle.ifft(Fh, dims=(1, 2, 3))
        e_inv = _rel64(Bh, ref_inv)
        print(f"mixed 512^3 ComplexF32: fwd {e_fwd:.3e} inv {e_inv:.3e} roundtrip {e_rt:.3e}")
        assert e_fwd <= MIXED_TOL and e_inv <= MIXED_TOL and e_rt <= MIXED_TOL
        assert dfft.device_error() == 0
    finally:
        oracle.WORKERS = old


def _rel64(a, b, chunk_elems=1 << 24):
    per = max(1, a.size // a.shape[-1])
    step = max(1, chunk_elems // per)
    num = den = 0.0
    for k in range(0, a.shape[-1], step):
        x = a[..., k:k + step].astype(np.complex128)
        y = b[..., k:k + step].astype(np.complex128)
        num += float(np.sum(np.abs(x - y) ** 2))
        den += float(np.sum(np.abs(y) ** 2))
    return float(np.sqrt(num / den))
