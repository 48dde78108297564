"""Fused 2-D slab pass: dims 1 and 2 of an L x L x O array transformed in
one sweep per slab (the Slab decomposition's first stage, src/fft.jl:735 /
src/fftgpu.jl:541), checked against the oracle and against the plan that
runs one pass per axis (DFFT_FLAG_NO_FUSE)."""
import numpy as np
import pytest
import torch

import dfft
import dfft_oracle as oracle
from helpers import rand, rel, to_gpu, to_np, tol_for

pytestmark = pytest.mark.gpu

# (L, O, dtype)
CASES = [(512, 24, np.complex64), (256, 80, np.complex64), (128, 320, np.complex64),
         (512, 20, np.complex128), (256, 64, np.complex128)]


def _plan(tag, g, dims, flags=dfft.FLAG_FUSE, decomp=None):
    # FLAG_FUSE: the fused kernel wherever one exists, so every length is covered
    return dfft.gpu_plan_transform(tag, g, dims, decomp=decomp, flags=flags)


def _run(p, g):
    out = dfft.empty_like_layout(p.out_shape, g.dtype, g)
    p.execute(g, out)
    return out


@pytest.mark.parametrize("L,O,dtype", CASES)
@pytest.mark.parametrize("dims", [(1, 2), (1, 2, 3)])
def test_fused_matches_oracle(L, O, dtype, dims):
    a = rand((L, L, O), dtype, seed=L + O)
    g = to_gpu(a)
    p = _plan(dfft.FFT(), g, dims, decomp=dfft.Slab())
    assert p.launches == len(dims) - 1  # dims 1 and 2 share one launch
    y = _run(p, g)
    assert dfft.device_error() == 0
    ref = oracle.fft(a, dims=dims)
    assert rel(to_np(y), ref) <= tol_for(dtype)
    q = _plan(dfft.IFFT(), y, dims, decomp=dfft.Slab())
    assert q.launches == len(dims) - 1
    z = _run(q, y)
    assert rel(to_np(z), a) <= tol_for(dtype)


@pytest.mark.parametrize("L,O,dtype", CASES[:2] + CASES[3:4])
def test_fused_equals_per_axis(L, O, dtype):
    a = rand((L, L, O), dtype, seed=3 * L + O)
    g = to_gpu(a)
    fused = _plan(dfft.FFT(), g, (1, 2, 3))
    split = _plan(dfft.FFT(), g, (1, 2, 3), flags=dfft.FLAG_NO_FUSE)
    assert fused.launches == 2 and split.launches == 3
    y1 = to_np(_run(fused, g))
    y2 = to_np(_run(split, g))
    # same radices and twiddles in both: only the rounding order differs
    assert rel(y1, y2) <= (1e-6 if dtype == np.complex64 else 1e-14)


@pytest.mark.parametrize("order", ["F", "C"])
def test_fused_c_order_and_dims_order(order):
    # row-major (O, L, L) tensors are column-major L x L x O arrays with the
    # dims reversed; dims (2, 1, 3) puts 1 and 2 next to each other too
    a = rand((256, 256, 48), np.complex64, seed=9)
    g = to_gpu(a, order)
    for dims in [(1, 2, 3), (2, 1, 3), (3, 1, 2)]:
        p = _plan(dfft.FFT(), g, dims)
        y = _run(p, g)
        assert rel(to_np(y), oracle.fft(a, dims=dims)) <= 1e-5


def test_fused_in_place():
    a = rand((512, 512, 32), np.complex64, seed=5)
    g = to_gpu(a)
    ptr = g.data_ptr()
    dfft.fft_(g, decomp=dfft.Slab(), dims=(1, 2, 3))
    assert g.data_ptr() == ptr
    assert rel(to_np(g), oracle.fft(a, dims=(1, 2, 3))) <= 1e-5
    dfft.ifft_(g, decomp=dfft.Slab(), dims=(1, 2, 3))
    assert rel(to_np(g), a) <= 1e-5
    assert dfft.device_error() == 0


def test_fused_known_answers():
    # a plane wave in (x, y) on every slab -> one spike per slab, scaled by L^2
    L, O = 256, 40
    x = np.arange(L)
    kx, ky = 3, 250
    wave = np.exp(2j * np.pi * (kx * x[:, None] + ky * x[None, :]) / L)
    a = np.repeat(wave[:, :, None], O, axis=2) * np.arange(1, O + 1)[None, None, :]
    y = to_np(dfft.fft(to_gpu(a.astype(np.complex128)), dims=(1, 2)))
    e = np.zeros((L, L, O), np.complex128)
    e[kx, ky, :] = L * L * np.arange(1, O + 1)
    assert np.abs(y - e).max() <= 1e-9 * L * L * O


@pytest.mark.parametrize("O", [1, 2, 3])
def test_few_slabs(O):
    # fewer slabs than rounds of lag: most of the job sequence is empty
    a = rand((256, 256, O), np.complex64, seed=2 + O)
    g = to_gpu(a)
    p = _plan(dfft.FFT(), g, (1, 2))
    assert p.launches == 1
    assert rel(to_np(_run(p, g)), oracle.fft(a, dims=(1, 2))) <= 1e-5
    assert dfft.device_error() == 0


def test_batch_repeats_plan_with_counters():
    # the same fused plan listed twice in one batch: its counters are shared,
    # so its two uses must not overlap
    a = rand((256, 256, 8), np.complex64, seed=21)
    b = rand((256, 256, 8), np.complex64, seed=22)
    ga, gb = to_gpu(a), to_gpu(b)
    p = _plan(dfft.FFT(), ga, (1, 2, 3))
    assert p.workspace_bytes > 0
    oa = dfft.empty_like_layout(p.out_shape, ga.dtype, ga)
    ob = dfft.empty_like_layout(p.out_shape, gb.dtype, gb)
    B = dfft.Batch([p, p])
    B.execute([ga, gb], [oa, ob])
    torch.cuda.synchronize()
    assert rel(to_np(oa), oracle.fft(a, dims=(1, 2, 3))) <= 1e-5
    assert rel(to_np(ob), oracle.fft(b, dims=(1, 2, 3))) <= 1e-5


def test_untuned_default_per_length():
    # without tuning, 256^2 slabs fuse and 128^2 slabs keep the per-axis
    # passes (faster at that size); both give the oracle's answer
    for L, fused in [(256, True), (128, False)]:
        a = rand((L, L, 16), np.complex64, seed=L)
        g = to_gpu(a)
        p = _plan(dfft.FFT(), g, (1, 2), flags=0)
        assert p.launches == (1 if fused else 2)
        assert rel(to_np(_run(p, g)), oracle.fft(a, dims=(1, 2))) <= 1e-5


# fused variants per (dtype, L), the order of the kernel table
N_VARIANTS = {(np.complex64, 512): 6, (np.complex64, 256): 4, (np.complex64, 128): 2,
              (np.complex128, 512): 3, (np.complex128, 256): 3}


def _forced_slab_plan(tag, g, v, tmp_path):
    # tune once to learn the slab wisdom key, then force variant v through
    # an edited wisdom file
    dfft.wisdom_forget()
    dfft.gpu_plan_transform(tag, g, (1, 2), decomp=dfft.Slab(), flags=dfft.FLAG_TUNE)
    f = tmp_path / "w.txt"
    dfft.wisdom_export(f)
    keys = [ln.split()[0] for ln in f.read_text().splitlines() if "|slab|" in ln]
    assert len(keys) == 1
    f.write_text(f"{keys[0]} {v} 0 0\n")
    dfft.wisdom_forget()
    dfft.wisdom_import(f)
    p = dfft.gpu_plan_transform(tag, g, (1, 2), decomp=dfft.Slab())
    dfft.wisdom_forget()
    return p


@pytest.mark.parametrize("dtype,L", list(N_VARIANTS))
@pytest.mark.parametrize("inverse", [False, True])
def test_every_fused_variant(dtype, L, inverse, tmp_path):
    O = 6
    a = rand((L, L, O), dtype, seed=L + 7 * inverse)
    g = to_gpu(a)
    tag = dfft.IFFT() if inverse else dfft.FFT()
    ref = (oracle.ifft if inverse else oracle.fft)(a, dims=(1, 2))
    radices = set()
    for v in range(N_VARIANTS[(dtype, L)]):
        p = _forced_slab_plan(tag, g, v, tmp_path)
        d = p.describe().strip()
        assert p.launches == 1 and d.startswith("slab-xy"), d
        radices.add(d.split("radices=")[1])
        y = _run(p, g)
        assert dfft.device_error() == 0
        assert rel(to_np(y), ref) <= tol_for(dtype), (v, d)
    if (dtype, L) == (np.complex64, 512):
        assert radices == {"8x8x8", "32x16"}
