"""The no-allocation irfft entry point (dfft_irfft_noalloc_f32), called
through the C ABI, against the regular irfft entry point.

That entry point serves callers that cannot call cudaMalloc while they
transform (code inside another framework's memory pool or under a fixed
HBM budget): its intermediate lives in a static device array and its
twiddles are computed in the kernel.  Two calls in a row must both match
the regular path, since the static array keeps the previous call's
contents.  This file is collected last on purpose."""
import ctypes

import numpy as np
import pytest
import torch

import dfft
from dfft import _lib
from helpers import rand, rel, to_gpu, to_np

pytestmark = pytest.mark.gpu


def _noalloc(F: torch.Tensor, shape):
    L = _lib.lib()
    L.dfft_irfft_noalloc_f32.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                         ctypes.POINTER(ctypes.c_int64), ctypes.c_void_p]
    L.dfft_irfft_noalloc_f32.restype = ctypes.c_int
    out = dfft.empty_like_layout(shape, torch.float32, F)
    st = L.dfft_irfft_noalloc_f32(ctypes.c_void_p(F.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                                  len(shape), _lib.i64_array(shape),
                                  ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    return st, out


@pytest.mark.parametrize("shape", [(64, 48, 20), (45, 16, 8), (96, 40), (50,)])
def test_noalloc_matches_irfft_twice(shape):
    for call, seed in enumerate((11, 12)):
        a = rand(shape, np.float32, seed=seed + len(shape))
        F = dfft.rfft(to_gpu(a), dims=tuple(range(1, len(shape) + 1)))
        ref = dfft.irfft(F, shape[0], dims=tuple(range(1, len(shape) + 1)))
        st, out = _noalloc(F, shape)
        assert st == 0, _lib.lib().dfft_last_error()
        torch.cuda.synchronize()
        assert rel(to_np(out), to_np(ref)) <= 1e-5, f"call {call}"
        assert rel(to_np(out), a) <= 1e-5


def test_noalloc_rejects_oversize():
    F = torch.zeros((129, 256, 128), dtype=torch.complex64, device="cuda")
    st, _ = _noalloc(F, (256, 256, 128))
    assert st == _lib.ERROR_INVALID_VALUE
    assert b"static workspace" in _lib.lib().dfft_last_error()
