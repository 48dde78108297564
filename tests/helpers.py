"""Shared helpers for the GPU parity tests: seeded inputs, layout control,
and the tolerances stated for each precision."""
import numpy as np
import torch

import dfft_oracle as oracle

# Relative-L2 bounds against the FP64 / long-double oracle.
TOL = {np.complex64: 1e-5, np.float32: 1e-5, np.complex128: 1e-12, np.float64: 1e-12}


def tol_for(dtype):
    return TOL[np.dtype(dtype).type]


def to_gpu(a: np.ndarray, order="F"):
    """Device copy of ``a`` (same logical indexing) with the requested memory
    order: "F" = column-major (Julia's layout), "C" = row-major."""
    if order == "C" or a.ndim <= 1:
        return torch.from_numpy(np.ascontiguousarray(a)).cuda()
    t = torch.from_numpy(np.ascontiguousarray(a.T)).cuda()
    return t.permute(*reversed(range(a.ndim)))


def to_np(t: torch.Tensor):
    return t.detach().cpu().numpy()


def rand(shape, dtype, seed=0, kind="normal"):
    rng = np.random.default_rng(seed)
    real = np.float32 if np.dtype(dtype) in (np.complex64, np.float32) else np.float64
    if kind == "normal":
        draw = lambda: rng.standard_normal(shape)
    elif kind == "uniform01":
        draw = lambda: rng.random(shape)
    else:
        draw = lambda: rng.random(shape) * 2 - 1
    if np.dtype(dtype).kind == "c":
        return (draw().astype(real) + 1j * draw().astype(real)).astype(dtype)
    return draw().astype(dtype)


def rel(a, b):
    return oracle.rel_l2(a, b)
