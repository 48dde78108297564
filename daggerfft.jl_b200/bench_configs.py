"""Measurements of the non-headline configurations (one JSON line each).

  c1  128^3 ComplexF64 fft+ifft, Pencil, uniform [0,1) -- beside the CPU
      pipeline (the oracle's Pencil restatement, Blocks(128,32,32)).
  c2  256^3 Float64 and Float32 rfft+irfft, Pencil, uniform [0,1).
  c4  64 independent 3-D C2C ComplexF32 grids, edges from
      {48,64,80,96,120,128,160,192}, uniform [-1,1), as one graph launch
      (dfft.Batch) vs the same plans launched one after another; plus the
      2-D DCT-II/III Float64 256x256x32 stack.

Usage: python daggerfft.jl_b200/bench_configs.py [c1 c2 c4 ...]
Times are CUDA-event averages after warm-up; bytes are algorithmic (one
read + one write of the field per axis pass).
"""
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

import numpy as np  # noqa: E402
import torch  # noqa: E402

import dfft  # noqa: E402


def timed(fn, reps=20, warm=3):
    for _ in range(warm):
        fn()
    torch.cuda.synchronize()
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(reps):
        fn()
    b.record()
    torch.cuda.synchronize()
    return a.elapsed_time(b) / reps


def fcol(t):
    """Column-major view of a contiguous C tensor of reversed shape."""
    return t.permute(*reversed(range(t.dim())))


def rel(a, b):
    return float(torch.linalg.vector_norm((a - b).to(torch.complex128)) /
                 torch.linalg.vector_norm(b.to(torch.complex128)))


def c1():
    n = 128
    g = torch.Generator(device="cuda").manual_seed(1)
    A = fcol(torch.complex(torch.rand((n, n, n), device="cuda", dtype=torch.float64, generator=g),
                           torch.rand((n, n, n), device="cuda", dtype=torch.float64, generator=g)))
    pf = dfft.gpu_plan_transform(dfft.FFT(), A, (1, 2, 3), decomp=dfft.Pencil(), flags=dfft.FLAG_TUNE)
    B = dfft.empty_like_layout(A.shape, A.dtype, A)
    C = dfft.empty_like_layout(A.shape, A.dtype, A)
    pi = dfft.gpu_plan_transform(dfft.IFFT(), B, (1, 2, 3), decomp=dfft.Pencil(), flags=dfft.FLAG_TUNE)
    ms = timed(lambda: (pf.execute(A, B), pi.execute(B, C)))
    step_bytes = 2 * 3 * 2 * n ** 3 * 16
    # the CPU pipeline of the reference (oracle port), one fwd+inv
    sys.path.insert(0, os.path.join(HERE, "..", "oracle"))
    import dfft_oracle as oracle
    oracle.WORKERS = os.cpu_count() or 1
    a = A.cpu().numpy()
    DA, DB, DC = oracle.pencil_layouts((n, n, n), 32, 1)
    oracle.distribute(a, DA)
    ws = [oracle.create_workspace(DA, DB, 0)], [oracle.create_workspace(DB, DC, 0)]
    t0 = time.perf_counter()
    oracle.fft_pencil(DC, DA, DB, ws[0], ws[1], (oracle.FFT_(),) * 3, (1, 2, 3), precision="native")
    t_cpu_f = time.perf_counter() - t0
    err = oracle.rel_l2(oracle.collect(DC), np.fft.fftn(a))
    print(json.dumps({"config": "c1 128^3 ComplexF64 fft+ifft Pencil", "gpu_ms_per_fwd_inv": round(ms, 4),
                      "gpu_GBps": round(step_bytes / ms / 1e6, 1),
                      "cpu_ms_fwd": round(t_cpu_f * 1e3, 2), "cpu_threads": oracle.WORKERS,
                      "roundtrip_rel_l2": rel(C, A), "cpu_fwd_rel_l2_vs_fftn": err}), flush=True)


def c2():
    n = 256
    for dt in (torch.float64, torch.float32):
        g = torch.Generator(device="cuda").manual_seed(2)
        A = fcol(torch.rand((n, n, n), device="cuda", dtype=dt, generator=g))
        pf = dfft.gpu_plan_transform(dfft.RFFT(), A, (1, 2, 3), flags=dfft.FLAG_TUNE)
        ct = torch.complex128 if dt == torch.float64 else torch.complex64
        F = dfft.empty_like_layout(pf.out_shape, ct, A)
        pi = dfft.gpu_plan_transform(dfft.IRFFT(), F, (1, 2, 3), n=n, flags=dfft.FLAG_TUNE)
        X = dfft.empty_like_layout(A.shape, dt, A)
        ms = timed(lambda: (pf.execute(A, F), pi.execute(F, X)))
        sr = 8 if dt == torch.float64 else 4
        sc = 2 * sr
        h = n // 2 + 1
        fwd = n ** 3 * sr + h * n * n * sc + 2 * 2 * h * n * n * sc
        step = 2 * fwd
        # forward vs the FP64 path of this library on the same input
        F64 = dfft.rfft(A.to(torch.float64), dims=(1, 2, 3))
        print(json.dumps({"config": f"c2 256^3 {'Float64' if dt == torch.float64 else 'Float32'} rfft+irfft Pencil",
                          "ms_per_fwd_inv": round(ms, 4), "GBps": round(step / ms / 1e6, 1),
                          "fwd_rel_l2_vs_fp64": rel(F.to(torch.complex128), F64),
                          "roundtrip_rel_l2": rel(X, A)}), flush=True)


def c4():
    edges = [48, 64, 80, 96, 120, 128, 160, 192]
    rng = np.random.default_rng(4)
    shapes = [tuple(int(e) for e in rng.choice(edges, 3)) for _ in range(64)]
    g = torch.Generator(device="cuda").manual_seed(4)
    ins = [fcol(torch.complex(torch.rand(tuple(reversed(s)), device="cuda", generator=g) * 2 - 1,
                              torch.rand(tuple(reversed(s)), device="cuda", generator=g) * 2 - 1))
           for s in shapes]
    plans = [dfft.gpu_plan_transform(dfft.FFT(), x, (1, 2, 3), flags=dfft.FLAG_TUNE) for x in ins]
    outs = [dfft.empty_like_layout(p.out_shape, x.dtype, x) for p, x in zip(plans, ins)]
    batch = dfft.Batch(plans)
    ms_graph = timed(lambda: batch.execute(ins, outs))
    ms_seq = timed(lambda: [p.execute(x, o) for p, x, o in zip(plans, ins, outs)])
    elems = sum(a * b * c for a, b, c in shapes)
    byts = 3 * 2 * elems * 8
    # DCT-II / DCT-III Float64 256x256 x 32 (dims 1,2)
    D = fcol(torch.rand((32, 256, 256), device="cuda", dtype=torch.float64, generator=g))
    p2 = dfft.gpu_plan_transform(dfft.R2R((dfft.REDFT10, dfft.REDFT10)), D, (1, 2))
    p3 = dfft.gpu_plan_transform(dfft.R2R((dfft.REDFT01, dfft.REDFT01)), D, (1, 2))
    E = dfft.empty_like_layout(D.shape, D.dtype, D)
    R = dfft.empty_like_layout(D.shape, D.dtype, D)
    ms_dct = timed(lambda: (p2.execute(D, E), p3.execute(E, R)))
    dbytes = 2 * 2 * 2 * 256 * 256 * 32 * 8
    err = rel(R / (4 * 256 * 256), D)
    print(json.dumps({"config": "c4 64 uneven C2C ComplexF32 grids, one graph launch",
                      "grids": len(shapes), "elements": elems, "kernel_launches_in_graph": batch.launches,
                      "ms_graph": round(ms_graph, 4), "ms_sequential_launches": round(ms_seq, 4),
                      "GBps_graph": round(byts / ms_graph / 1e6, 1),
                      "GBps_sequential": round(byts / ms_seq / 1e6, 1),
                      "dct2_dct3_256x256x32_f64_ms": round(ms_dct, 4),
                      "dct_GBps": round(dbytes / ms_dct / 1e6, 1),
                      "dct_roundtrip_rel_l2": err}), flush=True)


if __name__ == "__main__":
    todo = sys.argv[1:] or ["c1", "c2", "c4"]
    for name in todo:
        globals()[name]()
