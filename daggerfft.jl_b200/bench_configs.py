"""Measurements of the non-headline configurations (one JSON line each).

  c1  128^3 ComplexF64 fft+ifft, Pencil, uniform [0,1) -- beside the CPU
      pipeline (the oracle's Pencil restatement, Blocks(128,32,32)).
  c2  256^3 Float64 and Float32 rfft+irfft, Pencil, uniform [0,1).
  c4  64 independent 3-D C2C ComplexF32 grids, edges from
      {48,64,80,96,120,128,160,192}, uniform [-1,1), as one launch of the
      persistent batch kernel (dfft.Batch), beside the graph of the plans'
      passes and the same plans launched one after another; plus the
      2-D DCT-II/III Float64 256x256x32 stack.
  c5  serving: Poisson arrivals at swept rates into dfft.Server; each
      request a forward or inverse 3-D FFT (C2C ComplexF32 / ComplexF64 or
      R2C Float32) with cubic edge from {64,96,128,192,256,384} (weights
      30/20/20/15/10/5 %), standard-normal inputs from per-request seeds
      (a pool of resident inputs per kind and edge); results stay in the
      server arena and are released on completion; p50/p99 latency and
      throughput per rate.

Usage: python daggerfft.jl_b200/bench_configs.py [c1 c2 c4 ...]
(bench.py runs the same functions and puts their dicts in its JSON line).
Times are CUDA-event averages after warm-up; bytes are algorithmic (one
read + one write of the field per axis pass).  Every error is a relative L2
against a float64 host evaluation (scipy.fft / pocketfft on all host
cores) of the same input: the forward result against fftn / rfftn / dctn,
the inverse result against the host inverse of the GPU's own forward
output, and the round trip against the input.
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


WORKERS = os.cpu_count() or 1


def host(t):
    """Host float64 / complex128 copy of a device tensor, logical indexing."""
    x = t.detach().cpu().numpy()
    return x.astype(np.complex128 if np.iscomplexobj(x) else np.float64)


def hrel(a, b):
    """Relative L2 of host arrays (float64 accumulation)."""
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.sqrt(np.sum(np.abs(a - b) ** 2) / np.sum(np.abs(b) ** 2)))


def sfft():
    import scipy.fft
    return scipy.fft


def c1(cpu=True):
    """128^3 ComplexF64 fft + ifft, Pencil, U[0,1) real and imaginary parts."""
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
    pf.execute(A, B)
    pi.execute(B, C)
    torch.cuda.synchronize()
    a, Bh, Ch = host(A), host(B), host(C)
    fx = sfft()
    out = {"config": "c1 128^3 ComplexF64 fft+ifft Pencil, U[0,1)", "ms_per_fwd_inv": round(ms, 4),
           "GBps": round(step_bytes / ms / 1e6, 1),
           "fwd_rel_l2_vs_host_fp64": hrel(Bh, fx.fftn(a, workers=WORKERS)),
           "inv_rel_l2_vs_host_fp64": hrel(Ch, fx.ifftn(Bh, workers=WORKERS)),
           "roundtrip_rel_l2": hrel(Ch, a)}
    if cpu:
        # the reference's CPU pipeline (the oracle's Pencil restatement,
        # Blocks(128,32,32), pocketfft per chunk on all host threads), one forward
        sys.path.insert(0, os.path.join(HERE, "..", "oracle"))
        import dfft_oracle as oracle
        oracle.WORKERS = WORKERS
        DA, DB, DC = oracle.pencil_layouts((n, n, n), 32, 1)
        oracle.distribute(a, DA)
        ws = [oracle.create_workspace(DA, DB, 0)], [oracle.create_workspace(DB, DC, 0)]
        t0 = time.perf_counter()
        oracle.fft_pencil(DC, DA, DB, ws[0], ws[1], (oracle.FFT_(),) * 3, (1, 2, 3), precision="native")
        t_cpu_f = time.perf_counter() - t0
        out["cpu_baseline"] = {"ms_fwd": round(t_cpu_f * 1e3, 2), "threads": WORKERS, "kind": "port",
                               "sample": "one 128^3 forward (oracle Pencil pipeline, pocketfft stand-in for FFTW)"}
    return out


def c2():
    """256^3 Float64 and Float32 rfft + irfft, Pencil, U[0,1)."""
    n = 256
    res = []
    fx = sfft()
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
        pf.execute(A, F)
        pi.execute(F, X)
        torch.cuda.synchronize()
        a, Fh, Xh = host(A), host(F), host(X)
        # rfft halves the first (logical) axis: the real transform runs over
        # the last axis listed
        ref = fx.rfftn(a, axes=(2, 1, 0), workers=WORKERS)
        inv = fx.irfftn(Fh, s=(n, n, n), axes=(2, 1, 0), workers=WORKERS)
        res.append({"precision": "Float64" if dt == torch.float64 else "Float32",
                    "ms_per_fwd_inv": round(ms, 4), "GBps": round(step / ms / 1e6, 1),
                    "fwd_rel_l2_vs_host_fp64": hrel(Fh, ref),
                    "inv_rel_l2_vs_host_fp64": hrel(Xh, inv),
                    "roundtrip_rel_l2": hrel(Xh, a)})
    return {"config": "c2 256^3 rfft+irfft Pencil, U[0,1)", "results": res}


def c4():
    """64 uneven ComplexF32 grids as one batch launch, and the 2-D
    DCT-II / DCT-III Float64 256 x 256 x 32 stack."""
    edges = [48, 64, 80, 96, 120, 128, 160, 192]
    rng = np.random.default_rng(4)
    shapes = [tuple(int(e) for e in rng.choice(edges, 3)) for _ in range(64)]
    g = torch.Generator(device="cuda").manual_seed(4)
    ins = [fcol(torch.complex(torch.rand(tuple(reversed(s)), device="cuda", generator=g) * 2 - 1,
                              torch.rand(tuple(reversed(s)), device="cuda", generator=g) * 2 - 1))
           for s in shapes]
    plans = [dfft.gpu_plan_transform(dfft.FFT(), x, (1, 2, 3), flags=dfft.FLAG_TUNE) for x in ins]
    outs = [dfft.empty_like_layout(p.out_shape, x.dtype, x) for p, x in zip(plans, ins)]
    graph = dfft.Batch(plans)                     # the graph of the plans' own passes
    persist = dfft.Batch(plans, persistent=True)  # the persistent kernel: one launch
    ms_graph = timed(lambda: graph.execute(ins, outs))
    ms_persist = timed(lambda: persist.execute(ins, outs))
    by_lag = {}
    for lag in (1, 4, 16, 64):
        b = dfft.Batch(plans, persistent=True, lag=lag)
        by_lag[str(lag)] = round(timed(lambda: b.execute(ins, outs)), 4)
        del b
    ms_seq = timed(lambda: [p.execute(x, o) for p, x, o in zip(plans, ins, outs)])
    persist.execute(ins, outs)
    torch.cuda.synchronize()
    fx = sfft()
    err_p = max(hrel(host(o), fx.fftn(host(x), workers=WORKERS)) for x, o in zip(ins, outs))
    graph.execute(ins, outs)
    torch.cuda.synchronize()
    err = max(hrel(host(o), fx.fftn(host(x), workers=WORKERS)) for x, o in zip(ins, outs))
    elems = sum(a * b * c for a, b, c in shapes)
    byts = 3 * 2 * elems * 8
    # DCT-II / DCT-III Float64 256x256 x 32 (dims 1,2)
    D = fcol(torch.rand((32, 256, 256), device="cuda", dtype=torch.float64, generator=g))
    p2 = dfft.gpu_plan_transform(dfft.R2R((dfft.REDFT10, dfft.REDFT10)), D, (1, 2))
    p3 = dfft.gpu_plan_transform(dfft.R2R((dfft.REDFT01, dfft.REDFT01)), D, (1, 2))
    E = dfft.empty_like_layout(D.shape, D.dtype, D)
    R = dfft.empty_like_layout(D.shape, D.dtype, D)
    ms_dct = timed(lambda: (p2.execute(D, E), p3.execute(E, R)))
    p2.execute(D, E)
    p3.execute(E, R)
    torch.cuda.synchronize()
    dbytes = 2 * 2 * 2 * 256 * 256 * 32 * 8
    d, Eh, Rh = host(D), host(E), host(R)
    # scipy's unnormalised DCT-II / DCT-III are FFTW's REDFT10 / REDFT01
    return {"config": "c4 64 uneven C2C ComplexF32 grids as one graph launch (and as one persistent-kernel launch); DCT-II/III Float64 256x256x32",
            "grids": len(shapes), "elements": elems,
            "kernel_launches_in_graph": graph.launches,
            "ms_graph": round(ms_graph, 4), "GBps_graph": round(byts / ms_graph / 1e6, 1),
            "persistent_kernel_launches": persist.launches,
            "ms_persistent": round(ms_persist, 4), "GBps_persistent": round(byts / ms_persist / 1e6, 1),
            "ms_persistent_by_lag": by_lag,
            "ms_sequential_launches": round(ms_seq, 4),
            "GBps_sequential": round(byts / ms_seq / 1e6, 1),
            "grids_worst_fwd_rel_l2_vs_host_fp64": err,
            "grids_worst_fwd_rel_l2_vs_host_fp64_persistent": err_p,
            "dct2_dct3_256x256x32_f64_ms": round(ms_dct, 4),
            "dct_GBps": round(dbytes / ms_dct / 1e6, 1),
            "dct2_rel_l2_vs_host_fp64": hrel(Eh, fx.dctn(d, type=2, axes=(0, 1), workers=WORKERS)),
            "dct3_rel_l2_vs_host_fp64": hrel(Rh, fx.dctn(Eh, type=3, axes=(0, 1), workers=WORKERS)),
            "dct_roundtrip_rel_l2": hrel(Rh / (4 * 256 * 256), d)}


def c5(rates=(250, 500, 1000, 2000, 4000), seconds=2.0, budget=16 << 30, slots=8):
    import gc
    import random
    # plans and buffers of the configurations run before this one are freed
    # now, not by the garbage collector inside the measured window
    # (cudaFree waits for the device)
    gc.collect()
    dfft.gpu_cleanup_plans()
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    edges = [64, 96, 128, 192, 256, 384]
    weights = [30, 20, 20, 15, 10, 5]
    kinds = ["c2c32", "c2c64", "r2c32"]
    pool = {}
    g = torch.Generator(device="cuda").manual_seed(5)
    for k in kinds:
        for e in edges:
            vs = []
            for v in range(2):
                if k == "c2c32":
                    fwd_in = fcol(torch.randn((e, e, e), device="cuda", dtype=torch.complex64, generator=g))
                    inv_in = fwd_in
                elif k == "c2c64":
                    fwd_in = fcol(torch.randn((e, e, e), device="cuda", dtype=torch.complex128, generator=g))
                    inv_in = fwd_in
                else:
                    fwd_in = fcol(torch.randn((e, e, e), device="cuda", dtype=torch.float32, generator=g))
                    inv_in = dfft.rfft(fwd_in)
                vs.append((fwd_in, inv_in))
            pool[(k, e)] = vs
    srv = dfft.Server(budget, slots=slots)

    def submit(k, e, fwd, v):
        a_f, a_i = pool[(k, e)][v]
        if k == "r2c32":
            return srv.submit(dfft.RFFT(), a_f) if fwd else srv.submit(dfft.IRFFT(), a_i, n=e)
        return srv.submit(dfft.FFT() if fwd else dfft.IFFT(), a_f if fwd else a_i)

    # plans resident before timing: every kind/edge/direction `slots` times
    # at once, so plans that need one instance per running request exist
    warm = [submit(k, e, f, 0) for k in kinds for e in edges for f in (True, False) for _ in range(slots)]
    for rid in warm:
        srv.wait(rid, 60000)
        srv.release(rid)
    srv.poll()  # drop the warm-up ids from the finished list
    results = []
    rng = random.Random(7)
    for lam in rates:
        srv.reset_stats()
        t_end = time.perf_counter() + seconds
        t_next = time.perf_counter()
        outstanding = set()
        n_sub = 0
        while True:
            now = time.perf_counter()
            if now >= t_end:
                break
            while t_next <= now:
                e = rng.choices(edges, weights)[0]
                k = kinds[rng.randrange(3)]
                outstanding.add(submit(k, e, rng.random() < 0.5, rng.randrange(2)))
                n_sub += 1
                t_next += rng.expovariate(lam)
            for rid in srv.poll():
                if rid in outstanding:
                    srv.release(rid)
                    outstanding.discard(rid)
            time.sleep(0.0002)
        for rid in list(outstanding):
            srv.wait(rid, 120000)
            srv.release(rid)
        srv.poll()
        st = srv.stats()
        results.append({"rate_req_per_s": lam, "submitted": n_sub, "completed": st["completed"],
                        "p50_ms": round(st["p50_ms"], 3), "p99_ms": round(st["p99_ms"], 3),
                        "max_ms": round(st["max_ms"], 3),
                        "throughput_req_per_s": round(st["completed"] / st["elapsed_s"], 1),
                        "io_GBps": round(st["bytes_moved"] / st["elapsed_s"] / 1e9, 2),
                        "peak_running": st["peak_running"], "arena_peak_GB": round(st["arena_peak_bytes"] / 1e9, 2)})
    srv.close()
    return {"config": "c5 serving, Poisson arrivals, mixed fft/ifft/rfft/irfft",
            "slots": slots, "hbm_budget_GB": budget / 1e9, "seconds_per_rate": seconds,
            "rates": results}


if __name__ == "__main__":
    todo = sys.argv[1:] or ["c1", "c2", "c4"]
    for name in todo:
        print(json.dumps(globals()[name]()), flush=True)
