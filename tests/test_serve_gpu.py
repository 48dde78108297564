"""Serving runtime (continuous batching): each result is the same alone and
in the mix, admission respects the HBM budget, queued requests can be
cancelled, and latency statistics are reported."""
import numpy as np
import pytest
import torch

import dfft
import dfft_oracle as oracle
from helpers import rand, rel, to_gpu, to_np

pytestmark = [pytest.mark.gpu, pytest.mark.timeout(240, method="thread")]

EDGES = [16, 24, 32, 48, 64]


def _requests(n, seed=0):
    """Mixed requests: C2C ComplexF32/ComplexF64 forward or inverse, R2C
    Float32 forward (rfft) or inverse (irfft), cubic edges."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        e = int(rng.choice(EDGES))
        kind = int(rng.integers(3))
        fwd = bool(rng.integers(2))
        if kind == 0:
            a = rand((e, e, e), np.complex64, seed=1000 + i)
            out.append((dfft.FFT() if fwd else dfft.IFFT(), a, None))
        elif kind == 1:
            a = rand((e, e, e), np.complex128, seed=1000 + i)
            out.append((dfft.FFT() if fwd else dfft.IFFT(), a, None))
        else:
            a = rand((e, e, e), np.float32, seed=1000 + i)
            if fwd:
                out.append((dfft.RFFT(), a, None))
            else:
                out.append((dfft.IRFFT(), oracle.rfft(a).astype(np.complex64), e))
    return out


def _out_meta(t, a, n):
    if isinstance(t, dfft.RFFT):
        return (a.shape[0] // 2 + 1,) + a.shape[1:], torch.complex64
    if isinstance(t, dfft.IRFFT):
        return (n,) + a.shape[1:], torch.float32
    return a.shape, torch.complex64 if a.dtype == np.complex64 else torch.complex128


def _run(server, reqs, ins, concurrent):
    outs, ids = [], []
    for (t, a, n), g in zip(reqs, ins):
        shp, dt = _out_meta(t, a, n)
        o = dfft.empty_like_layout(shp, dt, g)
        outs.append(o)
        rid = server.submit(t, g, dims=(1, 2, 3), n=n, out=o)
        if concurrent:
            ids.append(rid)
        else:
            assert server.wait(rid, 20000) == 0
            server.release(rid)
    for rid in ids:
        assert server.wait(rid, 20000) == 0
        server.release(rid)
    torch.cuda.synchronize()
    return outs


def test_alone_equals_in_the_mix():
    reqs = _requests(40, seed=3)
    ins = [to_gpu(a) for _, a, _ in reqs]
    alone = _run(dfft.Server(1 << 28, slots=1), reqs, ins, concurrent=False)
    srv = dfft.Server(1 << 28, slots=8)
    mixed = _run(srv, reqs, ins, concurrent=True)
    st = srv.stats()
    assert st["completed"] == len(reqs) and st["failed"] == 0
    assert st["peak_running"] > 1, "requests must overlap on the device"
    assert st["p99_ms"] >= st["p50_ms"] > 0
    for (t, a, n), x, y in zip(reqs, alone, mixed):
        assert torch.equal(x, y), f"{t} differs alone vs in the mix"
        if isinstance(t, dfft.FFT):
            ref = oracle.fft(a, dims=(1, 2, 3))
        elif isinstance(t, dfft.IFFT):
            ref = oracle.ifft(a, dims=(1, 2, 3))
        elif isinstance(t, dfft.RFFT):
            ref = oracle.rfft(a, dims=(1, 2, 3))
        else:
            ref = oracle.irfft(a, n, dims=(1, 2, 3))
        tol = 1e-12 if a.dtype == np.complex128 else 1e-5
        assert rel(to_np(y), ref) <= tol


def test_workspace_plans_shared_under_concurrency():
    # plans whose executions need scratch memory -- fused slab-pass counters
    # (256 x 256 x 16 ComplexF32), Bluestein scratch (prime edges 17 and 31),
    # C2R scratch (irfft over three dims) -- run 8 at a time from one
    # resident plan each, every request with its own workspace from the arena
    a1 = rand((256, 256, 16), np.complex64, seed=1)
    a2 = rand((17, 31, 8), np.complex64, seed=2)
    a3 = oracle.rfft(rand((32, 24, 16), np.float32, seed=3)).astype(np.complex64)
    srv = dfft.Server(1 << 30, slots=8)
    jobs = []
    for t, a, n in [(dfft.FFT(), a1, None), (dfft.IFFT(), a2, None), (dfft.IRFFT(), a3, 32)]:
        g = to_gpu(a)
        shp, dt = _out_meta(t, a, n)
        for _ in range(8):
            o = dfft.empty_like_layout(shp, dt, g)
            jobs.append((t, a, n, o, srv.submit(t, g, dims=(1, 2, 3), n=n, out=o)))
    for *_, rid in jobs:
        assert srv.wait(rid, 20000) == 0
        srv.release(rid)
    torch.cuda.synchronize()
    st = srv.stats()
    assert st["completed"] == len(jobs) and st["failed"] == 0
    assert st["resident_plans"] == 3
    assert dfft.device_error() == 0
    first = {}
    for t, a, n, o, _ in jobs:
        if isinstance(t, dfft.FFT):
            ref = oracle.fft(a, dims=(1, 2, 3))
        elif isinstance(t, dfft.IFFT):
            ref = oracle.ifft(a, dims=(1, 2, 3))
        else:
            ref = oracle.irfft(a, n, dims=(1, 2, 3))
        assert rel(to_np(o), ref) <= 1e-5
        key = type(t)
        if key in first:
            assert torch.equal(first[key], o), f"{t}: concurrent copies differ"
        else:
            first[key] = o


def test_budget_admission_and_rejection():
    # host inputs and server-held outputs are staged in the arena: a 1 MiB
    # arena holds at most two 32^3 ComplexF32 requests (2 x 256 KiB each)
    srv = dfft.Server(1 << 20, slots=8)
    big = torch.zeros((64, 64, 64), dtype=torch.complex64).pin_memory()   # 2 MiB input
    with pytest.raises(dfft.DFFTError):
        srv.submit(dfft.FFT(), big)
    assert srv.stats()["rejected"] == 1
    xs = [torch.randn((32, 32, 32), dtype=torch.complex64) for _ in range(12)]
    ids = [srv.submit(dfft.FFT(), x.pin_memory()) for x in xs]
    for rid, x in zip(ids, xs):
        assert srv.wait(rid, 20000) == 0
        res = torch.empty((32, 32, 32), dtype=torch.complex64, device="cuda")
        srv.fetch(rid, res)
        torch.cuda.synchronize()
        srv.release(rid)
        assert rel(to_np(res), oracle.fft(x.numpy(), dims=(1, 2, 3))) <= 1e-5
    st = srv.stats()
    assert st["arena_peak_bytes"] <= st["arena_bytes"]
    assert st["completed"] == 12


def test_cancel_queued_request():
    srv = dfft.Server(1 << 20, slots=1)
    x = torch.zeros((32, 32, 32), dtype=torch.complex64).pin_memory()
    ids = [srv.submit(dfft.FFT(), x) for _ in range(6)]
    cancelled = 0
    for rid in ids[3:]:
        try:
            srv.cancel(rid)
            cancelled += 1
        except dfft.DFFTError:
            pass  # already admitted
    for rid in ids:
        st = srv.wait(rid, 20000)
        assert st in (0, 8)  # success or DFFT_ERROR_CANCELLED
        srv.release(rid)
    assert srv.stats()["cancelled"] == cancelled
