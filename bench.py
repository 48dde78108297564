"""Benchmark: 512^3 ComplexF32 C2C forward + inverse, Slab decomposition.

One step = one forward 3-D FFT plus one inverse 3-D FFT of a 512^3
ComplexF32 array (iid standard-normal real and imaginary parts,
decomp=Slab()), inputs resident in HBM.

value  : algorithmic GB/s = 2 transforms x 3 axis passes x (read + write of
         the 1 GiB field) = 12.885 GB per step, / step time, summed over ranks.
e2e    : the same bytes / the time per step of the public API call sequence
         with host buffers: pinned H2D of the step's input, fft, ifft, D2H of
         its result; steps double-buffered over three streams so uploads,
         transforms and downloads of consecutive steps overlap.
roofline: the slowest launch of the step (the fused dims-(1,2) slab pass or
         an axis pass), timed alone with CUDA events on its stream:
         algorithmic bytes per launch (2 x 1 GiB per axis it covers) / mean
         launch time vs the measured HBM copy bandwidth in
         MEASURED_PEAKS.json.  A fused launch covers two axes with one DRAM
         sweep, so its fraction can pass 1.0; dram_floor_* gives the rate of
         that single read + write of the field, and traffic the ncu bytes.
cpu_baseline: the oracle's restatement of the reference CPU pipeline
         (Blocks(N,N,64) slabs, per-chunk pocketfft with all host threads,
         block redistribution), one forward+inverse of the same 512^3 field.

--impl reference times that CPU pipeline alone (rank 0), one forward+inverse
per step, and prints its own JSON line (same metric, unit and workload).

errors : relative L2 of the forward result against a float64 host fftn
         (scipy.fft on all host cores) of the same input, of the inverse
         result against the host ifftn of the GPU's forward output, and of
         the round trip against the input.
mixed  : the same step in the mixed (tensor-core) form -- the 512-point
         axes as radix-32 x radix-16 complex matrix products on tcgen05
         with FP16 hi+lo split operands and FP32 accumulation -- timed the
         same way, with its per-launch times, its ratio to the plain step
         and its errors against the float64 host evaluation.
configs: (one GPU) the other configured workloads, each with its time,
         algorithmic GB/s and errors against a float64 host evaluation:
         c1 128^3 ComplexF64 Pencil, c2 256^3 Float64/Float32 rfft+irfft,
         c4 64 uneven ComplexF32 grids as one batch launch + the DCT-II/III
         Float64 stack, c5 serving p50/p99 latency per Poisson arrival rate.

Multi-GPU (torchrun): every rank transforms its own 512^3 field (weak
scaling, replicas: no data-path collective); timing is the max over ranks.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "daggerfft.jl_b200"))

N = 512
FIELD_BYTES = N ** 3 * 8                     # ComplexF32
STEP_BYTES = 2 * 3 * 2 * FIELD_BYTES         # fwd + inv, 3 passes, read + write
PASS_BYTES = 2 * FIELD_BYTES                 # one axis pass
CPU_CHUNK = 64
WORKLOAD = "512^3 ComplexF32 C2C fft+ifft, decomp=Slab(), dims=(1,2,3)"
METRIC = "512^3 C2C FFT GB/s (fwd+inv, algorithmic bytes)"


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def ncu_traffic():
    """Per-launch DRAM bytes of the axis-pass kernels from the committed ncu
    summary (profiles/ncu_traffic.json), or None."""
    p = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    try:
        with open(p) as f:
            return json.load(f)
    except Exception:
        return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id):
        self.gpu = gpu_id
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        try:
            for line in open(self.path):
                parts = [x.strip() for x in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    mx = float(parts[2])
                except ValueError:
                    continue
                for nm, v in zip(names, parts[5:9]):
                    if v.lower() == "active":
                        reasons.add(nm)
            os.unlink(self.path)
        except Exception:
            pass
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_pipeline_once(A, workers):
    """One forward + inverse of the oracle's Slab pipeline on host cores."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import dfft_oracle as oracle
    oracle.WORKERS = workers
    shape = A.shape
    DA, DB = oracle.slab_layouts(shape, CPU_CHUNK, 1)
    oracle.distribute(A, DA)
    wsAB = [oracle.create_workspace(DA, DB, 0)]
    wsBA = [oracle.create_workspace(DB, DA, 0)]
    t0 = time.perf_counter()
    oracle.fft_slab(DB, DA, wsAB, (oracle.FFT_(),) * 3, (1, 2, 3), precision="native")
    DA.chunks = []
    oracle.ifft_slab(DA, DB, wsBA, (oracle.IFFT_(),) * 3, (1, 2, 3), precision="native")
    return time.perf_counter() - t0


def host_input(seed=0):
    import numpy as np
    rng = np.random.default_rng(seed)
    re = rng.standard_normal((N, N, N), dtype=np.float32)
    im = rng.standard_normal((N, N, N), dtype=np.float32)
    a = np.empty((N, N, N), dtype=np.complex64, order="F")
    a.real = re
    a.imag = im
    return a


def run_reference(args, rank, world):
    if rank != 0:
        return
    import numpy as np  # noqa: F401
    workers = os.cpu_count() or 1
    A = host_input()
    for _ in range(args.warmup):
        cpu_pipeline_once(A, workers)
    ts = [cpu_pipeline_once(A, workers) for _ in range(args.steps)]
    t = sum(ts) / len(ts)
    v = STEP_BYTES / t / 1e9
    line = {
        "impl": "reference", "metric": METRIC,
        "value": round(v, 3), "unit": "GB/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(t * 1e3, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "complex64 (f32)", "data": "synthetic",
        "config": {"workload": WORKLOAD, "method": "plain", "global_batch": 1, "seq_len": N,
                   "parallelism": "host threads", "chunks": "Blocks(512,512,64)"},
        "cpu_baseline": {"value": round(v, 3), "unit": "GB/s", "cores": workers, "kind": "port",
                         "sample": "one full 512^3 forward+inverse per step (oracle Slab pipeline, "
                                   "pocketfft stand-in for FFTW)"},
        "e2e": {"value": round(v, 3), "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "gflops": round(5 * N ** 3 * 27 * 1e-9 / (t / 2), 2),
    }
    print(json.dumps(line), flush=True)


def host_errors(A_host, Fd, Bd):
    """Forward result Fd against a float64 host fftn of the input, inverse
    result Bd against the host ifftn of Fd (scipy.fft, all host cores).
    A_host is the pinned (z, y, x) C-order copy of the logical (x, y, z)
    input, so the transforms run over all three axes of the same memory."""
    import numpy as np
    import scipy.fft
    w = os.cpu_count() or 1

    def rel(a, b):
        num = den = 0.0
        for k in range(0, a.shape[0], 32):
            x = a[k:k + 32].astype(np.complex128)
            y = b[k:k + 32]
            num += float(np.sum(np.abs(x - y) ** 2))
            den += float(np.sum(np.abs(y) ** 2))
        return float(np.sqrt(num / den))

    a = A_host.numpy().astype(np.complex128)
    ref = scipy.fft.fftn(a, workers=w, overwrite_x=True)
    del a
    F = Fd.permute(2, 1, 0).cpu().numpy()          # (z, y, x) C order, as A_host
    e_fwd = rel(F, ref)
    del ref
    inv = scipy.fft.ifftn(F.astype(np.complex128), workers=w, overwrite_x=True)
    e_inv = rel(Bd.permute(2, 1, 0).cpu().numpy(), inv)
    return {"fwd_rel_l2_vs_host_fp64": e_fwd, "inv_rel_l2_vs_host_fp64": e_inv,
            "host_oracle": f"scipy.fft float64, {w} threads"}


def run_mixed(args, dfft, decomp, Ad, Bd, Cd, stream, plain_ms, A_host):
    """The step in the mixed form: fwd + inv through method="mixed" plans,
    warm-up, then args.steps steps between CUDA events on the stream."""
    import torch
    try:
        pf = dfft.get_or_create_gpu_plan(dfft.FFT(), Ad, (1, 2, 3), decomp=decomp, method="mixed")
        pi = dfft.get_or_create_gpu_plan(dfft.IFFT(), Bd, (1, 2, 3), decomp=decomp, method="mixed")
    except Exception as e:
        return {"error": f"{type(e).__name__}: {e}"}

    def step():
        pf.execute(Ad, Bd, stream)
        pi.execute(Bd, Cd, stream)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    out = {"ms_per_step": round(ms, 4), "value": round(STEP_BYTES / (ms * 1e-3) / 1e9, 2), "unit": "GB/s",
           "speedup_vs_plain": round(plain_ms / ms, 4), "launches_per_step": pf.launches + pi.launches,
           "kernels": pf.describe().strip().splitlines()}
    # each forward launch alone (one pass per axis)
    per = {}
    for dims in ((1,), (2,), (3,)):
        p = dfft.gpu_plan_transform(dfft.FFT(), Ad, dims, decomp=decomp, method="mixed")
        for _ in range(3):
            p.execute(Ad, Bd, stream)
        a0 = torch.cuda.Event(enable_timing=True)
        a1 = torch.cuda.Event(enable_timing=True)
        a0.record(stream)
        for _ in range(10):
            p.execute(Ad, Bd, stream)
        a1.record(stream)
        torch.cuda.synchronize()
        per[str(dims[0])] = round(a0.elapsed_time(a1) / 10, 4)
        del p
    out["per_launch_ms"] = per
    peak, _ = measured_peak()
    dom = max(per.values())
    out["dominant_frac_of_peak"] = round(PASS_BYTES / (dom * 1e-3) / 1e9 / peak, 4)
    if A_host is not None:
        step()
        torch.cuda.synchronize()
        err = host_errors(A_host, Bd, Cd)
        err["roundtrip_rel_l2"] = float(torch.linalg.vector_norm(Cd - Ad) / torch.linalg.vector_norm(Ad))
        out["errors"] = err
    return out


def run_configs():
    import bench_configs as bc
    out = {}
    for name in ("c1", "c2", "c4", "c5"):
        t0 = time.perf_counter()
        try:
            out[name] = getattr(bc, name)()
        except Exception as e:  # one failing configuration does not drop the headline
            out[name] = {"error": f"{type(e).__name__}: {e}"}
        out[name]["wall_s"] = round(time.perf_counter() - t0, 1)
    return out


def run_profile(args):
    """A short, untimed run for ncu: two executions of a forward C2C
    ComplexF32 plan over the --profile dims (one axis pass, or the fused
    dims-(1,2) slab pass for "12") on a column-major array."""
    import torch
    import dfft
    shape = tuple(int(x) for x in args.shape.split(","))
    torch.cuda.set_device(0)
    g = torch.Generator(device="cuda").manual_seed(0)
    if args.real:
        # Float32 rfft over the --profile dims (the R2C pass first)
        x = torch.randn(tuple(reversed(shape)), dtype=torch.float32, device="cuda", generator=g)
        X = x.permute(*reversed(range(len(shape))))
        dims = tuple(int(c) for c in args.profile)
        flags = 0 if args.no_tune else dfft.FLAG_TUNE
        p = dfft.gpu_plan_transform(dfft.RFFT(), X, dims, flags=flags)
        Y = dfft.empty_like_layout(p.out_shape, torch.complex64, X)
        for _ in range(2):
            p.execute(X, Y)
        torch.cuda.synchronize()
        print(f"profile: rfft dims {dims} of {shape}, {p.launches} launch(es) per call, 2 calls")
        return
    a = torch.randn(tuple(reversed(shape)), dtype=torch.complex64, device="cuda", generator=g)
    A = a.permute(*reversed(range(len(shape))))
    B = dfft.empty_like_layout(A.shape, A.dtype, A)
    dims = tuple(int(c) for c in args.profile)
    flags = (0 if args.no_tune else dfft.FLAG_TUNE) | (dfft.FLAG_NO_FUSE if args.no_fuse else 0)
    if args.slab_variant >= 0:
        # pin the fused slab kernel's variant through a one-line wisdom file
        # (key: device name with blanks as '_', '_sm' + SM count, 'slab',
        # double?, L, O, inverse), so no tuning launches precede the profiled ones
        prop = torch.cuda.get_device_properties(0)
        tag = prop.name.replace(" ", "_").replace("|", "_") + f"_sm{prop.multi_processor_count}"
        with tempfile.NamedTemporaryFile("w", suffix=".wisdom", delete=False) as f:
            f.write(f"{tag}|slab|0|{shape[0]}|{shape[2]}|0 {args.slab_variant} 0 0\n")
        dfft.wisdom_import(f.name)
        os.unlink(f.name)
    p = dfft.gpu_plan_transform(dfft.FFT(), A, dims, method=args.method, flags=flags)
    for _ in range(2):
        p.execute(A, B)
    torch.cuda.synchronize()
    print(f"profile: dims {dims} of {shape}, {p.launches} launch(es) per call, 2 calls")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--method", default="plain", choices=["plain", "mixed"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-mixed", action="store_true",
                    help="skip the mixed (tensor-core) form of the step")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the other configured workloads (c1, c2, c4, c5)")
    ap.add_argument("--no-tune", action="store_true", help="heuristic launch shapes, no autotuning")
    ap.add_argument("--profile", default="",
                    help="profiling mode: run the plan over these dims twice and exit "
                         "(e.g. 1 = the dim-1 pass, 12 = the fused dims-(1,2) slab pass)")
    ap.add_argument("--no-fuse", action="store_true",
                    help="one pass per axis (no fused dims-(1,2) slab pass)")
    ap.add_argument("--shape", default="512,512,512", help="profiling mode: ComplexF32 array shape")
    ap.add_argument("--real", action="store_true",
                    help="profiling mode: a Float32 rfft instead of a ComplexF32 fft")
    ap.add_argument("--slab-variant", type=int, default=-1,
                    help="profiling mode: the fused slab kernel's variant (index into its table)")
    args = ap.parse_args()
    if args.profile:
        run_profile(args)
        return
    args.warmup = max(args.warmup, 3)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        run_reference(args, rank, world)
        return

    import numpy as np
    import torch
    import dfft

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)
        pg = dist

    stream = torch.cuda.current_stream(dev)
    A_host = torch.from_numpy(np.ascontiguousarray(host_input(seed=rank).T)).pin_memory()  # (z,y,x) C = F(x,y,z)
    out_host = torch.empty_like(A_host).pin_memory()
    Ad = A_host.to(dev, non_blocking=False).permute(2, 1, 0)     # logical (x,y,z), column-major
    Bd = dfft.empty_like_layout(Ad.shape, Ad.dtype, Ad)
    Cd = dfft.empty_like_layout(Ad.shape, Ad.dtype, Ad)
    decomp = dfft.Slab()
    flags = (0 if args.no_tune else dfft.FLAG_TUNE) | (dfft.FLAG_NO_FUSE if args.no_fuse else 0)
    pf = dfft.get_or_create_gpu_plan(dfft.FFT(), Ad, (1, 2, 3), decomp=decomp, method=args.method,
                                     flags=flags)
    pi = dfft.get_or_create_gpu_plan(dfft.IFFT(), Bd, (1, 2, 3), decomp=decomp, method=args.method,
                                     flags=flags)
    launches_per_step = pf.launches + pi.launches

    def step():
        pf.execute(Ad, Bd, stream)
        pi.execute(Bd, Cd, stream)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if pg:
        pg.barrier()
    try:
        gid = "GPU-" + str(torch.cuda.get_device_properties(dev).uuid)
    except Exception:
        gid = str(local)
    clocks = ClockSampler(gid)
    clocks.start()
    time.sleep(0.3)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    if pg:
        pg.barrier()
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    t_ms = e0.elapsed_time(e1) / args.steps
    if pg:
        pg.barrier()
    clk = clocks.stop()
    if pg:
        tt = torch.tensor([t_ms], device=dev)
        pg.all_reduce(tt, op=pg.ReduceOp.MAX)
        t_ms = float(tt.item())
    value = world * STEP_BYTES / (t_ms * 1e-3) / 1e9

    # accuracy against a float64 host evaluation of the same input
    rt = float(torch.linalg.vector_norm(Cd - Ad) / torch.linalg.vector_norm(Ad))
    errors = host_errors(A_host, Bd, Cd) if rank == 0 else {}
    errors["roundtrip_rel_l2"] = rt

    # the mixed (tensor-core) form of the same step, unless it is the headline
    mixed = None
    if args.method == "plain" and not args.no_mixed:
        mixed = run_mixed(args, dfft, decomp, Ad, Bd, Cd, stream, t_ms, A_host if rank == 0 else None)

    # the step's launches timed alone (roofline of the dominant one): the
    # forward plan is either the fused dims-(1,2) slab pass + the dim-3 pass,
    # or one pass per axis
    groups = [(1, 2), (3,)] if pf.launches == 2 else [(1,), (2,), (3,)]
    per_launch = {}
    for dims in groups:
        p = dfft.gpu_plan_transform(dfft.FFT(), Ad, dims, decomp=decomp, method=args.method, flags=flags)
        for _ in range(3):
            p.execute(Ad, Bd, stream)
        a0 = torch.cuda.Event(enable_timing=True)
        a1 = torch.cuda.Event(enable_timing=True)
        reps = 10
        a0.record(stream)
        for _ in range(reps):
            p.execute(Ad, Bd, stream)
        a1.record(stream)
        torch.cuda.synchronize()
        per_launch[dims] = (a0.elapsed_time(a1) / reps / p.launches, len(dims) // p.launches)
        del p
    dom = max(per_launch, key=lambda k: per_launch[k][0])
    dom_ms, dom_axes = per_launch[dom]
    peak, peak_kind = measured_peak()
    # algorithmic bytes: each axis a launch covers reads and writes the field
    # once (a fused launch counts its two axes); the DRAM floor of any launch
    # is one read and one write of the field
    achieved = dom_axes * PASS_BYTES / (dom_ms * 1e-3) / 1e9
    dram_floor_gbs = PASS_BYTES / (dom_ms * 1e-3) / 1e9
    traffic = None
    tr = ncu_traffic()
    if tr:
        if len(dom) == 2:
            traffic = tr.get("slab_pass_bytes")
        elif str(dom[0]) in tr.get("axis_pass_bytes", {}):
            traffic = tr["axis_pass_bytes"][str(dom[0])]
    dom_name = ("fused slab pass dims (1,2)" if len(dom) == 2 else f"axis pass dim {dom[0]}")

    # end-to-end through the public API with host buffers: every step uploads
    # its input from pinned host memory, runs fft and ifft, and downloads the
    # result.  Steps are double-buffered over three streams, so the upload of
    # step i+1 and the download of step i-1 overlap step i's transforms (the
    # two copy directions run on separate copy engines); every step still
    # moves its own input and result over PCIe inside the timed region.
    torch.cuda.synchronize()
    if pg:
        pg.barrier()
    A2 = dfft.empty_like_layout(Ad.shape, Ad.dtype, Ad)
    B2 = dfft.empty_like_layout(Ad.shape, Ad.dtype, Ad)
    C2 = dfft.empty_like_layout(Ad.shape, Ad.dtype, Ad)
    out_host2 = torch.empty_like(A_host).pin_memory()
    sets = [(Ad, Bd, Cd, out_host), (A2, B2, C2, out_host2)]
    s_in, s_cmp, s_out = (torch.cuda.Stream(dev) for _ in range(3))
    ev_in = [torch.cuda.Event() for _ in range(2)]
    ev_cmp = [torch.cuda.Event() for _ in range(2)]
    ev_out = [torch.cuda.Event() for _ in range(2)]

    def e2e_step(i):
        k = i % 2
        A, B, C, host = sets[k]
        if i >= 2:
            s_in.wait_event(ev_cmp[k])   # step i-2 has finished reading A
        with torch.cuda.stream(s_in):
            A.permute(2, 1, 0).copy_(A_host, non_blocking=True)
        ev_in[k].record(s_in)
        s_cmp.wait_event(ev_in[k])
        if i >= 2:
            s_cmp.wait_event(ev_out[k])  # step i-2's download has read C
        pf.execute(A, B, s_cmp)
        pi.execute(B, C, s_cmp)
        ev_cmp[k].record(s_cmp)
        s_out.wait_event(ev_cmp[k])
        with torch.cuda.stream(s_out):
            host.copy_(C.permute(2, 1, 0), non_blocking=True)
        ev_out[k].record(s_out)

    for i in range(2):
        e2e_step(i)
    torch.cuda.synchronize()
    ee0 = torch.cuda.Event(enable_timing=True)
    ee1 = torch.cuda.Event(enable_timing=True)
    e2e_steps = max(4, min(args.steps, 10))
    ee0.record(s_in)
    for i in range(e2e_steps):
        e2e_step(i)
    ee1.record(s_out)
    torch.cuda.synchronize()
    e2e_ms = ee0.elapsed_time(ee1) / e2e_steps
    if pg:
        tt = torch.tensor([e2e_ms], device=dev)
        pg.all_reduce(tt, op=pg.ReduceOp.MAX)
        e2e_ms = float(tt.item())
    e2e = world * STEP_BYTES / (e2e_ms * 1e-3) / 1e9
    e2e_ok = bool(torch.equal(out_host, out_host2))  # both buffers hold ifft(fft(A))
    del A2, B2, C2
    torch.cuda.empty_cache()

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        workers = os.cpu_count() or 1
        a_np = A_host.numpy().T  # logical (x,y,z), Fortran order
        t_cpu = cpu_pipeline_once(a_np, workers)
        cpu = {"value": round(STEP_BYTES / t_cpu / 1e9, 3), "unit": "GB/s", "cores": workers,
               "kind": "port",
               "sample": "one 512^3 ComplexF32 forward+inverse (oracle Slab pipeline: Blocks(512,512,64) "
                         "chunks, pocketfft per chunk with all host threads, block redistribution)"}

    configs = None
    if rank == 0 and world == 1 and not args.no_configs:
        # the other configured workloads: the 512^3 buffers are freed first
        # (the serving arena takes 16 GiB)
        del Ad, Bd, Cd, pf, pi, sets
        import gc
        gc.collect()
        dfft.gpu_cleanup_plans()
        torch.cuda.synchronize()
        torch.cuda.empty_cache()
        configs = run_configs()

    if pg:
        pg.barrier()
    if rank == 0:
        line = {
            "metric": METRIC,
            "value": round(value, 2), "unit": "GB/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(t_ms, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "complex64 (f32)",
            "data": "synthetic",
            "config": {"workload": WORKLOAD,
                       "method": args.method, "global_batch": world, "seq_len": N,
                       "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                       "l2": "inputs (1 GiB) larger than L2 (126 MB); no flush needed"},
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak,
                         "peak_kind": peak_kind, "unit": "GB/s", "frac": round(achieved / peak, 4),
                         "traffic": traffic, "kernel": dom_name,
                         "algorithmic_bytes_per_launch": dom_axes * PASS_BYTES,
                         "dram_floor_gbs": round(dram_floor_gbs, 1),
                         "dram_floor_frac": round(dram_floor_gbs / peak, 4),
                         "per_launch_ms": {",".join(map(str, k)): round(v[0], 4) for k, v in per_launch.items()},
                         "step_frac_of_peak": round(value / world / peak, 4),
                         # B200 HBM3e nominal 8 TB/s, for context beside the measured peak
                         "nominal_gbs": 8000.0,
                         "frac_of_nominal": round(achieved / 8000.0, 4),
                         "step_frac_of_nominal": round(value / world / 8000.0, 4)},
            "e2e": {"value": round(e2e, 2), "unit": "GB/s", "ms_per_step": round(e2e_ms, 3),
                    "h2d_bytes_per_step": FIELD_BYTES, "d2h_bytes_per_step": FIELD_BYTES,
                    "overlap": "double-buffered: upload i+1 / transforms i / download i-1 on three streams",
                    "results_consistent": e2e_ok},
            "cpu_baseline": cpu,
            "gpu_launches": launches_per_step * args.steps,
            "gflops": round(5 * N ** 3 * 27 * 1e-9 / (t_ms * 1e-3 / 2), 1),
            "errors": errors,
            "clocks": clk,
        }
        if mixed is not None:
            line["mixed"] = mixed
        if configs is not None:
            line["configs"] = configs
        print(json.dumps(line), flush=True)
    if pg:
        pg.barrier()
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
