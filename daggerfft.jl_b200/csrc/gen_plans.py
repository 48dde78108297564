"""Generates the static-plan kernel instantiations (plans_<dtype>_<k>.cu).

For every 5-smooth length L (up to 4096 for single, 2048 for double
precision) it picks a radix sequence with the fewest stages drawn from
{2,3,4,5,6,8,10,12,15,16} (ties: most balanced), the thread count P per
column (one butterfly of the largest radix per thread and stage), and a
__launch_bounds__ that leaves room for the per-thread registers.  Each entry
is registered in a table the planner searches at plan time.

Run from this directory: ``python gen_plans.py`` (the Makefile does).
"""
import itertools
import math
import os

RADICES = [16, 15, 12, 10, 8, 6, 5, 4, 3, 2]
NFILES = 6


def smooth5(n):
    for p in (2, 3, 5):
        while n % p == 0:
            n //= p
    return n == 1


def factorizations(n, maxr=16):
    """All multisets of radices from RADICES whose product is n."""
    out = []

    def rec(rem, start, cur):
        if rem == 1:
            out.append(list(cur))
            return
        for i in range(start, len(RADICES)):
            r = RADICES[i]
            if r <= maxr and rem % r == 0:
                cur.append(r)
                rec(rem // r, i, cur)
                cur.pop()

    rec(n, 0, [])
    return out


def choose(n):
    if n == 1:
        return [1]
    best = None
    for f in factorizations(n):
        key = (len(f), max(f) - min(f), -max(f))
        if best is None or key < best[0]:
            best = (key, f)
    f = best[1]
    # stages without a twiddle multiply first: put the non-power-of-two
    # radices at the front, then the rest largest-first
    odd = sorted([r for r in f if r & (r - 1)], reverse=True)
    pow2 = sorted([r for r in f if not r & (r - 1)], reverse=True)
    return odd + pow2


def threads_per_column(n, rad):
    return max(1, math.ceil(n / max(rad)))


def elems_per_thread(n, rad, P):
    return max(math.ceil((n // r) / P) * r for r in rad)


def launch_bound(dbl, E):
    regs = (4 if dbl else 2) * E + 32
    if regs <= 64:
        return 1024
    if regs <= 128:
        return 512
    return 256


def has_tma(dt, n):
    """C2C lengths that get the TMA-pipelined kernels (three tile buffers of
    at least 4 columns must fit in shared memory)."""
    esz = 8 if dt == "float" else 16
    return 8 <= n and 3 * 4 * n * esz + 128 <= 227 * 1024 and n <= (1024 if dt == "float" else 512)


def tma_bound(dt, lb):
    """The tile loop keeps more state live than the one-tile kernel: double
    precision gets 128 registers per thread (512 threads per CTA)."""
    return min(lb, 512) if dt == "double" else lb


def strided_c(dt, n, P, tlb):
    """Columns per tile of the strided pipelined kernel (compile time): rows
    of 128 bytes (16 complex float / 8 complex double), halved until three
    tile buffers fit in shared memory and C*P threads fit the launch bound,
    but never below 2 (16-byte TMA rows)."""
    esz = 8 if dt == "float" else 16
    C = 16 if dt == "float" else 8
    while C > 2 and (C * P > tlb or 3 * C * n * esz + 128 > 227 * 1024):
        C //= 2
    return C


def main():
    here = os.path.dirname(os.path.abspath(__file__))
    entries = []
    for dt, lim in (("float", 4096), ("double", 2048)):
        for n in range(1, lim + 1):
            if not smooth5(n):
                continue
            rad = choose(n)
            P = threads_per_column(n, rad)
            E = elems_per_thread(n, rad, P)
            lb = launch_bound(dt == "double", E)
            entries.append((dt, n, P, rad, lb))
    for dt in ("float", "double"):
        es = [e for e in entries if e[0] == dt]
        chunks = [es[i::NFILES] for i in range(NFILES)]
        for fi, ch in enumerate(chunks):
            tag = "f32" if dt == "float" else "f64"
            path = os.path.join(here, f"plans_{tag}_{fi}.cu")
            lines = ["// Generated by gen_plans.py -- do not edit.",
                     '#include "static_plans.h"', "namespace dfft {"]
            for (_, n, P, rad, lb) in ch:
                rs = ",".join(str(r) for r in rad)
                lines.append(f"template __global__ void axis_pass_static<{dt},true,{lb},{n},{P},{rs}>(const PassDesc);")
                lines.append(f"template __global__ void axis_pass_static<{dt},false,{lb},{n},{P},{rs}>(const PassDesc);")
                if has_tma(dt, n):
                    tlb = tma_bound(dt, lb)
                    for cg, cs in (("false", strided_c(dt, n, P, tlb)), ("true", 0)):
                        lines.append(f"template __global__ void axis_pass_pipe<{dt},{tlb},{cg},{cs},{n},{P},{rs}>("
                                     "const PassDesc, const __grid_constant__ CUtensorMap, "
                                     "const __grid_constant__ CUtensorMap, const TmaGeom);")
            lines.append(f"extern const StaticPlan kPlans_{tag}_{fi}[];")
            lines.append(f"extern const int kPlansCount_{tag}_{fi};")
            lines.append(f"const StaticPlan kPlans_{tag}_{fi}[] = {{")
            for (_, n, P, rad, lb) in ch:
                rs = ",".join(str(r) for r in rad)
                radarr = "{" + ",".join(str(r) for r in rad) + "}"
                tlb = tma_bound(dt, lb)
                cs = strided_c(dt, n, P, tlb)
                ps = (f"(const void*)&axis_pass_pipe<{dt},{tlb},false,{cs},{n},{P},{rs}>" if has_tma(dt, n)
                      else "nullptr")
                pc = (f"(const void*)&axis_pass_pipe<{dt},{tlb},true,0,{n},{P},{rs}>" if has_tma(dt, n)
                      else "nullptr")
                lines.append(
                    f"  {{{n}, {P}, {len(rad)}, {radarr}, {lb}, "
                    f"(const void*)&axis_pass_static<{dt},true,{lb},{n},{P},{rs}>, "
                    f"(const void*)&axis_pass_static<{dt},false,{lb},{n},{P},{rs}>, {ps}, {pc}, {tlb}, "
                    f"{cs if has_tma(dt, n) else 0}}},")
            lines.append("};")
            lines.append(f"const int kPlansCount_{tag}_{fi} = {len(ch)};")
            lines.append("}  // namespace dfft")
            new = "\n".join(lines) + "\n"
            old = open(path).read() if os.path.exists(path) else None
            if new != old:
                with open(path, "w") as f:
                    f.write(new)
    # table of tables
    lines = ["// Generated by gen_plans.py -- do not edit.", '#include "static_plans.h"',
             "namespace dfft {"]
    for tag in ("f32", "f64"):
        for fi in range(NFILES):
            lines.append(f"extern const StaticPlan kPlans_{tag}_{fi}[]; extern const int kPlansCount_{tag}_{fi};")
    for tag in ("f32", "f64"):
        lines.append(f"const StaticPlanTable kTable_{tag}[] = {{")
        for fi in range(NFILES):
            lines.append(f"  {{kPlans_{tag}_{fi}, &kPlansCount_{tag}_{fi}}},")
        lines.append("};")
    lines.append(f"const int kTableParts = {NFILES};")
    lines.append("}  // namespace dfft")
    path = os.path.join(here, "plans_table.cu")
    new = "\n".join(lines) + "\n"
    old = open(path).read() if os.path.exists(path) else None
    if new != old:
        with open(path, "w") as f:
            f.write(new)


if __name__ == "__main__":
    main()
