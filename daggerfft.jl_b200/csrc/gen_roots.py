"""Writes roots.cuh: cos/sin(2*pi*e/R) literals for the in-register DFT codelets.

Run from this directory: ``python gen_roots.py > roots.cuh``.  The values are
mathematical constants evaluated with mpmath at 40 digits and rounded to
double by the C++ compiler."""
import mpmath as mp

mp.mp.dps = 40
RS = [3, 5, 6, 7, 8, 10, 11, 12, 13, 15, 16, 32]

print("// Generated by gen_roots.py -- do not edit.")
print("#pragma once")
print("// root_cos<R>(e) = cos(2*pi*e/R), root_sin<R>(e) = sin(2*pi*e/R), 0 <= e < R")
print("template <int R> __device__ __forceinline__ constexpr double root_cos(int e);")
print("template <int R> __device__ __forceinline__ constexpr double root_sin(int e);")
for R in RS:
    for fn, f in (("root_cos", mp.cos), ("root_sin", mp.sin)):
        print(f"template <> __device__ __forceinline__ constexpr double {fn}<{R}>(int e) {{")
        print("  switch (e) {")
        for e in range(R):
            v = f(2 * mp.pi * e / R)
            s = mp.nstr(v, 36, min_fixed=-100, max_fixed=100)
            if abs(v) < mp.mpf(10) ** -35:
                s = "0.0"
            print(f"    case {e}: return {s};")
        print("    default: return 0.0;")
        print("  }")
        print("}")
