"""Writes the golden vectors in this directory (run: python make_golden.py).

The reference (Julia + FFTW) cannot run in this environment and ships no
golden data, so the fixtures pin the oracle to closed-form answers of the
transform definitions it restates (FFTW/AbstractFFTs conventions):

  impulse.npz   x = e_j          -> X_k = exp(-2 pi i j k / n)
  tone.npz      x = exp(2 pi i k0 n / N) -> X = N e_{k0}
  cosine.npz    REDFT10 of cos(pi m (n+1/2)/N) -> N (m>0) / 2N (m=0) at k=m
  seeded.npz    small seeded inputs with long-double direct-sum outputs for
                fft/ifft (3-D), rfft/irfft (3-D) and each r2r kind (1-D)
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "oracle"))
import dfft_oracle as o  # noqa: E402

PI = o.PI_LD


def main():
    # impulse at j=3, n=12
    n, j = 12, 3
    x = np.zeros(n, np.complex128)
    x[j] = 1
    k = np.arange(n, dtype=np.longdouble)
    X = np.cos(-2 * PI * j * k / n) + 1j * np.sin(-2 * PI * j * k / n)
    np.savez(os.path.join(HERE, "impulse.npz"), x=x, X=X.astype(np.complex128))
    # tone k0=5, N=40
    N, k0 = 40, 5
    m = np.arange(N, dtype=np.longdouble)
    t = np.cos(2 * PI * k0 * m / N) + 1j * np.sin(2 * PI * k0 * m / N)
    T = np.zeros(N, np.complex128)
    T[k0] = N
    np.savez(os.path.join(HERE, "tone.npz"), x=t.astype(np.complex128), X=T)
    # cosine for REDFT10
    N, mm = 16, 4
    c = np.cos(PI * mm * (np.arange(N, dtype=np.longdouble) + 0.5) / N)
    Y = np.zeros(N)
    Y[mm] = N
    np.savez(os.path.join(HERE, "cosine.npz"), x=c.astype(np.float64), Y=Y)
    # seeded small cases, long-double direct sums
    rng = np.random.default_rng(20260101)
    a = (rng.random((6, 5, 4)) + 1j * rng.random((6, 5, 4)))
    F = o.dft_direct(o.dft_direct(o.dft_direct(a, 0), 1), 2)
    r = rng.random((8, 6, 5))
    R = o.dft_direct(o.dft_direct(r.astype(np.clongdouble), 1), 2)
    R = o.dft_direct(R, 0)[: 8 // 2 + 1]
    out = {"c2c_in": a, "c2c_out": F.astype(np.complex128),
           "r2c_in": r, "r2c_out": R.astype(np.complex128)}
    v = rng.standard_normal(10)
    for kind in o.R2R_SUPPORTED_KINDS:
        out[f"r2r_in_{kind}"] = v
        out[f"r2r_out_{kind}"] = o.r2r_direct(v, kind, 0).astype(np.float64)
    np.savez(os.path.join(HERE, "seeded.npz"), **out)


if __name__ == "__main__":
    main()
