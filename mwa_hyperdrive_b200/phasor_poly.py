"""Coefficients of the single-precision phasor polynomials used by the
tensor-core point predict and the chosen form's direct kernels
(csrc/common.cuh, `phasor_quarter_f32`).

The phase enters as r in quarter-turns, |r| <= 1/2 after the quadrant is
split off in FP64, so the polynomials approximate

    sin(pi/2 r) = r   * (s0 + s1 r^2 + s2 r^4 + s3 r^6)
    cos(pi/2 r) = c0 + c1 r^2 + c2 r^4 + c3 r^6 + c4 r^8

on [-1/2, 1/2].  Method: weighted least squares in float64 on Chebyshev
nodes of r^2 (relative error weighting for sin), then rounding to float32;
`max_error_f32` evaluates the rounded polynomials in float32 with Horner's
rule (fused multiply-adds emulated in float64 then rounded, as the GPU's FMA
does) against float64 numpy and reports the error in float32 ulps of 1.

Run `python -m mwa_hyperdrive_b200.phasor_poly` to print the constants that
csrc/common.cuh holds.
"""

from __future__ import annotations

import numpy as np

SIN_TERMS = 4
COS_TERMS = 5


def fit():
    k = np.arange(4000)
    # Chebyshev nodes on r^2 in [0, 1/4]
    x2 = 0.125 * (1.0 - np.cos(np.pi * (k + 0.5) / k.size))
    r = np.sqrt(x2)
    # sin(pi/2 r) / r as a polynomial in r^2 (relative error of sin)
    ts = np.where(r > 0, np.sin(0.5 * np.pi * r) / np.where(r > 0, r, 1.0), 0.5 * np.pi)
    A = np.vander(x2, SIN_TERMS, increasing=True)
    s = np.linalg.lstsq(A, ts, rcond=None)[0]
    A = np.vander(x2, COS_TERMS, increasing=True)
    c = np.linalg.lstsq(A, np.cos(0.5 * np.pi * r), rcond=None)[0]
    return s.astype(np.float32), c.astype(np.float32)


def _fma32(a, b, c):
    return (a.astype(np.float64) * b.astype(np.float64) + c.astype(np.float64)).astype(np.float32)


def evaluate_f32(r, s, c):
    """sin(pi/2 r), cos(pi/2 r) as the kernel evaluates them (float32)."""
    r = np.asarray(r, np.float32)
    r2 = (r * r).astype(np.float32)
    ps = np.full_like(r2, s[-1])
    for coef in s[-2::-1]:
        ps = _fma32(ps, r2, np.float32(coef))
    pc = np.full_like(r2, c[-1])
    for coef in c[-2::-1]:
        pc = _fma32(pc, r2, np.float32(coef))
    return (ps * r).astype(np.float32), pc


def max_error_f32(s, c, n=2_000_001):
    r = np.linspace(-0.5, 0.5, n).astype(np.float32)
    sv, cv = evaluate_f32(r, s, c)
    rd = r.astype(np.float64)
    es = np.abs(sv.astype(np.float64) - np.sin(0.5 * np.pi * rd))
    ec = np.abs(cv.astype(np.float64) - np.cos(0.5 * np.pi * rd))
    ulp = 2.0 ** -23
    return float(es.max() / ulp), float(ec.max() / ulp)


if __name__ == "__main__":
    s, c = fit()
    print("sin:", ", ".join(f"{float(x):.9e}f" for x in s))
    print("cos:", ", ".join(f"{float(x):.9e}f" for x in c))
    print("max error (float32 ulps of 1): sin %.2f, cos %.2f" % max_error_f32(s, c))
