"""The tensor-core predict's FP32 phasor: polynomial accuracy and the quadrant
mapping (a numpy emulation of csrc/common.cuh phasor_quarter_f32, FP64
reduction then FP32 polynomials), no GPU."""

import re
from pathlib import Path

import numpy as np

from mwa_hyperdrive_b200 import phasor_poly

SRC = Path(__file__).resolve().parents[1] / "mwa_hyperdrive_b200" / "csrc" / "common.cuh"


def kernel_constants():
    text = SRC.read_text()
    vals = {name: np.float32(float(v)) for name, v in re.findall(r"(P[SC]\d) = ([-+0-9.e]+)f", text)}
    s = [vals[f"PS{i}"] for i in range(phasor_poly.SIN_TERMS)]
    c = [vals[f"PC{i}"] for i in range(phasor_poly.COS_TERMS)]
    return np.array(s, np.float32), np.array(c, np.float32)


def test_kernel_holds_the_fitted_constants():
    s, c = phasor_poly.fit()
    ks, kc = kernel_constants()
    np.testing.assert_array_equal(ks, s)
    np.testing.assert_array_equal(kc, c)


def test_polynomials_within_one_ulp():
    s, c = kernel_constants()
    es, ec = phasor_poly.max_error_f32(s, c)
    assert es < 1.0 and ec < 1.0, (es, ec)


def emulate(z):
    """sin, cos of 2 pi z for z in quarter-turns (float64 input)."""
    z = np.asarray(z, np.float64)
    q = np.rint(z).astype(np.int64)
    r = (z - q).astype(np.float32)
    s, c = kernel_constants()
    ps, pc = phasor_poly.evaluate_f32(r, s, c)
    odd = (q & 1).astype(bool)
    a = np.where(odd, pc, ps)
    b = np.where(odd, ps, pc)
    sn = np.where(q & 2, -a, a)
    cs = np.where((q + 1) & 2, -b, b)
    return sn, cs


def test_quadrant_mapping_and_large_phases():
    rng = np.random.default_rng(0)
    z = np.concatenate([rng.uniform(-4.0, 4.0, 200_000), rng.uniform(-2e4, 2e4, 200_000),
                        np.arange(-8, 9) * 0.5])
    sn, cs = emulate(z)
    ang = 0.5 * np.pi * z
    # reference with the exact reduction, so only the polynomial error remains
    zr = z - 4.0 * np.round(z / 4.0)
    ref_s, ref_c = np.sin(0.5 * np.pi * zr), np.cos(0.5 * np.pi * zr)
    assert np.max(np.abs(sn - ref_s)) < 1.5 * 2.0 ** -23
    assert np.max(np.abs(cs - ref_c)) < 1.5 * 2.0 ** -23
    # and against the unreduced angle for small |z|
    small = np.abs(z) < 4
    assert np.max(np.abs(sn[small] - np.sin(ang[small]))) < 2e-7
