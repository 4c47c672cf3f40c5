"""The oracle's restatements of vis_average (averaging/mod.rs:537-648) and
CalVis::scale_by_weights (params/di_calibration.rs:578-625) pinned against
the reference's own known answers (averaging/tests.rs:408-820).  No GPU."""

import numpy as np
import pytest

IDENT = np.array([1, 0, 0, 0, 0, 0, 1, 0], np.float32)


def ramp(nt, nf):
    """The reference tests' input: identity x 1, 2, ... in (t, f) order, one
    baseline."""
    return (np.arange(1, nt * nf + 1, dtype=np.float32).reshape(nt, nf, 1, 1) * IDENT).astype(np.float32)


def check(to, wto, f, value, weight):
    np.testing.assert_allclose(to[f, 0], IDENT * value, rtol=1e-6, atol=1e-6)
    assert wto[f, 0] == pytest.approx(weight)


def test_average_1d_time(oracle):
    v = ramp(1, 4)
    to, wto = oracle.vis_average(v, np.ones((1, 4, 1), np.float32), 4)
    np.testing.assert_array_equal(to, v[0])
    np.testing.assert_array_equal(wto, np.ones((4, 1)))


def test_average_uniform_and_negative_weights(oracle):
    v = ramp(2, 4)
    w = np.ones((2, 4, 1), np.float32)
    to, wto = oracle.vis_average(v, w, 4)
    for i in range(4):
        check(to, wto, i, (2 * i + 6) / 2, 2.0)
    w[:, 0] = -1.0
    to, wto = oracle.vis_average(v, w, 4)
    check(to, wto, 0, 3.0, -2.0)
    w[:] = 1.0
    w[0, 0, 0] = -1.0
    to, wto = oracle.vis_average(v, w, 4)
    check(to, wto, 0, 5.0, 1.0)
    check(to, wto, 1, 4.0, 2.0)
    w[:] = 1.0
    to, wto = oracle.vis_average(v, w, 2)
    check(to, wto, 0, 14.0 / 4, 4.0)
    check(to, wto, 1, 22.0 / 4, 4.0)


def test_average_non_uniform_weights(oracle):
    v = ramp(2, 4)
    w = np.array([[[2.0], [3.0], [5.0], [7.0]], [[11.0], [13.0], [17.0], [19.0]]], np.float32)
    to, wto = oracle.vis_average(v, w, 4)
    for f, (num, den) in enumerate([(57, 13), (84, 16), (134, 22), (180, 26)]):
        check(to, wto, f, num / den, den)
    w[0, 0, 0] *= -1
    w[1, 0, 0] *= -1
    to, wto = oracle.vis_average(v, w, 4)
    check(to, wto, 0, 3.0, -13.0)
    w[1, 0, 0] *= -1
    to, wto = oracle.vis_average(v, w, 4)
    check(to, wto, 0, 5.0, 11.0)
    w[0, 0, 0] *= -1
    to, wto = oracle.vis_average(v, w, 2)
    check(to, wto, 0, 141.0 / 29, 29.0)
    check(to, wto, 1, 314.0 / 48, 48.0)


def test_average_non_integral_shapes(oracle):
    v = ramp(2, 3)
    w = np.array([[[2.0], [3.0], [5.0]], [[7.0], [11.0], [13.0]]], np.float32)
    to, wto = oracle.vis_average(v, w, 2)
    check(to, wto, 0, 91.0 / 23, 23.0)
    check(to, wto, 1, 93.0 / 18, 18.0)
    w[:, 0] *= -1
    to, wto = oracle.vis_average(v, w, 2)
    check(to, wto, 0, 61.0 / 14, 14.0)
    check(to, wto, 1, 93.0 / 18, 18.0)


def test_average_half_flagged(oracle):
    v = ramp(2, 4)
    w = np.array([[[1.0], [1.0], [0.0], [0.0]], [[1.0], [1.0], [0.0], [0.0]]], np.float32)
    to, wto = oracle.vis_average(v, w, 2)
    check(to, wto, 0, 14.0 / 4, 4.0)
    check(to, wto, 1, 22.0 / 4, 0.0)


def test_average_skips_flagged_chanblocks(oracle):
    """input_vis.rs:266-272 passes the flagged chanblock indices: their
    channel chunks are skipped and the outputs hold the others in order."""
    v = ramp(2, 6)
    w = np.ones((2, 6, 1), np.float32)
    to, wto = oracle.vis_average(v, w, 2, flagged=[1])
    check(to, wto, 0, (1 + 2 + 7 + 8) / 4, 4.0)
    check(to, wto, 1, (5 + 6 + 11 + 12) / 4, 4.0)


def test_scale_by_weights(oracle):
    rng = np.random.default_rng(1)
    nt, nf, nbl = 3, 5, 7
    d = rng.normal(size=(nt, nf, nbl, 8)).astype(np.float32)
    m = rng.normal(size=(nt, nf, nbl, 8)).astype(np.float32)
    w = rng.uniform(-0.5, 2.0, size=(nt, nf, nbl)).astype(np.float32)
    w[0, 0, 0] = 0.0
    bw = rng.uniform(0.0, 1.0, size=nbl)
    bw[3] = 0.0
    for b in (None, bw):
        dd, mm = oracle.scale_by_weights(d, m, w, b)
        tot = w.astype(np.float64) * (1.0 if b is None else b[None, None, :])
        exp_d = np.where(tot[..., None] > 0, (d.astype(np.float64) * tot[..., None]).astype(np.float32), 0)
        exp_m = np.where(tot[..., None] > 0, (m.astype(np.float64) * tot[..., None]).astype(np.float32), 0)
        np.testing.assert_array_equal(dd, exp_d)
        np.testing.assert_array_equal(mm, exp_m)
