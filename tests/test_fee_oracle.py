"""The FEE beam oracle (oracle/fee_ref.py) on the CPU: its Legendre terms
against scipy's lpmv and finite differences, its zenith limits, and the
model's own identities (linearity in the dipole gains, the delay phase, dead
dipoles, zenith normalisation, the parallactic rotation).  Parity with
mwa_hyperbeam itself is unpinned: neither it nor the beam file is in this
image."""

import math

import numpy as np
import pytest
from scipy.special import lpmv

from mwa_hyperdrive_b200 import synth
from oracle import fee_ref as fr

FILE = synth.fee_coeffs([167680000, 168960000, 170240000], [7, 9, 8], seed=3)
F0 = int(FILE["freqs_hz"][0])


@pytest.mark.parametrize("n", range(1, 10))
def test_assoc_legendre_matches_lpmv(n):
    th = np.linspace(0.05, math.pi - 0.05, 23)
    for m in range(0, n + 1):
        got = fr.assoc_legendre(n, m, th)
        ref = lpmv(m, n, np.cos(th))
        assert np.allclose(got, ref, rtol=1e-12, atol=1e-12 * max(1.0, np.max(np.abs(ref))))


def test_derivative_identity_against_finite_differences():
    th = np.array([0.1, 0.6, 1.1, 1.5, 2.4])
    h = 1e-6
    for n in range(1, 12):
        for m in range(0, n + 1):
            _, p1 = fr.legendre_terms(n, m, th)
            fd = (lpmv(m, n, np.cos(th + h)) - lpmv(m, n, np.cos(th - h))) / (2 * h)
            assert np.max(np.abs(p1 - fd)) <= 1e-7 * max(1.0, np.max(np.abs(fd))), (n, m)


def test_zenith_limits_are_continuous():
    for n in range(1, 10):
        for m in range(1, n + 1):
            p0, d0 = fr.legendre_terms(n, m, np.array([0.0]))
            p1, d1 = fr.legendre_terms(n, m, np.array([1e-10]))
            assert abs(p0[0] - p1[0]) <= 1e-5 * max(1.0, abs(p0[0]))
            assert abs(d0[0] - d1[0]) <= 1e-5 * max(1.0, abs(d0[0]))
        assert fr.legendre_terms(n, 1, np.array([0.0]))[0][0] == pytest.approx(-n * (n + 1) / 2, rel=1e-13)


def test_linear_in_the_dipole_gains():
    rng = np.random.default_rng(1)
    az, za = rng.uniform(0, 2 * math.pi, 9), rng.uniform(0, 1.5, 9)
    delays = rng.integers(0, 32, 16)
    amps = rng.uniform(0.5, 1.0, 32)
    full = fr.calc_jones(FILE, az, za, F0, delays, amps, norm_to_zenith=False)
    parts = 0
    for d in range(16):
        a = np.zeros(32)
        a[d], a[16 + d] = amps[d], amps[16 + d]
        parts = parts + fr.calc_jones(FILE, az, za, F0, delays, a, norm_to_zenith=False)
    assert np.max(np.abs(full - parts)) <= 1e-12 * np.max(np.abs(full))


def test_common_delay_is_a_phase():
    az, za = np.array([0.3, 2.0, 4.1]), np.array([0.2, 0.7, 1.3])
    base = fr.calc_jones(FILE, az, za, F0, np.zeros(16, int), np.ones(32), norm_to_zenith=True)
    d = fr.calc_jones(FILE, az, za, F0, np.full(16, 5), np.ones(32), norm_to_zenith=True)
    ph = np.exp(-2j * math.pi * F0 * 5 * fr.DELAY_STEP)
    assert np.allclose(d, base * ph, rtol=0, atol=1e-12 * np.max(np.abs(base)))


def test_dead_dipole_is_zero_gain():
    az, za = np.array([0.3, 2.0]), np.array([0.2, 1.1])
    delays = np.arange(16) % 7
    dead = delays.copy()
    dead[4] = fr.DEAD
    amps = np.ones(32)
    zero = amps.copy()
    zero[4] = zero[20] = 0.0
    delays4 = delays.copy()
    delays4[4] = 0
    a = fr.calc_jones(FILE, az, za, F0, dead, amps)
    b = fr.calc_jones(FILE, az, za, F0, delays4, zero)
    assert np.array_equal(a, b)


def test_zenith_normalisation():
    # the zenith-pointed beam at the zenith, at each element's peak azimuth,
    # has unit magnitude after normalisation (phi = pi/2 - az)
    for k in range(3):
        f = int(FILE["freqs_hz"][k])
        z = np.zeros(16, int)
        one = np.ones(32)
        for el, az in ((0, math.pi / 2), (1, math.pi), (2, 0.0), (3, math.pi / 2)):
            j = fr.calc_jones(FILE, az, 0.0, f, z, one, norm_to_zenith=True)[0]
            assert abs(abs(j[el]) - 1.0) < 1e-13


def test_parallactic_rotation_keeps_row_norms():
    rng = np.random.default_rng(4)
    az, za = rng.uniform(0, 2 * math.pi, 12), rng.uniform(0, 1.5, 12)
    j = fr.calc_jones(FILE, az, za, F0, np.zeros(16, int), np.ones(32))
    r = fr.calc_jones(FILE, az, za, F0, np.zeros(16, int), np.ones(32), latitude=synth.MWA_LAT_RAD)
    for a, b in ((0, 1), (2, 3)):
        assert np.allclose(np.abs(j[:, a]) ** 2 + np.abs(j[:, b]) ** 2, np.abs(r[:, a]) ** 2 + np.abs(r[:, b]) ** 2,
                           rtol=1e-12)
    assert not np.allclose(j, r)


def test_closest_frequency():
    ff = FILE["freqs_hz"]
    assert fr.closest_freq_index(ff, ff[1] + 100) == 1
    assert fr.closest_freq_index(ff, 1) == 0
    assert fr.closest_freq_index(ff, 10 ** 9) == 2
    mid = (int(ff[0]) + int(ff[1])) // 2  # an exact tie takes the first
    assert fr.closest_freq_index(ff, mid) == 0


def test_synthetic_file_layout():
    nm = FILE["num_freq_modes"]
    assert list(nm) == [2 * 7 * 9, 2 * 9 * 11, 2 * 8 * 10]
    modes = FILE["modes"]
    for k, n_k in enumerate((7, 9, 8)):
        cols = modes[:, :nm[k]]
        assert cols[2].max() == n_k
        assert {(int(s), int(m), int(n)) for s, m, n in cols.T} == \
            {(s, m, n) for n in range(1, n_k + 1) for s in (1, 2) for m in range(-n, n + 1)}
