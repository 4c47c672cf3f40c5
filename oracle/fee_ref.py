"""ORACLE (test infrastructure only): CPU restatement of the MWA FEE beam.
Only tests/ and bench.py's CPU leg import this module; the product never
does.

The reference takes its FEE Jones matrices from mwa_hyperbeam 0.11.0
(Cargo.lock:1590-1593), a crates.io dependency that is not part of the
reference tree.  Its call sites fix what is asked of it:
beam/fee.rs:98-118 (calc_jones_pair with norm_to_zenith = true, a latitude
for the parallactic rotation and iau_order = false) and beam/fee.rs:307-349
(gpu_prepare with each tile's delays and 32 dipole gains, then
calc_jones_device_pair_inner into [uniq tile][uniq freq][direction]).  This
module restates the published model, Sokolowski et al. 2017 (PASA 34,
e062), term by term and in the file's own mode order:

  Q1_mn, Q2_mn = sum_d g_d exp(-2 pi i f tau_d) Q_d(s = 1, 2; m, n)
      (f the file frequency closest to the channel, tau_d = delay_d x 435 ps,
       a dipole with delay 32 is dead: g_d = 0 and tau_d = 0)
  phi_comp = C_mn (-m/|m|)^m e^{i m phi} / sqrt(n (n + 1)),
  C_mn = sqrt((2n + 1)/2 (n - |m|)!/(n + |m|)!), (-m/|m|)^m = 1 for m <= 0
  E_theta = j^n (P1sin (|m| Q2 u - m Q1) + Q2 P1)
  E_phi = j^(n+1) (P1sin (m Q2 - |m| Q1 u) - Q1 P1)
  sigma_T = sum phi_comp E_theta, sigma_P = sum phi_comp E_phi
  Jones row of a polarisation = (sigma_T, -sigma_P), X row then Y row

with u = cos theta, theta = za, phi = pi/2 - az, P1sin = P_n^|m|(u)/sin theta
and P1 = dP_n^|m|(cos theta)/d theta, P_n^m the associated Legendre function
with the Condon-Shortley phase, here (-1)^m sin^m theta d^m P_n/du^m from
numpy's Legendre series (checked against scipy.special.lpmv by the tests),
so that P1sin stays exact at the zenith (-n(n+1)/2 for |m| = 1, 0 otherwise).  norm_to_zenith divides
each element by |that element| of the zenith-pointed beam (delays 0, gains 1)
at the zenith, at phi = 0, -pi/2, pi/2, 0.  The parallactic rotation uses
ERFA's ae2hd and hd2pa (marlu's AzEl::to_hadec and
HADec::get_parallactic_angle) and the angle + pi/2.

Parity unpinned: neither hyperbeam nor the FEE coefficient file
(mwa_full_embedded_element_pattern.h5) is in this image, and the reference's
FEE tests compare against hyperbeam's live output, not stored numbers.  The
file's coefficients are replaced by seeded synthetic ones
(mwa_hyperdrive_b200.synth.fee_coeffs) with the file's layout.
"""

from __future__ import annotations

import math

import numpy as np

DELAY_STEP = 435e-12
DEAD = 32


def closest_freq_index(file_freqs, freq_hz) -> int:
    """Index of the file frequency closest to freq_hz (the first on a tie)."""
    d = np.abs(np.asarray(file_freqs, np.int64) - int(freq_hz))
    return int(np.argmin(d))


def effective(delays, amps):
    """Per-dipole delays [16] and gains [32] with dead dipoles (delay 32)
    zeroed; 16 gains serve both polarisations."""
    delays = np.asarray(delays, np.int64).copy()
    amps = np.asarray(amps, np.float64)
    if amps.size == 16:
        amps = np.concatenate([amps, amps])
    amps = amps.copy()
    dead = delays == DEAD
    amps[:16][dead] = 0.0
    amps[16:][dead] = 0.0
    delays[dead] = 0
    return delays, amps


def beamformed(file, k, delays, amps):
    """{pol: {(m, n): [Q1, Q2]}} at file frequency index k, in the file's mode
    order."""
    delays, amps = effective(delays, amps)
    f = float(file["freqs_hz"][k])
    nm = int(file["num_freq_modes"][k])
    modes = file["modes"]
    q = file["q"][k]  # [2][16][num_modes][2]
    out = {}
    for p in range(2):
        w = amps[16 * p:16 * p + 16] * np.exp(-2j * math.pi * f * delays * DELAY_STEP)
        qc = q[p, :, :nm, 0] + 1j * q[p, :, :nm, 1]  # [16][nm]
        acc = w @ qc
        d = {}
        for c in range(nm):
            s, m, n = int(modes[0][c]), int(modes[1][c]), int(modes[2][c])
            d.setdefault((m, n), [0j, 0j])[s - 1] += acc[c]
        out[p] = d
    return out


def _dleg(n, k, u):
    """d^k P_n(u) / du^k (Legendre polynomial derivative, numpy's Legendre
    series; 0 for k > n)."""
    if k > n:
        return np.zeros_like(u)
    c = np.zeros(n + 1)
    c[n] = 1.0
    return np.polynomial.legendre.legval(u, np.polynomial.legendre.legder(c, k)) if k else \
        np.polynomial.legendre.legval(u, c)


def assoc_legendre(n, ma, theta):
    """P_n^ma(cos theta) = (-1)^ma sin^ma theta d^ma P_n/du^ma (the
    Condon-Shortley phase, as scipy.special.lpmv; written in theta so that it
    keeps its accuracy next to the poles, where cos theta rounds to 1)."""
    theta = np.asarray(theta, np.float64)
    return (-1.0) ** ma * np.sin(theta) ** ma * _dleg(n, ma, np.cos(theta))


def legendre_terms(n, ma, theta):
    """P1sin = P_n^ma(cos theta)/sin theta and P1 = dP_n^ma(cos theta)/d theta
    (arrays over theta).  P1sin = (-1)^ma sin^(ma-1) theta d^ma P_n/du^ma,
    finite at the poles (ma >= 1; 0 for ma = 0, where it is always multiplied
    by m = 0).  P1 uses dP_n^m/d theta = (P_n^{m+1} - (n+m)(n-m+1) P_n^{m-1}) / 2
    (m >= 1) and P_n^1 (m = 0); the tests check it against finite differences
    of scipy's lpmv."""
    theta = np.asarray(theta, np.float64)
    u, s = np.cos(theta), np.sin(theta)
    if ma == 0:
        return np.zeros_like(theta), assoc_legendre(n, 1, theta)
    p1sin = (-1.0) ** ma * s ** (ma - 1) * _dleg(n, ma, u)
    p1 = 0.5 * (assoc_legendre(n, ma + 1, theta) - (n + ma) * (n - ma + 1) * assoc_legendre(n, ma - 1, theta))
    return p1sin, p1


def sigmas(phi, theta, coeffs):
    """(sigma_T, -sigma_P) of one polarisation's {(m, n): [Q1, Q2]}."""
    phi = np.asarray(phi, np.float64)
    theta = np.asarray(theta, np.float64)
    u = np.cos(theta)
    st = np.zeros(np.broadcast(phi, theta).shape, np.complex128)
    sp = np.zeros_like(st)
    for (m, n), (q1, q2) in coeffs.items():
        ma = abs(m)
        c_mn = math.sqrt(0.5 * (2 * n + 1) * math.factorial(n - ma) / math.factorial(n + ma))
        sgn = (-1.0) ** m if m > 0 else 1.0
        phi_comp = c_mn * sgn * np.exp(1j * m * phi) / math.sqrt(n * (n + 1))
        p1sin, p1 = legendre_terms(n, ma, theta)
        jn = 1j ** n
        e_t = jn * (p1sin * (ma * q2 * u - m * q1) + q2 * p1)
        e_p = jn * 1j * (p1sin * (m * q2 - ma * q1 * u) - q1 * p1)
        st = st + phi_comp * e_t
        sp = sp + phi_comp * e_p
    return st, -sp


def zenith_norm(file, k):
    """|element| of the zenith-pointed beam at the zenith, per element."""
    ideal = beamformed(file, k, np.zeros(16, np.int64), np.ones(32))
    j00 = sigmas(0.0, 0.0, ideal[0])[0]
    j01 = sigmas(-math.pi / 2, 0.0, ideal[0])[1]
    j10 = sigmas(math.pi / 2, 0.0, ideal[1])[0]
    j11 = sigmas(0.0, 0.0, ideal[1])[1]
    return np.abs(np.array([j00, j01, j10, j11], np.complex128))


def parallactic_rotate(j, az, za, lat):
    """Rotate Jones [..., 4] complex by the parallactic angle + pi/2."""
    el = math.pi / 2 - np.asarray(za)
    sa, ca = np.sin(az), np.cos(az)
    se, ce = np.sin(el), np.cos(el)
    sp, cp = math.sin(lat), math.cos(lat)
    x = -ca * ce * sp + se * cp
    y = -sa * ce
    z = ca * ce * cp + se * sp
    r = np.sqrt(x * x + y * y)
    ha = np.where(r != 0.0, np.arctan2(y, x), 0.0)
    dec = np.arctan2(z, r)
    sqsz = cp * np.sin(ha)
    cqsz = sp * np.cos(dec) - cp * np.sin(dec) * np.cos(ha)
    pa = np.where((sqsz != 0.0) | (cqsz != 0.0), np.arctan2(sqsz, cqsz), 0.0)
    s, c = np.sin(pa + math.pi / 2), np.cos(pa + math.pi / 2)
    return np.stack([j[..., 0] * c - j[..., 1] * s, j[..., 0] * s + j[..., 1] * c,
                     j[..., 2] * c - j[..., 3] * s, j[..., 2] * s + j[..., 3] * c], -1)


def calc_jones(file, az, za, freq_hz, delays, amps, norm_to_zenith=True, latitude=None):
    """Jones [n][4] complex (XX XY YX YY) of one tile at one channel for
    directions (az, za) [rad]."""
    az = np.atleast_1d(np.asarray(az, np.float64))
    za = np.atleast_1d(np.asarray(za, np.float64))
    k = closest_freq_index(file["freqs_hz"], freq_hz)
    q = beamformed(file, k, delays, amps)
    phi = math.pi / 2 - az
    j00, j01 = sigmas(phi, za, q[0])
    j10, j11 = sigmas(phi, za, q[1])
    j = np.stack([j00, j01, j10, j11], -1)
    if norm_to_zenith:
        j = j / zenith_norm(file, k)
    if latitude is not None:
        j = parallactic_rotate(j, az, za, latitude)
    return j


def as_jones8(j):
    """[..., 4] complex -> [..., 8] reals (the JonesF64 layout)."""
    out = np.empty(j.shape[:-1] + (8,))
    out[..., 0::2] = j.real
    out[..., 1::2] = j.imag
    return out
