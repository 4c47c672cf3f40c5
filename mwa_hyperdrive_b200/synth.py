"""Seeded synthetic observations with the shapes of the benchmark
configurations (the reference publishes no dataset for this path).

Arrays: tiles uniform in a disk in the local east/north plane, converted to
geodetic XYZ at the MWA latitude.  Sky models: components uniform in a
spherical cap around the phase centre.
"""

from __future__ import annotations

import math
from dataclasses import dataclass
from typing import List, Optional

import numpy as np

from . import srclist as sl

MWA_LAT_RAD = -0.4660608448386394
SIDEREAL_RATE = 7.292115855306589e-5  # rad / s
VEL_C = 299792458.0


def enu_to_xyz(e, n, u, lat=MWA_LAT_RAD):
    """Local east/north/up [m] -> geodetic XYZ [m] (X in the meridian plane)."""
    sl_, cl = math.sin(lat), math.cos(lat)
    x = -sl_ * n + cl * u
    y = e
    z = cl * n + sl_ * u
    return np.stack([x, y, z], axis=-1)


def tiles_in_disk(num_tiles: int, radius_m: float, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    r = radius_m * np.sqrt(rng.random(num_tiles))
    th = rng.random(num_tiles) * 2 * math.pi
    return enu_to_xyz(r * np.cos(th), r * np.sin(th), np.zeros(num_tiles))


def cap_positions(n: int, centre, radius_rad: float, rng) -> np.ndarray:
    """Uniform positions (ra, dec) within a cap of angular radius around centre."""
    cosr = math.cos(radius_rad)
    z = 1.0 - rng.random(n) * (1.0 - cosr)  # cos of offset angle
    rho = np.arccos(z)
    phi = rng.random(n) * 2 * math.pi
    # offset direction in the tangent frame of the centre
    ra0, dec0 = centre
    sd, cd = math.sin(dec0), math.cos(dec0)
    sr, cr = np.sin(rho), np.cos(rho)
    dec = np.arcsin(sd * cr + cd * sr * np.cos(phi))
    ra = ra0 + np.arctan2(np.sin(phi) * sr * cd, cr - sd * np.sin(dec))
    return np.stack([ra, dec], axis=-1)


@dataclass
class Obs:
    tile_xyzs: np.ndarray
    freqs: np.ndarray
    phase_centre: tuple
    lsts: np.ndarray
    latitude: float = MWA_LAT_RAD

    @property
    def num_tiles(self):
        return self.tile_xyzs.shape[0]

    @property
    def num_baselines(self):
        n = self.num_tiles
        return n * (n - 1) // 2


def point_sky(n: int, centre, radius_deg: float, seed: int, curved_q_sigma: Optional[float] = None,
              ref_freq: float = 150e6) -> List[sl.SourceComponent]:
    rng = np.random.default_rng(seed)
    pos = cap_positions(n, centre, math.radians(radius_deg), rng)
    flux_i = rng.lognormal(0.0, 1.0, n)
    si = rng.normal(-0.8, 0.2, n)
    qs = rng.normal(0.0, curved_q_sigma, n) if curved_q_sigma else None
    comps = []
    for k in range(n):
        fd = sl.FluxDensity(ref_freq, float(flux_i[k]))
        ft = sl.CurvedPowerLaw(float(si[k]), fd, float(qs[k])) if qs is not None else sl.PowerLaw(float(si[k]), fd)
        comps.append(sl.SourceComponent(float(pos[k, 0]), float(pos[k, 1]), sl.Point(), ft))
    return comps


def config1():
    """Plain point-source predict, f64: 128 tiles in a 1.5 km disk, 1
    timestep at HA 0, 32 channels of 40 kHz from 170 MHz, 200 points within
    10 deg of (0, -27 deg), lognormal(0, 1) Jy at 150 MHz, SI N(-0.8, 0.2),
    no beam."""
    pc = (0.0, math.radians(-27.0))
    obs = Obs(tiles_in_disk(128, 750.0, 1), 170.0e6 + np.arange(32) * 40e3, pc, np.array([pc[0]]))
    sky = sl.SkyModelArrays.from_components(point_sky(200, pc, 10.0, 1))
    return obs, sky


def gaussians_and_shapelets(n_g: int, n_s: int, centre, seed: int, q_sigma: float = 0.2, ncoeff: int = 20):
    rng = np.random.default_rng(seed)
    arcmin = math.radians(1.0 / 60.0)
    comps = []
    pos = cap_positions(n_g + n_s, centre, math.radians(10.0), rng)
    for k in range(n_g + n_s):
        maj = rng.uniform(0.5, 5.0) * arcmin
        mn = maj * rng.uniform(0.3, 1.0)
        pa = rng.uniform(0.0, math.pi)
        fd = sl.FluxDensity(150e6, float(rng.lognormal(0.0, 1.0)))
        ft = sl.CurvedPowerLaw(float(rng.normal(-0.8, 0.2)), fd, float(rng.normal(0.0, q_sigma)))
        if k < n_g:
            ct = sl.Gaussian(maj, mn, pa)
        else:
            coeffs = [sl.ShapeletCoeff(int(rng.integers(0, 6)), int(rng.integers(0, 6)), float(rng.normal() * 0.1))
                      for _ in range(ncoeff)]
            ct = sl.Shapelet(maj, mn, pa, coeffs)
        comps.append(sl.SourceComponent(float(pos[k, 0]), float(pos[k, 1]), ct, ft))
    return comps


def config2(n_points=4000, n_gauss=500, n_shapelets=100, n_freqs=384, n_times=4):
    """Mixed-component predict: 128 tiles, 4 timesteps 8 s apart, 384
    channels of 80 kHz from 167 MHz, 4000 points + 500 Gaussians + 100
    shapelets (20 coefficients, n1, n2 <= 5), curved power laws with q ~
    N(0, 0.2), analytic dipole-array beam shared by all tiles."""
    pc = (0.0, math.radians(-27.0))
    lsts = pc[0] + np.arange(n_times) * 8.0 * SIDEREAL_RATE
    obs = Obs(tiles_in_disk(128, 750.0, 2), 167.0e6 + np.arange(n_freqs) * 80e3, pc, lsts)
    comps = point_sky(n_points, pc, 10.0, 2, curved_q_sigma=0.2)
    comps += gaussians_and_shapelets(n_gauss, n_shapelets, pc, 22)
    return obs, sl.SkyModelArrays.from_components(comps)


def sample_tiles(ntiles: int, k: int, seed: int):
    """A seeded random subset of k of ntiles tiles (sorted) and the indices,
    in the full set's baseline order, of the k (k - 1) / 2 baselines among
    them -- in the same order as the subset's own baselines.  Every baseline
    is equally likely to be in the sample."""
    rng = np.random.default_rng(seed)
    sub = np.sort(rng.choice(ntiles, size=k, replace=False))
    i, j = np.triu_indices(k, 1)
    p, q = sub[i], sub[j]
    bl = p * (2 * ntiles - p - 1) // 2 + (q - p - 1)
    return sub, bl.astype(np.int64)


def truth_gains(ntiles: int, nch: int, rng, amp_sigma=0.1, leak_sigma=0.01, phase_slope=None, freqs=None):
    """Per (tile, chanblock) Jones gains: diagonal amplitude N(1, amp_sigma),
    phase U(-pi, pi) (or a per-tile linear phase in frequency when
    phase_slope [rad/Hz] and freqs are given), complex off-diagonal leakage
    N(0, leak_sigma).  Returns [tile][chanblock][8] float64."""
    g = np.zeros((ntiles, nch, 8))
    amp = rng.normal(1.0, amp_sigma, (ntiles, 2))
    if phase_slope is not None:
        ph0 = rng.uniform(-np.pi, np.pi, (ntiles, 2))
        slope = rng.uniform(-phase_slope, phase_slope, (ntiles, 2))
        ph = ph0[:, None, :] + slope[:, None, :] * (np.asarray(freqs)[None, :, None] - freqs[0])
    else:
        ph = np.broadcast_to(rng.uniform(-np.pi, np.pi, (ntiles, 1, 2)), (ntiles, nch, 2))
    g[..., 0] = amp[:, None, 0] * np.cos(ph[..., 0])
    g[..., 1] = amp[:, None, 0] * np.sin(ph[..., 0])
    g[..., 6] = amp[:, None, 1] * np.cos(ph[..., 1])
    g[..., 7] = amp[:, None, 1] * np.sin(ph[..., 1])
    g[..., 2:6] = rng.normal(0.0, leak_sigma, (ntiles, nch, 4))
    return g


def _jmul(a, b):
    """Batched 2x2 complex products of [...][8] arrays."""
    ac = a[..., 0::2] + 1j * a[..., 1::2]
    bc = b[..., 0::2] + 1j * b[..., 1::2]
    r = np.empty_like(ac)
    r[..., 0] = ac[..., 0] * bc[..., 0] + ac[..., 1] * bc[..., 2]
    r[..., 1] = ac[..., 0] * bc[..., 1] + ac[..., 1] * bc[..., 3]
    r[..., 2] = ac[..., 2] * bc[..., 0] + ac[..., 3] * bc[..., 2]
    r[..., 3] = ac[..., 2] * bc[..., 1] + ac[..., 3] * bc[..., 3]
    out = np.empty(a.shape[:-1] + (8,))
    out[..., 0::2] = r.real
    out[..., 1::2] = r.imag
    return out


def _jh(a):
    out = a.copy()
    out[..., 2:4], out[..., 4:6] = a[..., 4:6].copy(), a[..., 2:4].copy()
    out[..., 1::2] *= -1
    return out


def corrupt(model_tfb, gains_tc, rng=None, snr=None):
    """data = G_p M G_q^H (+ complex Gaussian noise at per-visibility SNR)."""
    nt, nch, nbl = model_tfb.shape[:3]
    ntiles = gains_tc.shape[0]
    i, j = np.triu_indices(ntiles, 1)
    gp = gains_tc[i].transpose(1, 0, 2)[None]  # [1][ch][bl][8]
    gq = gains_tc[j].transpose(1, 0, 2)[None]
    d = _jmul(_jmul(np.broadcast_to(gp, model_tfb.shape), model_tfb.astype(np.float64)),
              _jh(np.broadcast_to(gq, model_tfb.shape)))
    if snr is not None:
        rms = np.sqrt(np.mean(d[..., [0, 1, 6, 7]] ** 2))
        d = d + rng.normal(0.0, rms / snr / np.sqrt(2.0), d.shape)
    return d.astype(np.float32)


def polarised_model(nt, nch, nbl, rng, cross=0.3):
    """A random model [t][chanblock][bl][8] whose four correlations have
    independent phases, XX and YY of similar amplitude and XY, YX at
    `cross` of it (an apparent sky seen through a polarised beam).  Unlike a
    Stokes-I dominated model this pins the relative X/Y phase of the gains,
    so MitchCal converges to a unique fixed point (up to one phase per
    chanblock)."""
    m = np.zeros((nt, nch, nbl, 8))
    amp = rng.lognormal(0.0, 0.5, (nt, nch, nbl))
    for k in range(4):
        a = amp * (1.0 if k in (0, 3) else cross) * rng.lognormal(0.0, 0.2, (nt, nch, nbl))
        ph = rng.uniform(-np.pi, np.pi, (nt, nch, nbl))
        m[..., 2 * k] = a * np.cos(ph)
        m[..., 2 * k + 1] = a * np.sin(ph)
    return m.astype(np.float32)


def polarised_model_device(nt, nch, nbl, gen, cross=0.3):
    """polarised_model on the CUDA device (torch, generator ``gen``): the
    same distribution, a different random stream; float32 [t][ch][bl][8]."""
    import torch

    amp = torch.empty((nt, nch, nbl), dtype=torch.float64, device="cuda").log_normal_(0.0, 0.5, generator=gen)
    m = torch.empty((nt, nch, nbl, 8), dtype=torch.float32, device="cuda")
    for k in range(4):
        a = amp * (1.0 if k in (0, 3) else cross) * torch.empty_like(amp).log_normal_(0.0, 0.2, generator=gen)
        ph = torch.empty_like(amp).uniform_(-np.pi, np.pi, generator=gen)
        m[..., 2 * k] = (a * torch.cos(ph)).float()
        m[..., 2 * k + 1] = (a * torch.sin(ph)).float()
    return m


def corrupt_device(model_tfb, gains_tc):
    """corrupt() on the device without noise: data = G_p M G_q^H, float32."""
    import torch

    nt, nch, nbl = (int(x) for x in model_tfb.shape[:3])
    ntiles = gains_tc.shape[0]
    i, j = np.triu_indices(ntiles, 1)
    g = torch.from_numpy(np.ascontiguousarray(gains_tc, np.float64)).cuda()
    g = torch.view_as_complex(g.reshape(ntiles, nch, 4, 2)).reshape(ntiles, nch, 2, 2)
    gp = g[torch.from_numpy(i).cuda()].permute(1, 0, 2, 3)  # [ch][bl][2][2]
    gqh = g[torch.from_numpy(j).cuda()].permute(1, 0, 2, 3).conj().transpose(-1, -2)
    out = torch.empty_like(model_tfb)
    for t in range(nt):
        m = torch.view_as_complex(model_tfb[t].double().reshape(nch, nbl, 4, 2)).reshape(nch, nbl, 2, 2)
        d = gp @ m @ gqh
        out[t] = torch.view_as_real(d.reshape(nch, nbl, 4)).reshape(nch, nbl, 8).float()
    return out


def random_model(nt, nch, nbl, rng):
    """A random, Stokes-I dominated model [t][chanblock][bl][8]."""
    m = np.zeros((nt, nch, nbl, 8))
    amp = rng.lognormal(0.0, 0.5, (nt, nch, nbl))
    ph = rng.uniform(-np.pi, np.pi, (nt, nch, nbl))
    m[..., 0] = amp * np.cos(ph)
    m[..., 1] = amp * np.sin(ph)
    m[..., 6] = m[..., 0] * 0.95
    m[..., 7] = m[..., 1] * 0.95
    m[..., 2:6] = rng.normal(0.0, 0.02, (nt, nch, nbl, 4)) * amp[..., None]
    return m.astype(np.float32)


def fee_coeffs(freqs_hz, nmax, seed: int = 11) -> dict:
    """Seeded stand-in for the MWA FEE beam file (the file is not in this
    image), in the layout HdcFeeCoeffs takes: ``freqs_hz`` [nf] (uint32),
    ``modes`` [3][M] (s, m, n; sorted by n, then s, then m, so that the first
    2 n_k (n_k + 2) columns hold every mode up to degree n_k), ``num_freq_modes``
    [nf] and ``q`` [nf][2 pols][16 dipoles][M][2] complex coefficients.
    ``nmax`` is one largest degree for all frequencies or one per frequency.
    Magnitudes fall as exp(-0.4 (n - 1)) with seeded random phases; each
    dipole's coefficients are a shared pattern plus a 20 % dipole-specific
    part."""
    freqs = np.asarray(freqs_hz, np.uint32)
    nf = freqs.size
    nmx = np.broadcast_to(np.asarray(nmax, np.int32), (nf,)).copy()
    top = int(nmx.max())
    cols = [(s, m, n) for n in range(1, top + 1) for s in (1, 2) for m in range(-n, n + 1)]
    modes = np.array(cols, np.int32).T.copy()
    M = modes.shape[1]
    rng = np.random.default_rng(seed)
    n_of = modes[2].astype(np.float64)
    scale = np.exp(-0.4 * (n_of - 1.0))
    base = (rng.normal(size=(nf, 2, 1, M)) + 1j * rng.normal(size=(nf, 2, 1, M))) * scale
    own = (rng.normal(size=(nf, 2, 16, M)) + 1j * rng.normal(size=(nf, 2, 16, M))) * scale * 0.2
    qc = base + own
    q = np.stack([qc.real, qc.imag], -1)
    num = np.array([2 * k * (k + 2) for k in nmx], np.int32)
    for f in range(nf):  # columns past a frequency's own modes are unused (zero, as padding in a file)
        q[f, :, :, num[f]:, :] = 0.0
    return {"freqs_hz": freqs, "modes": modes, "num_freq_modes": num, "q": np.ascontiguousarray(q)}
