"""uvfits visibilities (AIPS random groups) on either side of the
calibration path: the reader feeds `calibrate.vis_average` /
`scale_by_weights` and the DI solver, the writer makes files for it.

The reader follows mwa_hyperdrive's `UvfitsReader` (io/read/uvfits/mod.rs):

* group parameters by PTYPE (mod.rs:1559-1700): UU, VV, WW (seconds),
  BASELINE or ANTENNA1 + ANTENNA2, one or two DATE (JD = PZERO of the first
  + the sum of the DATE values, as the stored FP32 numbers), INTTIM; data axes
  by CTYPE: COMPLEX, STOKES, FREQ, RA, DEC (others, e.g. IF, of length 1);
* polarisations from CRVAL and NAXIS of STOKES (mod.rs:1228-1270): -5 with
  1, 2, 3, 4 pols = XX, XX_YY, XX_YY_XY, XX_XY_YX_YY (stored XX, YY, XY, YX),
  -6 with 1 = YY;
* timestamps: the distinct JDs in file order, rounded to 10 ms; the rows of
  a timestep are contiguous and every timestep has the same count
  (mod.rs:1312-1470); fine channel frequencies round(CRVAL + (i - round(CRPIX)
  + 1) CDELT) (mod.rs:480-488);
* tiles from the "AIPS AN" table: ANNAME, NOSTA (the numbers the baselines
  use), STABXYZ relative to ARRAYX/Y/Z in the ITRF frame; ARRAYX/Y/Z all zero
  (as casacore writes them) means STABXYZ are geocentric: the array position
  is then their mean and the tiles are rotated into the array's frame
  (mod.rs:118-200);
* the baseline convention: the first cross-correlation's UVW is compared
  with the UVWs of tile1 - tile2 and tile2 - tile1 at the phase centre; if it
  is closer to the latter the visibilities are conjugated (io/read/mod.rs:
  168-220, mod.rs:579-650);
* cross-correlation reads (mod.rs:695-880): visibilities of a timestep into
  [unflagged channel][unflagged baseline] Jones (XX, XY, YX, YY; absent pols
  zero), the weight of a visibility the smallest of its pols' weights (1.0
  when the file carries none), baselines of flagged tiles skipped, the
  YY-only layout moved into the YY slot (mod.rs:960-1020); autos likewise.

The UVW comparison uses the hour angle from the Earth rotation angle (IAU
2000 formula) and the array longitude, without precession or DUT1: the two
candidate UVWs are each other's negatives, so the choice does not depend on
those sub-degree corrections (the reference notes the same).  Geocentric
positions convert to WGS84 by an iteration converged to machine precision
(the published geodetic latitude fixed point), heights by
h = p cos(lat) + z sin(lat) - a sqrt(1 - e^2 sin^2(lat)).

Baseline numbers use the AIPS encoding: 256 a1 + a2 for antenna numbers
below 256, else 2048 a1 + a2 + 65536.
"""

from __future__ import annotations

import math
from dataclasses import dataclass
from pathlib import Path
from typing import List, Optional, Sequence, Tuple, Union

import numpy as np

from . import fits

VEL_C = 299792458.0
WGS84_A = 6378137.0
WGS84_F = 1.0 / 298.257223563
WGS84_E2 = WGS84_F * (2.0 - WGS84_F)

POLS = {(-5, 1): "XX", (-5, 2): "XX_YY", (-5, 3): "XX_YY_XY", (-5, 4): "XX_XY_YX_YY", (-6, 1): "YY"}
# stored order of each layout -> slot of the Jones (XX 0, XY 1, YX 2, YY 3)
_STORED_SLOTS = {"XX": (0,), "XX_YY": (0, 3), "XX_YY_XY": (0, 3, 1), "XX_XY_YX_YY": (0, 3, 1, 2), "YY": (0,)}

# TAI - UTC (s) from the start of each period (MJD), 1980 onwards (IERS)
_LEAP_MJD = [44239, 44786, 45151, 45516, 46247, 47161, 47892, 48257, 48804, 49169, 49534, 50083, 50630, 51179,
             53736, 54832, 56109, 57204, 57754]
_LEAP_TAI_UTC = [19, 20, 21, 22, 23, 24, 25, 26, 27, 28, 29, 30, 31, 32, 33, 34, 35, 36, 37]
MJD_JD = 2400000.5
GPS_EPOCH_JD = 2444244.5


class UvfitsError(ValueError):
    pass


# ------------------------------------------------------------------ geometry
def decode_baseline(bl: int) -> Tuple[int, int]:
    bl = int(bl)
    if bl < 65536:
        return bl >> 8, bl & 255
    bl -= 65536
    return bl >> 11, bl & 2047


def encode_baseline(a1: int, a2: int) -> int:
    if a1 < 256 and a2 < 256:
        return 256 * a1 + a2
    return 2048 * a1 + a2 + 65536


def geocentric_to_wgs84(x: float, y: float, z: float) -> Tuple[float, float, float]:
    """(longitude, latitude) [rad] and height [m] of a geocentric point."""
    lon = math.atan2(y, x)
    p = math.hypot(x, y)
    lat = math.atan2(z, p * (1.0 - WGS84_E2))
    for _ in range(50):
        s = math.sin(lat)
        n = WGS84_A / math.sqrt(1.0 - WGS84_E2 * s * s)
        nxt = math.atan2(z + WGS84_E2 * n * s, p)
        if nxt == lat:
            break
        lat = nxt
    s, c = math.sin(lat), math.cos(lat)
    h = p * c + z * s - WGS84_A * math.sqrt(1.0 - WGS84_E2 * s * s)
    return lon, lat, h


def wgs84_to_geocentric(lon: float, lat: float, h: float) -> Tuple[float, float, float]:
    s, c = math.sin(lat), math.cos(lat)
    n = WGS84_A / math.sqrt(1.0 - WGS84_E2 * s * s)
    return (n + h) * c * math.cos(lon), (n + h) * c * math.sin(lon), (n * (1.0 - WGS84_E2) + h) * s


def geocentric_to_array_frame(xyz: np.ndarray, lon: float, lat: float, h: float) -> np.ndarray:
    """Geocentric positions [n][3] to the array's frame (the uvfits STABXYZ
    frame: the geocentric offset from the array rotated by the longitude)."""
    x0, y0, z0 = wgs84_to_geocentric(lon, lat, h)
    d = np.asarray(xyz, np.float64) - np.array([x0, y0, z0])
    s, c = math.sin(lon), math.cos(lon)
    return np.stack([c * d[:, 0] + s * d[:, 1], -s * d[:, 0] + c * d[:, 1], d[:, 2]], axis=1)


def earth_rotation_angle(jd_ut1: float) -> float:
    """IAU 2000 Earth rotation angle [rad]."""
    d = jd_ut1 - 2451545.0
    return 2.0 * math.pi * ((0.7790572732640 + 1.00273781191135448 * d) % 1.0)


def uvw_from_xyz(dxyz: np.ndarray, ha: float, dec: float) -> np.ndarray:
    """UVW [m] of baseline vectors [n][3] (array frame) towards (ha, dec)."""
    sh, ch, sd, cd = math.sin(ha), math.cos(ha), math.sin(dec), math.cos(dec)
    x, y, z = dxyz[..., 0], dxyz[..., 1], dxyz[..., 2]
    return np.stack([sh * x + ch * y, -sd * ch * x + sd * sh * y + cd * z, cd * ch * x - cd * sh * y + sd * z], -1)


def jd_utc_to_gps(jd: float) -> float:
    """GPS seconds of a UTC Julian date (1980 onwards)."""
    mjd = jd - MJD_JD
    k = int(np.searchsorted(_LEAP_MJD, mjd, side="right")) - 1
    if k < 0:
        raise UvfitsError("dates before 1980 have no GPS time")
    return (jd - GPS_EPOCH_JD) * 86400.0 + (_LEAP_TAI_UTC[k] - 19)


def gps_to_jd_utc(gps: float) -> float:
    jd = GPS_EPOCH_JD + gps / 86400.0
    for _ in range(3):  # leap seconds depend on the UTC date itself
        jd = GPS_EPOCH_JD + (gps - (jd_utc_to_gps(jd) - (jd - GPS_EPOCH_JD) * 86400.0)) / 86400.0
    return jd


def _round_10ms(jd: float) -> float:
    return round(jd * 8640000.0) / 8640000.0


# ------------------------------------------------------------------- reading
@dataclass
class UvfitsObs:
    timestamps_jd: np.ndarray          # UTC Julian dates of the timesteps (10 ms rounding)
    timestamps_gps: np.ndarray         # the same as GPS seconds
    time_res: Optional[float]          # s (INTTIM, else the smallest gap; None with one timestep)
    fine_chan_freqs: np.ndarray        # Hz
    freq_res: float                    # Hz
    tile_names: List[str]
    tile_numbers: List[int]            # NOSTA
    tile_xyzs: np.ndarray              # [tile][3] m, array frame
    array_position: Tuple[float, float, float]           # lon, lat [rad], height [m] in use
    supplied_array_position: Tuple[float, float, float]  # from the file
    phase_centre: Tuple[float, float]  # RA, Dec [rad]
    polarisations: str
    autocorrelations_present: bool
    unavailable_tiles: List[int]
    flagged_tiles: List[int]
    dut1: Optional[float]
    conjugate_vis: bool
    num_rows: int
    rows_per_timestep: int


def _params_index(h: fits.Header):
    ptypes = []
    i = 1
    while f"PTYPE{i}" in h:
        ptypes.append(str(h[f"PTYPE{i}"]).strip())
        i += 1
    idx = {}
    dates = []
    for k, name in enumerate(ptypes):
        if name in ("UU", "VV", "WW", "BASELINE", "ANTENNA1", "ANTENNA2", "INTTIM") and name not in idx:
            idx[name] = k
        elif name in ("DATE", "_DATE") and len(dates) < 2:
            dates.append(k)
    for key in ("UU", "VV", "WW"):
        if key not in idx:
            raise UvfitsError(f"uvfits has no {key} group parameter")
    if not dates:
        raise UvfitsError("uvfits has no DATE group parameter")
    if "BASELINE" not in idx and not ("ANTENNA1" in idx and "ANTENNA2" in idx):
        if "ANTENNA1" in idx or "ANTENNA2" in idx:
            raise UvfitsError("uvfits has only one of ANTENNA1 and ANTENNA2")
        raise UvfitsError("uvfits has neither BASELINE nor ANTENNA1/ANTENNA2")
    return idx, dates


def _axis_index(h: fits.Header):
    axes = {}
    i = 2
    while f"CTYPE{i}" in h:
        name = str(h[f"CTYPE{i}"]).strip()
        if name in ("COMPLEX", "STOKES", "FREQ", "RA", "DEC"):
            axes[name] = i
        i += 1
    for key in ("COMPLEX", "STOKES", "FREQ", "RA", "DEC"):
        if key not in axes:
            raise UvfitsError(f"uvfits has no {key} axis")
    if axes["COMPLEX"] != 2 or axes["STOKES"] != 3 or axes["FREQ"] != 4:
        raise UvfitsError("uvfits data axes must be COMPLEX, STOKES, FREQ in that order")
    return axes


class UvfitsReader:
    """uvfits file reader with the reference's UvfitsReader semantics."""

    def __init__(self, path: Union[str, Path], array_position: Optional[Tuple[float, float, float]] = None):
        self.path = Path(path)
        if not self.path.exists():
            raise UvfitsError(f"no such uvfits file: {self.path}")
        h, hdus = fits.read(self.path)
        groups = [x for x in hdus if x.kind == "GROUPS"]
        if not groups or h.get("GROUPS") is not True:
            raise UvfitsError("not a random-groups (uvfits) file")
        an = fits.find(hdus, "AIPS AN")
        if an is None:
            raise UvfitsError("uvfits has no AIPS AN table")
        self.header = h
        rows = groups[0].data
        pcount = int(h["PCOUNT"])
        self._params = rows[:, :pcount]
        idx, dates = _params_index(h)
        axes = _axis_index(h)
        self._idx, self._dates = idx, dates

        nfloat = int(h["NAXIS2"])
        if nfloat not in (2, 3):
            raise UvfitsError(f"uvfits NAXIS2 (floats per pol) is {nfloat}; 2 or 3 expected")
        npol = int(h[f"NAXIS{axes['STOKES']}"])
        pol_type = int(round(float(h[f"CRVAL{axes['STOKES']}"])))
        pols = POLS.get((pol_type, npol))
        if pols is None:
            raise UvfitsError(f"unsupported uvfits polarisations (CRVAL {pol_type}, {npol} pols)")
        nchan = int(h[f"NAXIS{axes['FREQ']}"])
        extra = int(np.prod([int(h[f"NAXIS{i}"]) for i in range(5, int(h["NAXIS"]) + 1)]))
        if extra != 1:
            raise UvfitsError("uvfits axes beyond FREQ must have length 1")
        self._vis = rows[:, pcount:].reshape(rows.shape[0], nchan, npol, nfloat)
        self._nfloat, self._npol, self._pols = nfloat, npol, pols

        # timestamps: JD zero (PZERO of the first DATE, to the hour unless 0)
        # plus the sum of the DATE parameters, as the stored FP32 values
        jd_zero = float(h.get(f"PZERO{dates[0] + 1}", 0.0))
        if abs(jd_zero) > 0.0:
            jd_zero = round(jd_zero * 24.0) / 24.0
        frac = self._params[:, dates[0]].astype(np.float64)
        if len(dates) > 1:
            frac = frac + self._params[:, dates[1]].astype(np.float64)
        self._jd_frac = frac
        uniq, first = [], {}
        for r, v in enumerate(frac):
            if v not in first:
                first[v] = r
                uniq.append(v)
        step = next((first[v] for v in uniq[1:]), len(frac))
        if len(frac) % step:
            raise UvfitsError("uvfits timesteps hold different numbers of baselines")
        for t in range(len(uniq)):
            if not np.all(frac[t * step:(t + 1) * step] == uniq[t]):
                raise UvfitsError("uvfits rows of a timestep are not contiguous")
        jds = np.array([_round_10ms(jd_zero + v) for v in uniq])

        a1, a2 = self._antennas(np.arange(rows.shape[0]))
        tile_numbers = [int(v) for v in np.atleast_1d(an.data["NOSTA"])]
        tile_names = list(an.data["ANNAME"])
        self._tile_map = {n: i for i, n in enumerate(tile_numbers)}
        present = set(int(v) for v in a1) | set(int(v) for v in a2)
        unavailable = sorted(i for n, i in self._tile_map.items() if n not in present)

        # array position and tile positions
        ax, ay, az = (float(an.header.get(k, 0.0)) for k in ("ARRAYX", "ARRAYY", "ARRAYZ"))
        stab = np.asarray(an.data["STABXYZ"], np.float64).reshape(-1, 3)
        blessed = abs(ax) < np.finfo(float).eps and abs(ay) < np.finfo(float).eps and abs(az) < np.finfo(float).eps
        if blessed:
            mean = [0.0, 0.0, 0.0]
            for row in stab:  # in row order
                mean[0] += row[0]
                mean[1] += row[1]
                mean[2] += row[2]
            n = float(len(stab))
            supplied = geocentric_to_wgs84(mean[0] / n, mean[1] / n, mean[2] / n)
            pos = array_position or supplied
            tile_xyzs = geocentric_to_array_frame(stab, *pos)
        else:
            supplied = geocentric_to_wgs84(ax, ay, az)
            pos = array_position or supplied
            tile_xyzs = stab.copy()

        ra = math.radians(float(h[f"CRVAL{axes['RA']}"]))
        dec = math.radians(float(h[f"CRVAL{axes['DEC']}"]))
        dut1 = an.header.get("UT1UTC")

        # time resolution: INTTIM, else the smallest gap between timestamps
        time_res = None
        if "INTTIM" in idx:
            time_res = float(self._params[0, idx["INTTIM"]])
        elif len(jds) > 1:
            # the timestamps are whole multiples of 10 ms
            time_res = min(round((b - a) * 8640000.0) for a, b in zip(jds[:-1], jds[1:])) / 100.0

        freqs_key = axes["FREQ"]
        base, res = float(h[f"CRVAL{freqs_key}"]), float(h[f"CDELT{freqs_key}"])
        crpix = int(round(float(h[f"CRPIX{freqs_key}"])))
        fine = np.array([round(base + (i - crpix + 1) * res) for i in range(nchan)], np.float64)

        # baseline convention from the first cross-correlation row
        conj = False
        cross = np.nonzero(a1 != a2)[0]
        if cross.size:
            r = int(cross[0])
            t1, t2 = self._tile_map[int(a1[r])], self._tile_map[int(a2[r])]
            data_uvw = self._params[r, [idx["UU"], idx["VV"], idx["WW"]]].astype(np.float64) * VEL_C
            ha = earth_rotation_angle(jds[0] + (float(dut1) if dut1 is not None else 0.0) / 86400.0) + pos[0] - ra
            d = tile_xyzs[t1] - tile_xyzs[t2]
            u1 = uvw_from_xyz(d[None, :], ha, dec)[0]
            d1 = np.abs(data_uvw - u1).sum()
            d2 = np.abs(data_uvw + u1).sum()
            conj = bool(d2 < d1)

        self.obs = UvfitsObs(
            timestamps_jd=jds, timestamps_gps=np.array([jd_utc_to_gps(j) for j in jds]), time_res=time_res,
            fine_chan_freqs=fine, freq_res=res, tile_names=tile_names, tile_numbers=tile_numbers,
            tile_xyzs=tile_xyzs, array_position=tuple(pos), supplied_array_position=tuple(supplied),
            phase_centre=(ra, dec), polarisations=pols, autocorrelations_present=bool(np.any(a1 == a2)),
            unavailable_tiles=unavailable, flagged_tiles=list(unavailable),
            dut1=None if dut1 is None else float(dut1), conjugate_vis=conj, num_rows=rows.shape[0],
            rows_per_timestep=step)

    def _antennas(self, rows: np.ndarray):
        p = self._params
        if "BASELINE" in self._idx:
            bl = p[rows, self._idx["BASELINE"]].astype(np.int64)
            a1 = np.where(bl < 65536, bl >> 8, (bl - 65536) >> 11)
            a2 = np.where(bl < 65536, bl & 255, (bl - 65536) & 2047)
            return a1, a2
        return p[rows, self._idx["ANTENNA1"]].astype(np.int64), p[rows, self._idx["ANTENNA2"]].astype(np.int64)

    def _rows(self, timestep: int) -> np.ndarray:
        step = self.obs.rows_per_timestep
        if not 0 <= timestep < len(self.obs.timestamps_jd):
            raise UvfitsError(f"timestep {timestep} is not in the uvfits")
        return np.arange(timestep * step, (timestep + 1) * step)

    def _jones(self, rows: np.ndarray, chans: np.ndarray):
        """Jones [row][chan][8] float32 and weights [row][chan] of the rows."""
        d = self._vis[rows][:, chans]  # [r][c][pol][float]
        out = np.zeros(d.shape[:2] + (8,), np.float32)
        for k, slot in enumerate(_STORED_SLOTS[self._pols]):
            out[..., 2 * slot] = d[..., k, 0]
            out[..., 2 * slot + 1] = d[..., k, 1]
        if self._nfloat == 3:
            w = d[..., 0, 2].copy()
            for k in range(1, self._npol):
                w = np.where(d[..., k, 2] < w, d[..., k, 2], w)
        else:
            w = np.ones(d.shape[:2], np.float32)
        return out, w.astype(np.float32)

    def _finish(self, vis: np.ndarray) -> np.ndarray:
        if self.obs.conjugate_vis:
            vis[..., 1::2] = -vis[..., 1::2]
        if self._pols == "YY":  # the one stored pol was read into XX
            vis[..., 6:8] = vis[..., 0:2]
            vis[..., 0:2] = 0.0
        return vis

    def read_crosses(self, timestep: int, flagged_tiles: Sequence[int] = (),
                     flagged_fine_chans: Sequence[int] = ()):
        """Cross-correlations of a timestep: (vis [chan][bl][8] float32,
        weights [chan][bl] float32) over the unflagged channels and the
        baselines (i < j) of the unflagged tiles in tile order.  Baselines the
        file lacks stay zero with zero weight."""
        n = len(self.obs.tile_names)
        flagged = set(int(t) for t in flagged_tiles)
        keep = [t for t in range(n) if t not in flagged]
        pos = {t: k for k, t in enumerate(keep)}
        nk = len(keep)
        chans = np.array([c for c in range(len(self.obs.fine_chan_freqs)) if c not in set(flagged_fine_chans)], int)
        rows = self._rows(timestep)
        a1, a2 = self._antennas(rows)
        sel, bls = [], []
        for r, x, y in zip(rows, a1, a2):
            t1, t2 = self._tile_map[int(x)], self._tile_map[int(y)]
            if t1 == t2 or t1 not in pos or t2 not in pos or t1 > t2:
                continue
            i, j = pos[t1], pos[t2]
            sel.append(r)
            bls.append(i * nk - i * (i + 1) // 2 + (j - i - 1))
        nbl = nk * (nk - 1) // 2
        vis = np.zeros((chans.size, nbl, 8), np.float32)
        wts = np.zeros((chans.size, nbl), np.float32)
        if sel:
            v, w = self._jones(np.array(sel), chans)
            vis[:, bls] = np.transpose(v, (1, 0, 2))
            wts[:, bls] = w.T
        return self._finish(vis), wts

    def read_autos(self, timestep: int, flagged_tiles: Sequence[int] = (), flagged_fine_chans: Sequence[int] = ()):
        """Auto-correlations of a timestep: (vis [chan][tile][8], weights
        [chan][tile]) over the unflagged tiles and channels."""
        n = len(self.obs.tile_names)
        flagged = set(int(t) for t in flagged_tiles)
        keep = [t for t in range(n) if t not in flagged]
        pos = {t: k for k, t in enumerate(keep)}
        chans = np.array([c for c in range(len(self.obs.fine_chan_freqs)) if c not in set(flagged_fine_chans)], int)
        rows = self._rows(timestep)
        a1, a2 = self._antennas(rows)
        sel, tiles = [], []
        for r, x, y in zip(rows, a1, a2):
            t = self._tile_map[int(x)]
            if int(x) == int(y) and t in pos:
                sel.append(r)
                tiles.append(pos[t])
        vis = np.zeros((chans.size, len(keep), 8), np.float32)
        wts = np.zeros((chans.size, len(keep)), np.float32)
        if sel:
            v, w = self._jones(np.array(sel), chans)
            vis[:, tiles] = np.transpose(v, (1, 0, 2))
            wts[:, tiles] = w.T
        return self._finish(vis), wts


# ------------------------------------------------------------------- writing
def write_uvfits(path: Union[str, Path], vis: np.ndarray, weights: np.ndarray, timestamps_jd: Sequence[float],
                 fine_chan_freqs: Sequence[float], tile_names: Sequence[str], tile_xyzs: np.ndarray,
                 array_position: Tuple[float, float, float], phase_centre: Tuple[float, float],
                 autos: Optional[Tuple[np.ndarray, np.ndarray]] = None, int_time: Optional[float] = None,
                 ant2_minus_ant1: bool = False, telescope: str = "MWA") -> None:
    """Write cross-correlations vis [t][f][bl][8] (Jones XX, XY, YX, YY as
    re, im; baselines i < j in tile order) with weights [t][f][bl], and
    optionally autos (vis [t][f][tile][8], weights [t][f][tile]), as a
    uvfits file: rows per timestep in (i, j) order with i <= j, four pols
    stored XX, YY, XY, YX with weights, one BASELINE and two DATE parameters
    (JD zero at the first timestamp's midnight), UVWs of tile_i - tile_j at
    each timestamp (or tile_j - tile_i, with every visibility conjugated, as
    a reader of that convention conjugates them back, if ant2_minus_ant1),
    and an AIPS AN table relative to the array position."""
    vis = np.asarray(vis, np.float32)
    weights = np.asarray(weights, np.float32)
    nt, nf, nbl = vis.shape[:3]
    n = len(tile_names)
    if nbl != n * (n - 1) // 2:
        raise UvfitsError("vis must hold every baseline i < j of the tiles")
    xyz = np.asarray(tile_xyzs, np.float64)
    lon, lat, height = array_position
    ra, dec = phase_centre
    jd0 = math.floor(float(timestamps_jd[0]) - 0.5) + 0.5  # midnight
    pairs = [(i, j) for i in range(n) for j in range(i, n) if autos is not None or i != j]
    bl_index = {}
    k = 0
    for i in range(n):
        for j in range(i + 1, n):
            bl_index[(i, j)] = k
            k += 1
    pcount = 6
    ncell = nf * 4 * 3
    rows = np.zeros((nt * len(pairs), pcount + ncell), np.float32)
    order = (0, 3, 1, 2)  # stored XX, YY, XY, YX
    for t in range(nt):
        jd = float(timestamps_jd[t])
        ha = earth_rotation_angle(jd) + lon - ra
        for r, (i, j) in enumerate(pairs):
            row = rows[t * len(pairs) + r]
            d = (xyz[j] - xyz[i]) if ant2_minus_ant1 else (xyz[i] - xyz[j])
            row[0:3] = uvw_from_xyz(d[None, :], ha, dec)[0] / VEL_C
            row[3] = encode_baseline(i + 1, j + 1)
            frac = jd - jd0
            row[4] = np.float32(frac)
            row[5] = np.float32(frac - float(np.float32(frac)))
            if i == j:
                jv, jw = autos[0][t, :, i], autos[1][t, :, i]
            else:
                jv, jw = vis[t, :, bl_index[(i, j)]], weights[t, :, bl_index[(i, j)]]
            cell = np.zeros((nf, 4, 3), np.float32)
            for k2, slot in enumerate(order):
                cell[:, k2, 0] = jv[:, 2 * slot]
                cell[:, k2, 1] = -jv[:, 2 * slot + 1] if ant2_minus_ant1 else jv[:, 2 * slot + 1]
                cell[:, k2, 2] = jw
            row[pcount:] = cell.reshape(-1)
    freqs = np.asarray(fine_chan_freqs, np.float64)
    res = float(freqs[1] - freqs[0]) if freqs.size > 1 else 1.0

    h = fits.Header()
    h.set("SIMPLE", True, "conforms to FITS standard")
    h.set("BITPIX", -32, "32-bit floating point")
    h.set("NAXIS", 6, "number of axes")
    for ax, v in enumerate([0, 3, 4, nf, 1, 1], start=1):
        h.set(f"NAXIS{ax}", v, "random groups" if ax == 1 else "")
    h.set("EXTEND", True, "tables follow")
    h.set("GROUPS", True, "random group visibility data")
    h.set("PCOUNT", pcount, "parameters per group")
    h.set("GCOUNT", int(rows.shape[0]), "number of groups (rows)")
    h.set("OBJECT", "Undefined", "")
    h.set("TELESCOP", telescope, "")
    h.set("BSCALE", 1.0, "")
    h.set("BZERO", 0.0, "")
    h.set("BUNIT", "Jy", "")
    for ax, (ctype, crval, cdelt, crpix) in enumerate(
            [("COMPLEX", 1.0, 1.0, 1.0), ("STOKES", -5.0, -1.0, 1.0), ("FREQ", float(freqs[0]), res, 1.0),
             ("RA", math.degrees(ra), 1.0, 1.0), ("DEC", math.degrees(dec), 1.0, 1.0)], start=2):
        h.set(f"CTYPE{ax}", ctype, "")
        h.set(f"CRVAL{ax}", crval, "")
        h.set(f"CDELT{ax}", cdelt, "")
        h.set(f"CRPIX{ax}", crpix, "")
    for k2, (ptype, pzero) in enumerate([("UU", 0.0), ("VV", 0.0), ("WW", 0.0), ("BASELINE", 0.0),
                                          ("DATE", jd0), ("DATE", 0.0)], start=1):
        h.set(f"PTYPE{k2}", ptype, "")
        h.set(f"PSCAL{k2}", 1.0, "")
        h.set(f"PZERO{k2}", pzero, "")
    h.set("OBSRA", math.degrees(ra), "phase centre RA [deg]")
    h.set("OBSDEC", math.degrees(dec), "phase centre Dec [deg]")
    h.set("EPOCH", 2000.0, "")
    if int_time is not None:
        h.set("INTTIM", float(int_time), "integration time [s]")

    ax, ay, az = wgs84_to_geocentric(lon, lat, height)
    cols = [fits.Column("ANNAME", "8A", [str(s)[:8] for s in tile_names]),
            fits.Column("STABXYZ", "3D", xyz),
            fits.Column("NOSTA", "1J", np.arange(1, n + 1, dtype=np.int32)),
            fits.Column("MNTSTA", "1J", np.zeros(n, np.int32)),
            fits.Column("STAXOF", "1E", np.zeros(n, np.float32)),
            fits.Column("POLTYA", "1A", ["X"] * n),
            fits.Column("POLAA", "1E", np.zeros(n, np.float32)),
            fits.Column("POLCALA", "1E", np.zeros(n, np.float32)),
            fits.Column("POLTYB", "1A", ["Y"] * n),
            fits.Column("POLAB", "1E", np.full(n, 90.0, np.float32)),
            fits.Column("POLCALB", "1E", np.zeros(n, np.float32))]
    tab = fits.table_hdu("AIPS AN", cols, n)
    for key, val in (("ARRAYX", ax), ("ARRAYY", ay), ("ARRAYZ", az), ("FREQ", float(freqs[0])),
                     ("TIMSYS", "UTC"), ("FRAME", "ITRF"), ("ARRNAM", telescope)):
        tab.header.set(key, val, "")
    fits.write(path, h, [tab], primary_data=rows)
