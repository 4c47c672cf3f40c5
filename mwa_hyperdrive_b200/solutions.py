"""Calibration solutions: the device step that completes them after DI
calibration (into_cal_sols, di_calibrate/mod.rs:89-262) and the two file
formats the reference reads and writes (solutions/mod.rs:140-200):
hyperdrive FITS (solutions/hyperdrive.rs) and the "André Offringa" binary
format (solutions/ao.rs).

``di_jones`` is ``[timeblock][tile][chanblock][8]`` float64 (XX re, XX im,
XY re, XY im, YX re, YX im, YY re, YY im), the data->model solutions of every
tile and chanblock with NaN where flagged.  Timestamps are GPS seconds.
"""

from __future__ import annotations

import math
import struct
import sys
from dataclasses import dataclass, field
from pathlib import Path
from typing import List, Optional, Sequence, Union

import numpy as np

from . import _lib
from . import fits
from .model import POLS, _stream_ptr

VEL_C = 299792458.0
PFB_FLAVOURS = ("none", "jake", "cotter2014", "empirical", "levine")


class SolutionsError(ValueError):
    pass


@dataclass
class RawDataCorrections:
    """io/read/mod.rs RawDataCorrections (PFB flavour and three switches)."""

    pfb_flavour: str = "jake"
    digital_gains: bool = True
    cable_length: bool = True
    geometric: bool = True


@dataclass
class CalibrationSolutions:
    """solutions/mod.rs:54-130"""

    di_jones: np.ndarray
    flagged_tiles: List[int] = field(default_factory=list)
    flagged_chanblocks: List[int] = field(default_factory=list)
    chanblock_freqs: Optional[np.ndarray] = None
    obsid: Optional[int] = None
    start_timestamps: Optional[List[float]] = None
    end_timestamps: Optional[List[float]] = None
    average_timestamps: Optional[List[float]] = None
    max_iterations: Optional[int] = None
    stop_threshold: Optional[float] = None
    min_threshold: Optional[float] = None
    raw_data_corrections: Optional[RawDataCorrections] = None
    tile_names: Optional[List[str]] = None
    dipole_gains: Optional[np.ndarray] = None  # [tile][32]
    dipole_delays: Optional[np.ndarray] = None  # [tile][16]
    beam_file: Optional[str] = None
    calibration_results: Optional[np.ndarray] = None  # [timeblock][chanblock] precisions
    baseline_weights: Optional[np.ndarray] = None  # [all baselines]
    uvw_min: Optional[float] = None
    uvw_max: Optional[float] = None
    freq_centroid: Optional[float] = None
    modeller: Optional[str] = None


# ------------------------------------------------------------ device step
def into_cal_sols_device(d_di_jones, flagged_tiles: Sequence[int], flagged_chanblocks: Sequence[int],
                         pols: str = "XX_XY_YX_YY", stream=None):
    """The Jones part of into_cal_sols on the device: a CUDA float64 tensor
    [timeblock][unflagged tile][unflagged chanblock][8] of model->data gains
    to a new [timeblock][tile][chanblock][8] tensor of inverted solutions
    with NaN rows and columns for the flagged tiles and chanblocks."""
    import torch

    if d_di_jones.dtype != torch.float64 or d_di_jones.dim() != 4 or d_di_jones.shape[3] != 8 or \
            not d_di_jones.is_contiguous():
        raise ValueError("into_cal_sols: di_jones must be contiguous float64 [timeblock][tile][chanblock][8]")
    ntb, nut, nuc = (int(x) for x in d_di_jones.shape[:3])
    ft = np.ascontiguousarray(sorted(int(t) for t in flagged_tiles), np.int32)
    fc = np.ascontiguousarray(sorted(int(c) for c in flagged_chanblocks), np.int32)
    out = torch.empty((ntb, nut + ft.size, nuc + fc.size, 8), dtype=torch.float64, device=d_di_jones.device)
    rc = _lib.lib().hdc_into_cal_sols(d_di_jones.data_ptr(), ntb, nut, nuc, ft.ctypes.data if ft.size else None,
                                      int(ft.size), fc.ctypes.data if fc.size else None, int(fc.size), POLS[pols],
                                      out.data_ptr(), _stream_ptr(stream))
    _lib.check(rc, "hdc_into_cal_sols")
    return out


def into_cal_sols(d_di_jones, flagged_tiles: Sequence[int], flagged_chanblocks: Sequence[int],
                  pols: str = "XX_XY_YX_YY", calibration_results=None, unflagged_baseline_weights=None,
                  **metadata) -> CalibrationSolutions:
    """into_cal_sols (di_calibrate/mod.rs:89-262): the inverted, NaN-padded
    solutions (on the device), then on the host the precisions padded with
    NaN for flagged chanblocks (``calibration_results`` is [timeblock]
    [unflagged chanblock]) and the baseline weights with NaN for baselines
    of flagged tiles.  ``metadata`` fills the remaining fields."""
    out = into_cal_sols_device(d_di_jones, flagged_tiles, flagged_chanblocks, pols)
    ntb, ntiles, nch = (int(x) for x in out.shape[:3])
    fc = set(int(c) for c in flagged_chanblocks)
    ft = set(int(t) for t in flagged_tiles)
    results = None
    if calibration_results is not None:
        cr = np.asarray(calibration_results, np.float64)
        results = np.full((ntb, nch), np.nan)
        keep = [c for c in range(nch) if c not in fc]
        if cr.shape != (ntb, len(keep)):
            raise ValueError(f"calibration_results must be [{ntb}][{len(keep)}]")
        results[:, keep] = cr
    bw = None
    if unflagged_baseline_weights is not None:
        w = np.asarray(unflagged_baseline_weights, np.float64)
        bw = np.full(ntiles * (ntiles - 1) // 2, np.nan)
        k = i = 0
        for t1 in range(ntiles):
            for t2 in range(t1 + 1, ntiles):
                if t1 not in ft and t2 not in ft:
                    bw[i] = w[k]
                    k += 1
                i += 1
        if k != w.size:
            raise ValueError(f"{w.size} baseline weights for {k} unflagged baselines")
    return CalibrationSolutions(di_jones=out.cpu().numpy(), flagged_tiles=sorted(ft), flagged_chanblocks=sorted(fc),
                                calibration_results=results, baseline_weights=bw, **metadata)


# ------------------------------------------------------- flags from NaNs
def _flags_from_nans(dj: np.ndarray):
    """Tiles (chanblocks) all of whose Jones matrices hold a NaN are flagged
    (hyperdrive.rs:119-139, ao.rs:80-96)."""
    any_nan = np.isnan(dj).any(axis=3)  # [tb][tile][cb]
    tiles = [int(t) for t in np.nonzero(any_nan.all(axis=(0, 2)))[0]]
    chans = [int(c) for c in np.nonzero(any_nan.all(axis=(0, 1)))[0]]
    return tiles, chans


# -------------------------------------------------------- hyperdrive FITS
def _software() -> str:
    from . import __version__

    return f"Created by mwa_hyperdrive_b200 v{__version__}"


def write_fits(sols: CalibrationSolutions, path: Union[str, Path]) -> None:
    """hyperdrive.rs:547-965: primary keys, SOLUTIONS image, TIMEBLOCKS,
    TILES and CHANBLOCKS tables, RESULTS and BASELINES images."""
    dj = np.ascontiguousarray(sols.di_jones, np.float64)
    if dj.ndim != 4 or dj.shape[3] != 8:
        raise SolutionsError("di_jones must be [timeblock][tile][chanblock][8]")
    ntb, ntiles, nch = dj.shape[:3]
    p = fits.primary_header()
    p.set("LONGSTRN", "OGIP 1.0", "The OGIP long string convention may be used.")
    p.comment("This FITS file may contain long string keyword values that are")
    p.comment("continued over multiple keywords.  This convention uses the  '&'")
    p.comment("character at the end of a string which is then continued")
    p.comment("on subsequent keywords whose name = 'CONTINUE'.")
    p.comment("The contents of this file are documented at:")
    p.comment("https://mwatelescope.github.io/mwa_hyperdrive/defs/cal_sols_hyp.html")
    if sols.obsid is not None:
        p.set("OBSID", str(sols.obsid), "The MWA observation ID")
    rdc = sols.raw_data_corrections
    if rdc is not None:
        p.set("PFB", rdc.pfb_flavour)
        p.set("D_GAINS", "Y" if rdc.digital_gains else "N")
        p.set("CABLELEN", "Y" if rdc.cable_length else "N")
        p.set("GEOMETRY", "Y" if rdc.geometric else "N")
    if sols.max_iterations is not None:
        p.set("MAXITER", int(sols.max_iterations))
    if sols.stop_threshold is not None:
        p.set("S_THRESH", float(sols.stop_threshold))
    if sols.min_threshold is not None:
        p.set("M_THRESH", float(sols.min_threshold))
    for key, cut in (("UVW_MIN", sols.uvw_min), ("UVW_MAX", sols.uvw_max)):
        if cut is None:
            continue
        p.set(key, "inf" if math.isinf(cut) else float(cut))
        if sols.freq_centroid is not None:
            p.set(key + "_L", "inf" if math.isinf(cut) else float(cut) * sols.freq_centroid / VEL_C)
    if sols.beam_file is not None:
        p.set("BEAMFILE", str(sols.beam_file))
    if sols.modeller is not None:
        p.set("MODELLER", sols.modeller)
    p.set("SOFTWARE", _software())
    p.set("CMDLINE", " ".join(sys.argv), "Command-line call")

    hdus = [fits.image_hdu("SOLUTIONS", dj)]
    times = [(n, v) for n, v in (("Start", sols.start_timestamps), ("End", sols.end_timestamps),
                                 ("Average", sols.average_timestamps)) if v is not None]
    if times:
        rows = max(len(v) for _, v in times)
        cols = []
        for n, v in times:
            a = np.zeros(rows)
            a[:len(v)] = v
            cols.append(fits.Column(n, "D", a))
        hdus.append(fits.table_hdu("TIMEBLOCKS", cols, rows))
    flagged_tiles = set(int(t) for t in sols.flagged_tiles)
    cols = [fits.Column("Antenna", "J", np.arange(ntiles, dtype=np.int32)),
            fits.Column("Flag", "I", np.array([t in flagged_tiles for t in range(ntiles)], np.int16))]
    if sols.tile_names is not None:
        if len(sols.tile_names) != ntiles:
            raise SolutionsError(f"{len(sols.tile_names)} tile names for {ntiles} tiles")
        cols.append(fits.Column("TileName", "8A", list(sols.tile_names)))
    if sols.dipole_gains is not None:
        cols.append(fits.Column("DipoleGains", "32D", np.asarray(sols.dipole_gains, np.float64).reshape(ntiles, 32)))
    if sols.dipole_delays is not None:
        cols.append(fits.Column("DipoleDelays", "16J", np.asarray(sols.dipole_delays, np.int32).reshape(ntiles, 16)))
    hdus.append(fits.table_hdu("TILES", cols, ntiles))
    flagged_chans = set(int(c) for c in sols.flagged_chanblocks)
    freqs = np.full(nch, np.nan) if sols.chanblock_freqs is None else np.asarray(sols.chanblock_freqs, np.float64)
    hdus.append(fits.table_hdu("CHANBLOCKS", [
        fits.Column("Index", "J", np.arange(nch, dtype=np.int32)),
        fits.Column("Flag", "1X", np.array([c in flagged_chans for c in range(nch)], bool)),
        fits.Column("Freq", "D", freqs)], nch))
    if sols.calibration_results is not None:
        hdus.append(fits.image_hdu("RESULTS", np.ascontiguousarray(sols.calibration_results, np.float64)))
    if sols.baseline_weights is not None:
        hdus.append(fits.image_hdu("BASELINES", np.ascontiguousarray(sols.baseline_weights, np.float64)))
    fits.write(path, p, hdus)


def _opt_float(h: fits.Header, key: str) -> Optional[float]:
    v = h.get(key)
    if v is None:
        return None
    if isinstance(v, str):
        if v.strip().lower() in ("inf", "+inf"):
            return math.inf
        return float(v)
    return float(v)


def read_fits(path: Union[str, Path]) -> CalibrationSolutions:
    """hyperdrive.rs:37-545.  Flagged tiles and chanblocks come from the
    NaNs of SOLUTIONS, not the Flag columns (a tile can be flagged by
    calibration alone)."""
    p, hdus = fits.read(path)
    sol = fits.find(hdus, "SOLUTIONS")
    if sol is None:
        raise SolutionsError(f"{path}: no SOLUTIONS HDU")
    dj = np.asarray(sol.data, np.float64)
    if dj.ndim != 4:
        raise SolutionsError(f"{path}: SOLUTIONS must have 4 axes")
    if dj.shape[3] != 8:
        raise SolutionsError(f"{path}: SOLUTIONS NAXIS1 must be 8 (4 polarisations)")
    ntb, ntiles, nch = dj.shape[:3]
    tiles, chans = _flags_from_nans(dj)
    s = CalibrationSolutions(di_jones=dj, flagged_tiles=tiles, flagged_chanblocks=chans)
    obsid = p.get("OBSID")
    s.obsid = int(obsid) if obsid is not None else None
    s.max_iterations = int(p["MAXITER"]) if "MAXITER" in p else None
    s.stop_threshold = _opt_float(p, "S_THRESH")
    s.min_threshold = _opt_float(p, "M_THRESH")
    s.uvw_min, s.uvw_max = _opt_float(p, "UVW_MIN"), _opt_float(p, "UVW_MAX")
    umin_l, umax_l = _opt_float(p, "UVW_MIN_L"), _opt_float(p, "UVW_MAX_L")
    if s.uvw_min is not None and umin_l is not None:
        s.freq_centroid = VEL_C / (s.uvw_min / umin_l)
    elif s.uvw_max is not None and umax_l is not None:
        s.freq_centroid = VEL_C / (s.uvw_max / umax_l)
    s.beam_file = p.get("BEAMFILE")
    s.modeller = p.get("MODELLER")
    keys = [p.get(k) for k in ("PFB", "D_GAINS", "CABLELEN", "GEOMETRY")]
    if all(k is not None for k in keys):
        if keys[0].lower() not in PFB_FLAVOURS:
            raise SolutionsError(f"{path}: unknown PFB flavour {keys[0]!r}")
        s.raw_data_corrections = RawDataCorrections(keys[0].lower(), keys[1] == "Y", keys[2] == "Y", keys[3] == "Y")
    tb = fits.find(hdus, "TIMEBLOCKS")
    if tb is not None:
        for name, attr in (("Start", "start_timestamps"), ("End", "end_timestamps"),
                           ("Average", "average_timestamps")):
            v = tb.data.get(name)
            if v is None or np.all(np.asarray(v) == 0.0):
                continue
            if len(v) != ntb:
                raise SolutionsError(f"{path}: {len(v)} {name} timeblocks for {ntb}")
            setattr(s, attr, [float(x) for x in v])
    cb = fits.find(hdus, "CHANBLOCKS")
    if cb is not None and "Freq" in cb.data:
        f = np.asarray(cb.data["Freq"], np.float64)
        if f.size != nch:
            raise SolutionsError(f"{path}: {f.size} chanblock frequencies for {nch}")
        s.chanblock_freqs = None if np.isnan(f).any() else f
    tl = fits.find(hdus, "TILES")
    if tl is not None:
        if "TileName" in tl.data:
            names = list(tl.data["TileName"])
            if len(names) != ntiles:
                raise SolutionsError(f"{path}: {len(names)} tile names for {ntiles}")
            s.tile_names = names
        if "DipoleGains" in tl.data:
            s.dipole_gains = np.asarray(tl.data["DipoleGains"], np.float64).reshape(ntiles, 32)
        if "DipoleDelays" in tl.data:
            s.dipole_delays = np.asarray(tl.data["DipoleDelays"], np.int64).reshape(ntiles, 16).astype(np.uint32)
    res = fits.find(hdus, "RESULTS")
    if res is not None and res.data is not None:
        r = np.asarray(res.data, np.float64)
        if r.shape != (ntb, nch):
            raise SolutionsError(f"{path}: RESULTS is {r.shape}, expected {(ntb, nch)}")
        s.calibration_results = r
    bl = fits.find(hdus, "BASELINES")
    if bl is not None and bl.data is not None:
        w = np.asarray(bl.data, np.float64).reshape(-1)
        if w.size != ntiles * (ntiles - 1) // 2:
            raise SolutionsError(f"{path}: {w.size} baseline weights for {ntiles} tiles")
        s.baseline_weights = w
    return s


# ----------------------------------------------------------- AO binary
_AO_HEADER = struct.Struct("<7s9x4I2d")


def write_ao(sols: CalibrationSolutions, path: Union[str, Path]) -> None:
    """ao.rs:132-183: "MWAOCAL", nine zero bytes, four u32 sizes, start and
    end GPS time (0 if unknown), then the Jones matrices as f64, all
    little-endian."""
    dj = np.ascontiguousarray(sols.di_jones, np.float64)
    ntb, ntiles, nch = dj.shape[:3]
    st = list(sols.start_timestamps or [])
    en = list(sols.end_timestamps or [])
    av = list(sols.average_timestamps or [])
    if st and en:
        start, end = st[0], en[-1]
    elif sols.start_timestamps is not None and sols.end_timestamps is not None and not st and not en and av:
        start, end = av[0], av[-1]
    elif st:
        start, end = st[0], 0.0
    elif en:
        start, end = 0.0, en[-1]
    else:
        start, end = 0.0, 0.0
    with open(path, "wb") as f:
        f.write(_AO_HEADER.pack(b"MWAOCAL", ntb, ntiles, nch, 4, start, end))
        f.write(dj.astype("<f8").tobytes())


def read_ao(path: Union[str, Path]) -> CalibrationSolutions:
    """ao.rs:22-130."""
    buf = Path(path).read_bytes()
    if len(buf) < _AO_HEADER.size or buf[:7] != b"MWAOCAL":
        raise SolutionsError(f"{path}: does not start with MWAOCAL")
    if any(buf[7:16]):
        raise SolutionsError(f"{path}: expected nine zero bytes after MWAOCAL")
    _, ntb, ntiles, nch, npol, t0, t1 = _AO_HEADER.unpack_from(buf)
    n = ntb * ntiles * nch * 2 * npol
    body = buf[_AO_HEADER.size:_AO_HEADER.size + 8 * n]
    if len(body) != 8 * n:
        raise SolutionsError(f"{path}: truncated")
    dj = np.frombuffer(body, "<f8").astype(np.float64).reshape(ntb, ntiles, nch, 2 * npol)
    tiles, chans = _flags_from_nans(dj)
    eps = np.finfo(np.float64).eps
    start = None if abs(t0) < eps else t0
    end = None if abs(t1) < eps else t1
    s = CalibrationSolutions(di_jones=dj, flagged_tiles=tiles, flagged_chanblocks=chans)
    if start is not None:
        s.start_timestamps = [start]
    if end is not None:
        s.end_timestamps = [end]
    if start is not None and end is not None:
        s.average_timestamps = [(start + end) / 2.0]
    return s


# ------------------------------------------------------------- dispatch
def read_solutions(path: Union[str, Path]) -> CalibrationSolutions:
    """solutions/mod.rs:145-175: by extension, .fits or .bin."""
    ext = Path(path).suffix.lower()
    if ext == ".fits":
        return read_fits(path)
    if ext == ".bin":
        return read_ao(path)
    raise SolutionsError(f"cannot read calibration solutions from a {ext or '<no extension>'} file")


def write_solutions(sols: CalibrationSolutions, path: Union[str, Path]) -> None:
    """solutions/mod.rs:176-200."""
    ext = Path(path).suffix.lower()
    if ext == ".fits":
        write_fits(sols, path)
    elif ext == ".bin":
        write_ao(sols, path)
    else:
        raise SolutionsError(f"cannot write calibration solutions to a {ext or '<no extension>'} file")
