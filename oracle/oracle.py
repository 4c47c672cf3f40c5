"""ORACLE (test infrastructure only): ctypes wrapper around oracle/oracle.cpp,
the CPU FP64 restatement of mwa_hyperdrive's predict / DI-calibrate / peel
algorithms.  Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
arm import this module; the product never does.

Sky models are passed as any object with the struct-of-arrays attributes of
``mwa_hyperdrive_b200.srclist.SkyModelArrays`` (duck-typed).
"""

from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "liboracle.so"

SBF_N, SBF_L = 101, 10001


def build(force: bool = False) -> Path:
    """Compile oracle.cpp with g++ (OpenMP, no FMA contraction)."""
    src = HERE / "oracle.cpp"
    if LIB.exists() and not force and LIB.stat().st_mtime >= src.stat().st_mtime:
        return LIB
    LIB.parent.mkdir(exist_ok=True)
    cmd = ["g++", "-std=c++17", "-O3", "-march=x86-64-v3", "-ffp-contract=off", "-fopenmp", "-fPIC", "-shared",
           "-o", str(LIB), str(src)]
    subprocess.check_call(cmd)
    return LIB


class OrSky(ctypes.Structure):
    _fields_ = [
        ("num_components", ctypes.c_int),
        ("comp_type", ctypes.c_void_p), ("ra", ctypes.c_void_p), ("dec", ctypes.c_void_p),
        ("maj", ctypes.c_void_p), ("min", ctypes.c_void_p), ("pa", ctypes.c_void_p),
        ("flux_type", ctypes.c_void_p), ("si", ctypes.c_void_p), ("q", ctypes.c_void_p),
        ("fd_start", ctypes.c_void_p), ("fd_count", ctypes.c_void_p), ("fds", ctypes.c_void_p),
        ("coeff_start", ctypes.c_void_p), ("coeff_count", ctypes.c_void_p), ("coeff_n1", ctypes.c_void_p),
        ("coeff_n2", ctypes.c_void_p), ("coeff_value", ctypes.c_void_p),
    ]


class OrBeam(ctypes.Structure):
    _fields_ = [
        ("kind", ctypes.c_int),
        ("beam_jones", ctypes.c_void_p * 3),
        ("tile_map", ctypes.c_void_p),
        ("freq_map", ctypes.c_void_p),
        ("num_unique_freqs", ctypes.c_int),
    ]


class OrCalResult(ctypes.Structure):
    _fields_ = [("num_iterations", ctypes.c_int), ("converged", ctypes.c_int), ("max_precision", ctypes.c_double),
                ("num_failed", ctypes.c_int)]


class OrIono(ctypes.Structure):
    _fields_ = [("alpha", ctypes.c_double), ("beta", ctypes.c_double), ("gain", ctypes.c_double)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        _lib = ctypes.CDLL(str(LIB))
    return _lib


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None else ctypes.c_void_p(0)


def _keep(*arrays):
    return arrays


def sky_struct(sky):
    keep = []

    def arr(a, dt, minlen=1):
        a = np.ascontiguousarray(a, dtype=dt)
        if a.size == 0:
            a = np.zeros(minlen, dtype=dt)
        keep.append(a)
        return ctypes.c_void_p(a.ctypes.data)

    s = OrSky()
    s.num_components = int(len(sky.ra))
    s.comp_type = arr(sky.comp_type, np.int32)
    s.ra = arr(sky.ra, np.float64)
    s.dec = arr(sky.dec, np.float64)
    s.maj = arr(sky.maj, np.float64)
    s.min = arr(sky.min, np.float64)
    s.pa = arr(sky.pa, np.float64)
    s.flux_type = arr(sky.flux_type, np.int32)
    s.si = arr(sky.si, np.float64)
    s.q = arr(sky.q, np.float64)
    s.fd_start = arr(sky.fd_start, np.int32)
    s.fd_count = arr(sky.fd_count, np.int32)
    s.fds = arr(sky.fds, np.float64, 5)
    s.coeff_start = arr(sky.coeff_start, np.int32)
    s.coeff_count = arr(sky.coeff_count, np.int32)
    s.coeff_n1 = arr(sky.coeff_n1, np.int32)
    s.coeff_n2 = arr(sky.coeff_n2, np.int32)
    s.coeff_value = arr(sky.coeff_value, np.float64)
    return s, keep


def beam_struct(kind=0, beam_jones=(None, None, None), tile_map=None, freq_map=None, num_unique_freqs=0):
    b = OrBeam()
    b.kind = kind
    keep = []
    for t in range(3):
        if beam_jones[t] is not None:
            a = np.ascontiguousarray(beam_jones[t], dtype=np.float64)
            keep.append(a)
            b.beam_jones[t] = a.ctypes.data
        else:
            b.beam_jones[t] = None
    if tile_map is not None:
        tm = np.ascontiguousarray(tile_map, dtype=np.int32)
        keep.append(tm)
        b.tile_map = tm.ctypes.data
    if freq_map is not None:
        fm = np.ascontiguousarray(freq_map, dtype=np.int32)
        keep.append(fm)
        b.freq_map = fm.ctypes.data
    b.num_unique_freqs = num_unique_freqs
    return b, keep


def set_num_threads(n: int) -> None:
    lib().or_set_num_threads(int(n))


def num_threads() -> int:
    return int(lib().or_num_threads())


def shapelet_basis() -> np.ndarray:
    out = np.zeros((SBF_N, SBF_L), np.float64)
    lib().or_shapelet_basis(_ptr(out))
    return out


def inst_flux(sky, freqs) -> np.ndarray:
    s, keep = sky_struct(sky)
    freqs = np.ascontiguousarray(freqs, np.float64)
    out = np.zeros((freqs.size, len(sky.ra), 8), np.float64)
    lib().or_inst_flux(ctypes.byref(s), _ptr(freqs), ctypes.c_int(freqs.size), _ptr(out))
    return out


def lmn_rime(ra, dec, pc_ra, pc_dec):
    out = np.zeros(3)
    lib().or_lmn_rime(ctypes.c_double(ra), ctypes.c_double(dec), ctypes.c_double(pc_ra), ctypes.c_double(pc_dec),
                      _ptr(out))
    return out


def xyzs_to_cross_uvws(xyzs, ha, dec) -> np.ndarray:
    xyzs = np.ascontiguousarray(xyzs, np.float64)
    n = xyzs.shape[0]
    out = np.zeros((n * (n - 1) // 2, 3))
    lib().or_xyzs_to_cross_uvws(_ptr(xyzs), ctypes.c_int(n), ctypes.c_double(ha), ctypes.c_double(dec), _ptr(out))
    return out


def hadec_to_azel(ha, dec, lat):
    az, el = ctypes.c_double(), ctypes.c_double()
    lib().or_hadec_to_azel(ctypes.c_double(ha), ctypes.c_double(dec), ctypes.c_double(lat), ctypes.byref(az),
                           ctypes.byref(el))
    return az.value, el.value


def analytic_beam(az, el, freq) -> np.ndarray:
    out = np.zeros(8)
    lib().or_analytic_beam(ctypes.c_double(az), ctypes.c_double(el), ctypes.c_double(freq), _ptr(out))
    return out


def shapelet_uvws(sky, xyzs, lst) -> np.ndarray:
    s, keep = sky_struct(sky)
    xyzs = np.ascontiguousarray(xyzs, np.float64)
    n = xyzs.shape[0]
    nsh = int(np.sum(np.asarray(sky.comp_type) == 2))
    out = np.zeros((n * (n - 1) // 2, max(nsh, 1), 3))
    lib().or_shapelet_uvws(ctypes.byref(s), _ptr(xyzs), ctypes.c_int(n), ctypes.c_double(lst), _ptr(out))
    return out[:, :nsh]


def model_type(comp_type, sky, xyzs, freqs, pc, lst, lat, uvws, beam=None, out_f64=False, vis=None):
    s, keep = sky_struct(sky)
    xyzs = np.ascontiguousarray(xyzs, np.float64)
    freqs = np.ascontiguousarray(freqs, np.float64)
    uvws = np.ascontiguousarray(uvws, np.float64)
    n = xyzs.shape[0]
    nbl = n * (n - 1) // 2
    if vis is None:
        vis = np.zeros((freqs.size, nbl, 8), np.float64 if out_f64 else np.float32)
    b, kb = beam if beam is not None else beam_struct(0)
    lib().or_model_type(ctypes.c_int(comp_type), ctypes.byref(s), _ptr(xyzs), ctypes.c_int(n), _ptr(freqs),
                        ctypes.c_int(freqs.size), ctypes.c_double(pc[0]), ctypes.c_double(pc[1]), ctypes.c_double(lst),
                        ctypes.c_double(lat), _ptr(uvws), ctypes.byref(b), _ptr(vis), ctypes.c_int(1 if out_f64 else 0))
    return vis


def model_timestep(sky, xyzs, freqs, pc, lst, lat, beam=None, pols=0, out_f64=False, vis=None):
    s, keep = sky_struct(sky)
    xyzs = np.ascontiguousarray(xyzs, np.float64)
    freqs = np.ascontiguousarray(freqs, np.float64)
    n = xyzs.shape[0]
    nbl = n * (n - 1) // 2
    if vis is None:
        vis = np.zeros((freqs.size, nbl, 8), np.float64 if out_f64 else np.float32)
    uvws = np.zeros((nbl, 3))
    b, kb = beam if beam is not None else beam_struct(0)
    lib().or_model_timestep(ctypes.byref(s), _ptr(xyzs), ctypes.c_int(n), _ptr(freqs), ctypes.c_int(freqs.size),
                            ctypes.c_double(pc[0]), ctypes.c_double(pc[1]), ctypes.c_double(lst), ctypes.c_double(lat),
                            ctypes.byref(b), ctypes.c_int(pols), _ptr(vis), ctypes.c_int(1 if out_f64 else 0),
                            _ptr(uvws))
    return vis, uvws


def model_autos(sky, ntiles, freqs, lst, lat, beam=None, vis=None):
    s, keep = sky_struct(sky)
    freqs = np.ascontiguousarray(freqs, np.float64)
    if vis is None:
        vis = np.zeros((freqs.size, ntiles, 8), np.float32)
    b, kb = beam if beam is not None else beam_struct(0)
    lib().or_model_autos(ctypes.byref(s), ctypes.c_int(ntiles), _ptr(freqs), ctypes.c_int(freqs.size),
                         ctypes.c_double(lst), ctypes.c_double(lat), ctypes.byref(b), _ptr(vis))
    return vis


def calibrate(data, model, ch, di_jones, max_iter=50, stop=1e-8, min_thr=1e-4, pols=0):
    """calibrate() on chanblock ``ch`` of data/model [t][chan][bl][8] f32."""
    data = np.ascontiguousarray(data, np.float32)
    model = np.ascontiguousarray(model, np.float32)
    dj = np.ascontiguousarray(di_jones, np.float64).copy()
    nt, nchan, nbl = data.shape[:3]
    r = OrCalResult()
    lib().or_calibrate(_ptr(data), _ptr(model), ctypes.c_int(nt), ctypes.c_int(nchan), ctypes.c_int(ch),
                       ctypes.c_int(nbl), _ptr(dj), ctypes.c_int(max_iter), ctypes.c_double(stop),
                       ctypes.c_double(min_thr), ctypes.c_int(pols), ctypes.byref(r))
    return dj, r


def calibrate_timeblock(data, model, di_jones_tc, t0=None, t1=None, max_iter=50, stop=1e-8, min_thr=1e-4, pols=0):
    """calibrate_timeblock; di_jones_tc is [tile][chanblock][8] f64 (copied)."""
    data = np.ascontiguousarray(data, np.float32)
    model = np.ascontiguousarray(model, np.float32)
    nt, nch, nbl = data.shape[:3]
    t0 = 0 if t0 is None else t0
    t1 = nt if t1 is None else t1
    dj = np.ascontiguousarray(di_jones_tc, np.float64).copy()
    res = (OrCalResult * nch)()
    lib().or_calibrate_timeblock(_ptr(data), _ptr(model), ctypes.c_int(nt), ctypes.c_int(t0), ctypes.c_int(t1),
                                 ctypes.c_int(nch), ctypes.c_int(nbl), _ptr(dj), ctypes.c_int(max_iter),
                                 ctypes.c_double(stop), ctypes.c_double(min_thr), ctypes.c_int(pols), res)
    return dj, [dict(num_iterations=r.num_iterations, converged=bool(r.converged), max_precision=r.max_precision,
                     num_failed=r.num_failed) for r in res]


# ---- peel kernels (reference GPU semantics) ----
def xyzs_to_uvws(xyzs_t, lmsts, pc):
    xyzs_t = np.ascontiguousarray(xyzs_t, np.float64)
    nt, ntiles = xyzs_t.shape[:2]
    nbl = ntiles * (ntiles - 1) // 2
    lmsts = np.ascontiguousarray(lmsts, np.float64)
    out = np.zeros((nt, nbl, 3))
    lib().or_xyzs_to_uvws(_ptr(xyzs_t), _ptr(lmsts), _ptr(out), ctypes.c_double(pc[0]), ctypes.c_double(pc[1]),
                          ctypes.c_int(ntiles), ctypes.c_int(nbl), ctypes.c_int(nt))
    return out


def rotate(vis, uvws_from, uvws_to, lambdas):
    vis = np.ascontiguousarray(vis, np.float32).copy()
    nt, nf, nbl = vis.shape[:3]
    lib().or_rotate(_ptr(vis), ctypes.c_int(nt), ctypes.c_int(nbl), ctypes.c_int(nf),
                    _ptr(np.ascontiguousarray(uvws_from, np.float64)), _ptr(np.ascontiguousarray(uvws_to, np.float64)),
                    _ptr(np.ascontiguousarray(lambdas, np.float64)))
    return vis


def average(hi, w, favg):
    hi = np.ascontiguousarray(hi, np.float32)
    w = np.ascontiguousarray(w, np.float32)
    nt, nf, nbl = hi.shape[:3]
    lo = np.zeros((nf // favg, nbl, 8), np.float32)
    lib().or_average(_ptr(hi), _ptr(w), _ptr(lo), ctypes.c_int(nt), ctypes.c_int(nbl), ctypes.c_int(nf),
                     ctypes.c_int(favg))
    return lo


def scale_by_weights(data, model, weights, baseline_weights=None):
    """CalVis::scale_by_weights on [t][f][bl][8] FP32 arrays (returns copies)."""
    data = np.array(data, np.float32, order="C", copy=True)
    model = np.array(model, np.float32, order="C", copy=True)
    weights = np.ascontiguousarray(weights, np.float32)
    nt, nf, nbl = weights.shape
    blw = None if baseline_weights is None else np.ascontiguousarray(baseline_weights, np.float64)
    lib().or_scale_by_weights(_ptr(data), _ptr(model), _ptr(weights), ctypes.c_int(nt), ctypes.c_int(nf),
                              ctypes.c_int(nbl), _ptr(blw) if blw is not None else None)
    return data, model


def vis_average(vis, weights, num_chanblocks, flagged=()):
    """vis_average over one time chunk: [t][f][bl][8] -> [chanblock][bl][8]
    and weights [chanblock][bl]."""
    vis = np.ascontiguousarray(vis, np.float32)
    weights = np.ascontiguousarray(weights, np.float32)
    nt, nf, nbl = weights.shape
    fl = np.ascontiguousarray(sorted(flagged), np.int32)
    to = np.zeros((num_chanblocks, nbl, 8), np.float32)
    wto = np.zeros((num_chanblocks, nbl), np.float32)
    rc = lib().or_vis_average(_ptr(vis), _ptr(weights), ctypes.c_int(nt), ctypes.c_int(nf), ctypes.c_int(nbl),
                              _ptr(fl) if fl.size else None, ctypes.c_int(fl.size), _ptr(to), _ptr(wto),
                              ctypes.c_int(num_chanblocks))
    if rc:
        raise ValueError("vis_average: the channels do not make that many chunks")
    return to, wto


def into_cal_sols(di_jones, flagged_tiles, flagged_chanblocks, pols=0):
    """into_cal_sols' Jones part: [tb][unflagged tile][unflagged cb][8] ->
    [tb][tile][cb][8] inverted, NaN where flagged."""
    dj = np.ascontiguousarray(di_jones, np.float64)
    ntb, nut, nuc = dj.shape[:3]
    ft = np.ascontiguousarray(flagged_tiles, np.int32)
    fc = np.ascontiguousarray(flagged_chanblocks, np.int32)
    out = np.empty((ntb, nut + ft.size, nuc + fc.size, 8))
    lib().or_into_cal_sols(_ptr(dj), ctypes.c_int(ntb), ctypes.c_int(nut), ctypes.c_int(nuc),
                           _ptr(ft) if ft.size else None, ctypes.c_int(ft.size), _ptr(fc) if fc.size else None,
                           ctypes.c_int(fc.size), ctypes.c_int(pols), _ptr(out))
    return out


def iono_loop(resid, weights, model, consts, niter, uvws, lambdas, convergence):
    resid = np.ascontiguousarray(resid, np.float32)
    weights = np.ascontiguousarray(weights, np.float32)
    model = np.ascontiguousarray(model, np.float32)
    nf, nbl = resid.shape[:2]
    rot = np.zeros_like(model)
    c = OrIono(*consts)
    lib().or_iono_loop(_ptr(resid), _ptr(weights), _ptr(model), _ptr(rot), ctypes.byref(c), ctypes.c_int(nbl),
                       ctypes.c_int(nf), ctypes.c_int(niter), _ptr(np.ascontiguousarray(uvws, np.float64)),
                       _ptr(np.ascontiguousarray(lambdas, np.float64)), ctypes.c_double(convergence))
    return (c.alpha, c.beta, c.gain), rot


def subtract_iono(resid, model, consts, old, uvws, lambdas):
    resid = np.ascontiguousarray(resid, np.float32).copy()
    model = np.ascontiguousarray(model, np.float32)
    nt, nf, nbl = resid.shape[:3]
    lib().or_subtract_iono(_ptr(resid), _ptr(model), OrIono(*consts), OrIono(*old),
                           _ptr(np.ascontiguousarray(uvws, np.float64)), _ptr(np.ascontiguousarray(lambdas, np.float64)),
                           ctypes.c_int(nt), ctypes.c_int(nbl), ctypes.c_int(nf))
    return resid


def add_model(resid, model, consts, lambdas, uvws):
    resid = np.ascontiguousarray(resid, np.float32).copy()
    model = np.ascontiguousarray(model, np.float32)
    nt, nf, nbl = resid.shape[:3]
    lib().or_add_model(_ptr(resid), _ptr(model), OrIono(*consts), _ptr(np.ascontiguousarray(lambdas, np.float64)),
                       _ptr(np.ascontiguousarray(uvws, np.float64)), ctypes.c_int(nt), ctypes.c_int(nf),
                       ctypes.c_int(nbl))
    return resid


def iono_fit(resid, weights, model, lambdas, tile_uvs):
    resid = np.ascontiguousarray(resid, np.float32)
    nt, nf, nbl = resid.shape[:3]
    tile_uvs = np.ascontiguousarray(tile_uvs, np.float64)
    ntiles = tile_uvs.shape[1]
    out = np.zeros(4)
    lib().or_iono_fit(_ptr(resid), _ptr(np.ascontiguousarray(weights, np.float32)),
                      _ptr(np.ascontiguousarray(model, np.float32)), _ptr(np.ascontiguousarray(lambdas, np.float64)),
                      _ptr(tile_uvs), ctypes.c_int(nt), ctypes.c_int(nf), ctypes.c_int(ntiles), _ptr(out))
    return out


def weights_rts(tile_uvs, lambdas, sigma):
    tile_uvs = np.ascontiguousarray(tile_uvs, np.float64)
    nt, ntiles = tile_uvs.shape[:2]
    lambdas = np.ascontiguousarray(lambdas, np.float64)
    out = np.zeros((nt, lambdas.size, ntiles * (ntiles - 1) // 2), np.float32)
    lib().or_weights_rts(_ptr(tile_uvs), ctypes.c_int(nt), ctypes.c_int(ntiles), _ptr(lambdas),
                         ctypes.c_int(lambdas.size), ctypes.c_double(sigma), _ptr(out))
    return out


def peel_cpu(resid, weights, freqs, xyzs, lmsts, average_lmst, pc, sources, positions, consts, num_passes, num_loops,
             convergence, favg, lat):
    """peel_cpu (params/peel/mod.rs:1121-1475) on the CPU: resid [t][f][bl][8]
    float32 is peeled in place (a copy is returned), consts [(alpha, beta,
    gain)] per source are the starting values; returns (resid, consts)."""
    resid = np.ascontiguousarray(resid, np.float32).copy()
    nt, nf, nbl = resid.shape[:3]
    xyzs = np.ascontiguousarray(xyzs, np.float64)
    structs = [sky_struct(s) for s in sources]
    arr = (ctypes.POINTER(OrSky) * len(sources))(*[ctypes.pointer(st) for st, _ in structs])
    pos = np.ascontiguousarray(np.asarray(positions, np.float64).reshape(-1, 2))
    cs = (OrIono * len(sources))(*[OrIono(*c) for c in consts])
    lib().or_peel_cpu(_ptr(resid), _ptr(np.ascontiguousarray(weights, np.float32)), ctypes.c_int(nt), ctypes.c_int(nf),
                      _ptr(np.ascontiguousarray(freqs, np.float64)), _ptr(xyzs), ctypes.c_int(xyzs.shape[0]),
                      _ptr(np.ascontiguousarray(lmsts, np.float64)), ctypes.c_double(average_lmst),
                      ctypes.c_double(pc[0]), ctypes.c_double(pc[1]), ctypes.c_int(len(sources)), arr, _ptr(pos), cs,
                      ctypes.c_int(num_passes), ctypes.c_int(num_loops), ctypes.c_double(convergence),
                      ctypes.c_int(favg), ctypes.c_double(lat))
    return resid, [(c.alpha, c.beta, c.gain) for c in cs]


def tile_beam_table(sky, comp_type, lst, lat, gains, ufreqs):
    """Per-tile analytic beam Jones [uniq][nuf][n_type][8] of the sky's
    components of one type (this project's dipole-gain model)."""
    s, keep = sky_struct(sky)
    gains = np.ascontiguousarray(gains, np.float64).reshape(-1, 32)
    ufreqs = np.ascontiguousarray(ufreqs, np.float64)
    n = int(np.sum(np.asarray(sky.comp_type) == comp_type))
    out = np.zeros((gains.shape[0], ufreqs.size, n, 8))
    lib().or_tile_beam_table(ctypes.byref(s), ctypes.c_int(comp_type), ctypes.c_double(lst), ctypes.c_double(lat),
                             _ptr(gains), ctypes.c_int(gains.shape[0]), _ptr(ufreqs), ctypes.c_int(ufreqs.size),
                             _ptr(out))
    return out


def unique_tile_beams(dipole_gains, freqs, freq_res_hz=1.28e6):
    """The unique tiles (by their 32 dipole gains, first appearance order), the
    unique beam frequencies (nearest multiple of freq_res_hz) and the maps, as
    the native modeller forms them."""
    g = np.asarray(dipole_gains, np.float64).reshape(-1, 32)
    uniq, tile_map = [], np.zeros(g.shape[0], np.int32)
    for p in range(g.shape[0]):
        for u, row in enumerate(uniq):
            if np.array_equal(row, g[p]):
                tile_map[p] = u
                break
        else:
            tile_map[p] = len(uniq)
            uniq.append(g[p])
    bins = np.floor(np.asarray(freqs) / freq_res_hz + 0.5).astype(np.int64)  # as C's llround for positives
    ub = np.unique(bins)
    freq_map = np.searchsorted(ub, bins).astype(np.int32)
    return np.array(uniq), tile_map, ub * freq_res_hz, freq_map
