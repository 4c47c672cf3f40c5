"""Direction-independent calibration: the host-side mirror of
mwa_hyperdrive's calibrate_timeblocks / calibrate_timeblock
(di_calibrate/mod.rs:272-618) over libhdc's GPU solver, and the two steps
that prepare its inputs: vis_average (averaging/mod.rs:537-648) and
CalVis::scale_by_weights (params/di_calibration.rs:578-625).

Visibilities are ``[timestep][chanblock][baseline][8]`` float32 (torch CUDA
tensors for the device entry point, numpy arrays for the host-buffer
convenience); solutions follow the reference's layout
``di_jones[timeblock][tile][chanblock][8]`` float64, holding the model->data
gains (not inverted) with NaN where calibration failed.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import List, Sequence, Tuple

import numpy as np

from . import _lib
from .model import POLS, _stream_ptr

FORMS = {"plain": 0, "collapsed": 1, "collapsed_f32": 2}


@dataclass
class CalibrationResult:
    """di_calibrate/mod.rs:620-632"""

    num_iterations: int
    converged: bool
    max_precision: float
    num_failed: int
    chanblock: int = -1


def num_tiles_from_baselines(nbl: int) -> int:
    n = int(round((1 + (1 + 8 * nbl) ** 0.5) / 2))
    if n * (n - 1) // 2 != nbl:
        raise ValueError(f"{nbl} is not a triangular number of baselines")
    return n


def calibrate_timeblock(d_data, d_model, d_di_jones_tc, timeblock: Tuple[int, int], max_iterations: int = 50,
                        stop_threshold: float = 1e-8, min_threshold: float = 1e-4, pols: str = "XX_XY_YX_YY",
                        form: str = "plain", stream=None) -> List[CalibrationResult]:
    """Calibrate one timeblock on the device.  ``d_di_jones_tc`` is a CUDA
    float64 tensor [tile][chanblock][8] holding the initial guesses; it is
    overwritten with the solutions."""
    nt, nch, nbl = int(d_data.shape[0]), int(d_data.shape[1]), int(d_data.shape[2])
    res = (_lib.HdcCalResult * nch)()
    rc = _lib.lib().hdc_calibrate_timeblock(d_data.data_ptr(), d_model.data_ptr(), nt, int(timeblock[0]),
                                            int(timeblock[1]), nch, nbl, d_di_jones_tc.data_ptr(),
                                            int(max_iterations), float(stop_threshold), float(min_threshold),
                                            POLS[pols], res, FORMS[form], _stream_ptr(stream))
    _lib.check(rc, "hdc_calibrate_timeblock")
    return [CalibrationResult(r.num_iterations, bool(r.converged), r.max_precision, r.num_failed, i)
            for i, r in enumerate(res)]


def calibrate_timeblocks(vis_data_tfb, vis_model_tfb, timeblocks: Sequence[Tuple[int, int]],
                         max_iterations: int = 50, stop_threshold: float = 1e-8, min_threshold: float = 1e-4,
                         pols: str = "XX_XY_YX_YY", form: str = "plain", stream=None):
    """calibrate_timeblocks (di_calibrate/mod.rs:272-361) through
    hdc_calibrate_timeblocks: the first pass of every timeblock runs as one
    CUDA graph, failed chanblocks are retried per timeblock.  Accepts host
    (numpy) or device (torch) visibilities; returns (di_jones
    [timeblock][tile][chanblock][8] numpy, results [timeblock][chanblock])."""
    import torch

    host = isinstance(vis_data_tfb, np.ndarray)
    d_data = torch.from_numpy(np.ascontiguousarray(vis_data_tfb, np.float32)).cuda() if host else vis_data_tfb
    d_model = torch.from_numpy(np.ascontiguousarray(vis_model_tfb, np.float32)).cuda() if host else vis_model_tfb
    nt, nch, nbl = (int(x) for x in d_data.shape[:3])
    ntiles = num_tiles_from_baselines(nbl)
    ntb = len(timeblocks)
    dj = torch.empty((ntb, ntiles, nch, 8), dtype=torch.float64, device=d_data.device)
    bounds = np.ascontiguousarray(np.array(timeblocks, dtype=np.int32).reshape(-1))
    res = (_lib.HdcCalResult * (ntb * nch))()
    rc = _lib.lib().hdc_calibrate_timeblocks(d_data.data_ptr(), d_model.data_ptr(), nt, bounds.ctypes.data, ntb, nch,
                                             nbl, dj.data_ptr(), int(max_iterations), float(stop_threshold),
                                             float(min_threshold), POLS[pols], res, FORMS[form], _stream_ptr(stream))
    _lib.check(rc, "hdc_calibrate_timeblocks")
    results = [[CalibrationResult(r.num_iterations, bool(r.converged), r.max_precision, r.num_failed, i)
                for i, r in enumerate(res[k * nch:(k + 1) * nch])] for k in range(ntb)]
    return dj.cpu().numpy(), results


def scale_by_weights(d_data, d_model, d_weights, baseline_weights=None, stream=None) -> None:
    """CalVis::scale_by_weights (params/di_calibration.rs:578-625), in place on
    CUDA tensors: data and model [timestep][chanblock][baseline][8] float32
    times weight [timestep][chanblock][baseline] float32 x baseline weight
    (float64 per baseline, or None), zero where that product is <= 0."""
    import torch

    nt, nch, nbl = (int(x) for x in d_weights.shape)
    if d_weights.dtype != torch.float32 or not d_weights.is_contiguous():
        raise ValueError("scale_by_weights: weights must be contiguous float32 [t][chanblock][bl]")
    for t in (d_data, d_model):
        if tuple(t.shape) != (nt, nch, nbl, 8) or t.dtype != torch.float32 or not t.is_contiguous():
            raise ValueError("scale_by_weights: data and model must be contiguous float32 [t][chanblock][bl][8]")
    bw = None
    if baseline_weights is not None:
        bw = torch.as_tensor(baseline_weights, dtype=torch.float64).to(d_data.device).contiguous()
        if bw.numel() != nbl:
            raise ValueError(f"scale_by_weights: {bw.numel()} baseline weights for {nbl} baselines")
    rc = _lib.lib().hdc_scale_by_weights(d_data.data_ptr(), d_model.data_ptr(), d_weights.data_ptr(), nt, nch, nbl,
                                         bw.data_ptr() if bw is not None else None, _stream_ptr(stream))
    _lib.check(rc, "hdc_scale_by_weights")


def vis_average(d_vis_tfb, d_weights_tfb, num_chanblocks: int, flagged_chanblocks=(), stream=None):
    """vis_average (averaging/mod.rs:537-600) of one time chunk on the device:
    [timestep][freq][baseline][8] float32 visibilities and their weights into
    ([chanblock][baseline][8], [chanblock][baseline]) CUDA tensors; the
    flagged chanblock indices (of num_chanblocks + len(flagged) chunks) are
    skipped."""
    import torch

    nt, nf, nbl = (int(x) for x in d_weights_tfb.shape)
    if tuple(d_vis_tfb.shape) != (nt, nf, nbl, 8) or d_vis_tfb.dtype != torch.float32 or \
            d_weights_tfb.dtype != torch.float32 or not d_vis_tfb.is_contiguous() or not d_weights_tfb.is_contiguous():
        raise ValueError("vis_average: visibilities must be contiguous float32 [t][freq][bl][8] with matching weights")
    fl = np.ascontiguousarray(sorted(int(c) for c in flagged_chanblocks), np.int32)
    to = torch.empty((int(num_chanblocks), nbl, 8), dtype=torch.float32, device=d_vis_tfb.device)
    wto = torch.empty((int(num_chanblocks), nbl), dtype=torch.float32, device=d_vis_tfb.device)
    rc = _lib.lib().hdc_vis_average(d_vis_tfb.data_ptr(), d_weights_tfb.data_ptr(), nt, nf, nbl,
                                    fl.ctypes.data if fl.size else None, int(fl.size), to.data_ptr(), wto.data_ptr(),
                                    int(num_chanblocks), _stream_ptr(stream))
    _lib.check(rc, "hdc_vis_average")
    return to, wto
