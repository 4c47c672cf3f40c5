"""Peeling: the host-side mirror of mwa_hyperdrive's peel loop
(params/peel/gpu.rs:25-757 peel_gpu; params/peel/mod.rs:207-224
PeelLoopParams) over libhdc's native peel.

Residual visibilities are ``[timestep][channel][baseline][8]`` float32
(CUDA tensor, peeled in place); weights ``[t][f][bl]`` float32 (>= 0).
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import List, Sequence, Tuple

import numpy as np

from . import _lib
from .model import BEAMS, _as_sky, _stream_ptr


@dataclass
class IonoConsts:
    """params/peel/mod.rs:56-70 (alpha, beta scale lambda^2; gain)."""

    alpha: float = 0.0
    beta: float = 0.0
    gain: float = 1.0


@dataclass
class PeelLoopParams:
    """params/peel/mod.rs:207-224."""

    num_passes: int = 3
    num_loops: int = 10
    convergence: float = 1.0

    def get(self) -> Tuple[int, int, float]:
        return self.num_passes, self.num_loops, self.convergence


def peel_timeblock(d_resid_tfb, d_weights_tfb, freqs, tile_xyzs, lmsts, average_lmst, phase_centre, sources,
                   source_positions, iono_consts: Sequence[IonoConsts], num_passes: int, num_loops: int,
                   convergence: float, freq_average_factor: int, array_latitude_rad: float, beam: str = "none",
                   stream=None, batched: bool = False, batch_size: int = 0, fee_beam=None) -> List[IonoConsts]:
    """Peel ``sources`` (a list of SourceList / Source / SkyModelArrays, one per
    source) with explicit pass and loop counts.  ``batched`` selects
    hdc_peel_timeblock_batched (the sources of a sub-batch fitted together
    against the residual at the start of the sub-batch; sub-batches of
    ``batch_size`` sources in list order, 0 for all in one) instead of the
    reference's source-by-source order.  ``beam`` "fee" models the sources
    with ``fee_beam`` (a :class:`mwa_hyperdrive_b200.fee.FeeBeam` prepared
    for these tiles and channels), as the reference's peel uses its beam."""
    nt, nf, nbl = (int(x) for x in d_resid_tfb.shape[:3])
    freqs = np.ascontiguousarray(freqs, np.float64)
    xyzs = np.ascontiguousarray(tile_xyzs, np.float64).reshape(-1, 3)
    lmsts = np.ascontiguousarray(lmsts, np.float64)
    skies = [_as_sky(s) for s in sources]
    n = len(skies)
    from .srclist import HdcSkyModel

    structs = (HdcSkyModel * max(n, 1))()
    for i, sk in enumerate(skies):
        structs[i] = sk.struct()
    pos = (_lib.RADec * max(n, 1))(*[_lib.RADec(*p) for p in source_positions])
    consts = (_lib.IonoConsts * max(n, 1))(*[_lib.IonoConsts(c.alpha, c.beta, c.gain) for c in iono_consts])
    if beam == "fee" and fee_beam is None:
        raise ValueError('beam "fee" needs fee_beam')
    params = _lib.HdcPeelParams(int(num_passes), int(num_loops), float(convergence), int(freq_average_factor),
                                BEAMS[beam], float(array_latitude_rad), int(batch_size),
                                fee_beam.handle if beam == "fee" else None)
    fn = _lib.lib().hdc_peel_timeblock_batched if batched else _lib.lib().hdc_peel_timeblock
    rc = fn(d_resid_tfb.data_ptr(), d_weights_tfb.data_ptr(), nt, nf, freqs.ctypes.data, xyzs.ctypes.data,
            xyzs.shape[0], lmsts.ctypes.data, float(average_lmst), _lib.RADec(*phase_centre), n,
            ctypes.addressof(structs), ctypes.addressof(pos), ctypes.addressof(consts), ctypes.byref(params),
            _stream_ptr(stream))
    _lib.check(rc, "hdc_peel_timeblock_batched" if batched else "hdc_peel_timeblock")
    return [IonoConsts(consts[i].alpha, consts[i].beta, consts[i].gain) for i in range(n)]


def peel_gpu(d_resid_tfb, d_weights_tfb, freqs, tile_xyzs, lmsts, average_lmst, phase_centre, sources,
             source_positions, iono_consts, peel_loop_params: PeelLoopParams, freq_average_factor: int,
             array_latitude_rad: float, beam: str = "none", stream=None) -> List[IonoConsts]:
    """peel_gpu as the reference calls it: it destructures
    PeelLoopParams::get() as (num_loops, num_passes, convergence)
    (params/peel/gpu.rs:41) although get() returns (passes, loops, conv), so
    the configured pass count becomes the iono-loop count and vice versa.
    This wrapper reproduces that behaviour; call peel_timeblock for the
    intended meaning."""
    num_loops, num_passes, convergence = peel_loop_params.get()
    return peel_timeblock(d_resid_tfb, d_weights_tfb, freqs, tile_xyzs, lmsts, average_lmst, phase_centre, sources,
                          source_positions, iono_consts, num_passes, num_loops, convergence, freq_average_factor,
                          array_latitude_rad, beam, stream)


def batched_tuning():
    """(bins per CTA, sources per CTA, ms) the batched peel's autotuner chose
    for the last new problem shape; (16, 0) is the variant that stages the
    residual of 16 baselines in shared memory for every source."""
    bx, sy, ms = ctypes.c_int(), ctypes.c_int(), ctypes.c_float()
    _lib.check(_lib.lib().hdc_peel_batched_tuning(ctypes.byref(bx), ctypes.byref(sy), ctypes.byref(ms)),
               "hdc_peel_batched_tuning")
    return bx.value, sy.value, ms.value
