"""Spreading the predict and DI calibration over several GPUs, one process
per GPU (torch.distributed; NCCL between GPUs, gloo on CPU ranks).

Both paths shard with no exchange in their hot loops:

* Predict: channels are independent, so each rank predicts a contiguous
  range of channels with its own modeller (component tables replicated) and
  the visibilities are gathered once (`gather_channels`).
* DI calibration: chanblocks are independent, except for the reference's
  retry of failed chanblocks (di_calibrate/mod.rs:473-614), which seeds a run
  of failures from the converged chanblocks on either side -- possibly on
  another rank.  `calibrate_timeblock_sharded` runs each rank's first pass
  (`hdc_calibrate_chanblocks`), then repeats: gather every chanblock's
  convergence flag and solutions (6 MB for 128 tiles x 768 chanblocks),
  form the reference's seeds over the whole band on every rank (the same
  arithmetic everywhere), and re-run each rank's own failed chanblocks from
  them -- until no new chanblock converges.  Since every chanblock's solve
  depends only on its own data and start, the result is the single-GPU
  `calibrate_timeblock`'s exactly.

The solver is a parameter (`chanblock_solver`), so the exchange logic is
tested on CPU ranks with the CPU oracle as the solver
(tests/test_multi_rank.py).
"""

from __future__ import annotations

from typing import Callable, List, Optional, Sequence, Tuple

import numpy as np


def ranges(n: int, world: int) -> List[Tuple[int, int]]:
    """Contiguous near-equal ranges [lo, hi) of n items over world ranks
    (the first n % world ranks take one more)."""
    base, extra = divmod(n, world)
    out, lo = [], 0
    for r in range(world):
        hi = lo + base + (1 if r < extra else 0)
        out.append((lo, hi))
        lo = hi
    return out


def _all_gather(obj, group=None):
    import torch.distributed as dist

    out = [None] * dist.get_world_size(group)
    dist.all_gather_object(out, obj, group=group)
    return out


def gather_channels(local: np.ndarray, axis: int = 0, group=None) -> np.ndarray:
    """Concatenate every rank's channel range (in rank order) along `axis`:
    the predict's one exchange, at the end."""
    return np.concatenate(_all_gather(np.ascontiguousarray(local), group), axis=axis)


def retry_pairs(converged: Sequence[bool]) -> List[Tuple[int, int]]:
    """The reference's (left, right) converged neighbours around each run of
    failed chanblocks (mod.rs:487-504); left -1 for a leading run.  A
    trailing run has no pair and keeps its start."""
    pairs, left, in_fail = [], -1, False
    for c, ok in enumerate(converged):
        if not in_fail and ok:
            left = c
        elif not in_fail and not ok:
            in_fail = True
        elif in_fail and ok:
            in_fail = False
            pairs.append((left, c))
            left = c
    return pairs


def seed(sols_ct: np.ndarray, pairs: Sequence[Tuple[int, int]]) -> np.ndarray:
    """Starting gains of failed chanblocks from their converged neighbours
    (mod.rs:506-530): the distance-weighted mean of the pair, or the right
    one for a leading run.  sols_ct [chanblock][tile][8]; returns a copy."""
    out = sols_ct.copy()
    for l, r in pairs:
        rs = sols_ct[r]
        if l >= 0:
            ls = sols_ct[l]
            for i in range(l + 1, r):
                out[i] = (ls * (r - i) + rs * (i - l)) / (r - l)
        else:
            out[:r] = rs
    return out


ChanblockSolver = Callable[[Optional[List[int]], np.ndarray], Tuple[np.ndarray, List[dict]]]


def calibrate_timeblock_sharded(solver: ChanblockSolver, start_tc: np.ndarray, c0: int, nch_total: int,
                                group=None) -> Tuple[np.ndarray, List[dict]]:
    """calibrate_timeblock over chanblocks spread across ranks.

    solver(list, starts_tc) calibrates this rank's chanblocks (all when list
    is None, else the listed local indices) from starts_tc [tile][local
    chanblock][8] and returns (solutions [tile][local chanblock][8], results
    per local chanblock as dicts with at least "converged", only the listed
    entries meaningful).  start_tc: this rank's starting gains; c0: its first
    chanblock; nch_total: the band's chanblocks.  Returns this rank's
    solutions and results after the band-wide retry."""
    nloc = start_tc.shape[1]
    sols, res = solver(None, start_tc)
    res = list(res)
    while True:
        parts = _all_gather((c0, [bool(r["converged"]) for r in res], sols), group)
        conv = np.zeros(nch_total, bool)
        band = np.full((nch_total,) + sols.shape[:1] + sols.shape[2:], np.nan)
        for lo, flags, s in parts:
            conv[lo:lo + len(flags)] = flags
            band[lo:lo + len(flags)] = np.moveaxis(s, 1, 0)
        total = int(conv.sum())
        if total == 0 or total == nch_total:
            break
        seeded = seed(band, retry_pairs(conv))
        mine = [c - c0 for c in range(c0, c0 + nloc) if not conv[c]]
        starts = sols.copy()
        for k in mine:
            starts[:, k] = seeded[c0 + k]
        new_sols, new_res = solver(mine, starts) if mine else (sols, res)
        for k in mine:
            sols[:, k] = new_sols[:, k]
            res[k] = new_res[k]
        after = _all_gather(sum(bool(r["converged"]) for r in res), group)
        if sum(after) == total:
            break
    return sols, res


def gpu_chanblock_solver(d_data, d_model, timeblock, max_iterations=50, stop_threshold=1e-8, min_threshold=1e-4,
                         pols: str = "XX_XY_YX_YY", form: str = "collapsed_f32", stream=None) -> ChanblockSolver:
    """The chanblock solver of one GPU: hdc_calibrate_chanblocks on this
    rank's data and model [t][local chanblock][bl][8] (CUDA tensors)."""
    import ctypes

    import torch

    from . import _lib
    from .calibrate import FORMS
    from .model import POLS, _stream_ptr

    nt, nch, nbl = (int(x) for x in d_data.shape[:3])

    def solve(chanblocks, starts_tc):
        dj = torch.from_numpy(np.ascontiguousarray(starts_tc, np.float64)).to(d_data.device)
        res = (_lib.HdcCalResult * nch)()
        lst = None if chanblocks is None else (ctypes.c_int * max(len(chanblocks), 1))(*chanblocks)
        rc = _lib.lib().hdc_calibrate_chanblocks(d_data.data_ptr(), d_model.data_ptr(), nt, int(timeblock[0]),
                                                 int(timeblock[1]), nch, nbl, dj.data_ptr(), int(max_iterations),
                                                 float(stop_threshold), float(min_threshold), POLS[pols], lst,
                                                 0 if chanblocks is None else len(chanblocks), res, FORMS[form],
                                                 _stream_ptr(stream))
        _lib.check(rc, "hdc_calibrate_chanblocks")
        out = [{"converged": bool(r.converged), "num_iterations": r.num_iterations, "max_precision": r.max_precision,
                "num_failed": r.num_failed} for r in res]
        return dj.cpu().numpy(), out

    return solve
