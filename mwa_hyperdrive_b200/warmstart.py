"""Learned warm start for DI calibration (this project's addition; the
reference's solver always starts each timeblock from identity,
di_calibrate/mod.rs:283-287).

A small MLP (trained and evaluated by libhdc's own FP32 CUDA kernels) maps,
for each (tile, chanblock), the previous timeblock's solutions at chanblocks
c-2 .. c+2 (5 Jones = 40 reals) to a proposed gain for the current
timeblock.  The solver judges every chanblock's proposal by its calibration
residual and falls back to the identity start wherever the proposal's
residual is worse, then refines with the unchanged MitchCal iteration.

Frames.  DI solutions are defined up to one unit-modulus phase per chanblock
(G -> e^{i phi} G leaves G M G^H unchanged); solutions are first aligned so
that the reference tile's XX gain is real and positive.  Each tile's absolute
X and Y phases are arbitrary (uniform over the circle), which no small
network learns to rotate; so features and targets are expressed in the frame
of the previous centre gain: every Jones is right-multiplied by
diag(1/a, 1/d), a and d the previous centre's XX and YY, which leaves the
centre's diagonal at 1 and turns neighbours into gain ratios.  The network
predicts a correction to the centre input (its output layer starts at zero,
so the untrained net proposes the previous solution), and the proposal is
mapped back by diag(a, d).  Neighbours beyond the band edge continue the line
through the centre and the mirrored in-band neighbour (2 N_0 - N_-j), so an
edge chanblock still sees its phase slope.
"""

from __future__ import annotations

import ctypes
import hashlib
import struct
import time
from dataclasses import dataclass
from pathlib import Path
from typing import List, Optional, Sequence, Tuple

import numpy as np

from . import _lib
from . import calibrate as cal
from .model import _stream_ptr

NEIGHBOURS = 2          # chanblocks on each side
IN_DIM = 8 * (2 * NEIGHBOURS + 1)
OUT_DIM = 8
CENTRE = 8 * NEIGHBOURS


def gauge_align(sol_tc: np.ndarray, ref_tile: int = 0) -> np.ndarray:
    """Rotate each chanblock's solutions by one phase so that the reference
    tile's XX gain is real and positive (NaN chanblocks stay NaN)."""
    s = np.array(sol_tc, np.float64, copy=True)
    xx = s[ref_tile, :, 0] + 1j * s[ref_tile, :, 1]
    with np.errstate(invalid="ignore"):  # NaN chanblocks stay NaN
        ph = np.where(np.abs(xx) > 0, np.conj(xx) / np.maximum(np.abs(xx), 1e-300), 1.0 + 0j)
    c = s[..., 0::2] + 1j * s[..., 1::2]
    c = c * ph[None, :, None]
    s[..., 0::2] = c.real
    s[..., 1::2] = c.imag
    return s


def _frame(p_aligned: np.ndarray) -> Tuple[np.ndarray, np.ndarray]:
    """Complex XX and YY of each (tile, chanblock), 1 where unusable."""
    a = p_aligned[..., 0] + 1j * p_aligned[..., 1]
    d = p_aligned[..., 6] + 1j * p_aligned[..., 7]
    ok = np.isfinite(a) & np.isfinite(d) & (np.abs(a) > 1e-6) & (np.abs(d) > 1e-6)
    return np.where(ok, a, 1.0 + 0j), np.where(ok, d, 1.0 + 0j)


def _scale_columns(p: np.ndarray, ca: np.ndarray, cd: np.ndarray) -> np.ndarray:
    """J diag(ca, cd) for Jones [.., 8] = [xx, xy, yx, yy] (re, im)."""
    c = p[..., 0::2] + 1j * p[..., 1::2]
    c[..., 0] *= ca
    c[..., 2] *= ca
    c[..., 1] *= cd
    c[..., 3] *= cd
    out = np.empty(p.shape)
    out[..., 0::2] = c.real
    out[..., 1::2] = c.imag
    return out


def _aligned(prev_tc: np.ndarray) -> np.ndarray:
    p = gauge_align(prev_tc)
    bad = ~np.isfinite(p).all(axis=-1)
    p[bad] = [1, 0, 0, 0, 0, 0, 1, 0]
    return p


def features(prev_tc: np.ndarray) -> np.ndarray:
    """[tile][chanblock][8] previous solutions -> [tile*chanblock][40] float32
    in the frame of each previous centre gain (NaN solutions replaced by the
    identity; out-of-band neighbours extrapolated through the centre)."""
    p = _aligned(prev_tc)
    nt, nc = p.shape[:2]
    a, d = _frame(p)
    ia, id_ = (1.0 / a)[:, :, None], (1.0 / d)[:, :, None]
    chans = np.arange(nc)[:, None]
    raw = chans + np.arange(-NEIGHBOURS, NEIGHBOURS + 1)[None, :]
    n = _scale_columns(p[:, np.clip(raw, 0, nc - 1), :], ia, id_)
    mirror = _scale_columns(p[:, np.clip(2 * chans - raw, 0, nc - 1), :], ia, id_)
    outside = ((raw < 0) | (raw >= nc))[None, :, :, None]
    n = np.where(outside, 2.0 * n[:, :, NEIGHBOURS:NEIGHBOURS + 1, :] - mirror, n)
    return np.ascontiguousarray(n.reshape(nt * nc, IN_DIM), np.float32)


def targets(prev_tc: np.ndarray, cur_tc: np.ndarray) -> np.ndarray:
    """The current timeblock's aligned solutions in the frame of the previous
    centre gains: [tile*chanblock][8] float32 training targets."""
    a, d = _frame(_aligned(prev_tc))
    t = _scale_columns(gauge_align(cur_tc), 1.0 / a, 1.0 / d)
    return np.ascontiguousarray(t.reshape(-1, OUT_DIM), np.float32)


class WarmStartMLP:
    """40 -> 256 -> 256 -> 256 -> 8 ReLU MLP with a residual on the centre
    input (hdc_mlp_*)."""

    def __init__(self, hidden: int = 256, num_hidden: int = 3, seed: int = 0):
        self.dims = [IN_DIM] + [hidden] * num_hidden + [OUT_DIM]
        d = (ctypes.c_int * len(self.dims))(*self.dims)
        h = ctypes.c_void_p()
        _lib.check(_lib.lib().hdc_mlp_new(len(self.dims) - 1, d, CENTRE, seed, ctypes.byref(h)), "hdc_mlp_new")
        self._h = h
        self.losses: List[float] = []

    def close(self):
        if getattr(self, "_h", None):
            _lib.lib().hdc_mlp_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def num_params(self) -> int:
        return int(_lib.lib().hdc_mlp_num_params(self._h))

    def get_params(self) -> np.ndarray:
        out = np.zeros(self.num_params, np.float32)
        _lib.check(_lib.lib().hdc_mlp_get_params(self._h, out.ctypes.data), "hdc_mlp_get_params")
        return out

    def set_params(self, p: np.ndarray) -> None:
        p = np.ascontiguousarray(p, np.float32)
        assert p.size == self.num_params
        _lib.check(_lib.lib().hdc_mlp_set_params(self._h, p.ctypes.data), "hdc_mlp_set_params")

    def forward_device(self, d_x, d_y, stream=None):
        _lib.check(_lib.lib().hdc_mlp_forward(self._h, d_x.data_ptr(), int(d_x.shape[0]), d_y.data_ptr(),
                                              _stream_ptr(stream)), "hdc_mlp_forward")

    def gradients(self, d_x, d_t, stream=None):
        g = np.zeros(self.num_params, np.float32)
        loss = ctypes.c_double()
        _lib.check(_lib.lib().hdc_mlp_gradients(self._h, d_x.data_ptr(), d_t.data_ptr(), int(d_x.shape[0]),
                                                g.ctypes.data, ctypes.byref(loss), _stream_ptr(stream)),
                   "hdc_mlp_gradients")
        return loss.value, g

    def train(self, X, Y, epochs: int = 20, batch: int = 4096, lr: float = 1e-3,
              seed: int = 0, schedule: str = "cosine") -> List[float]:
        """Mini-batch Adam on the device (X [n][40], Y [n][8]: numpy arrays,
        moved to HBM once, or CUDA tensors).  The
        learning rate follows a cosine from lr down to lr/100 over the run
        ("cosine") or stays at lr ("constant"); the decay makes the final fit
        insensitive to the seed and to rounding differences between runs."""
        import torch

        def dev(a):
            if isinstance(a, torch.Tensor):
                return a.to(device="cuda", dtype=torch.float32).contiguous()
            return torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()

        d_x, d_y = dev(X), dev(Y)
        n = X.shape[0]
        rng = np.random.default_rng(seed)
        lib = _lib.lib()
        loss = ctypes.c_double()
        total = max(epochs * (n // batch), 1)
        step = 0
        for ep in range(epochs):
            perm = torch.from_numpy(rng.permutation(n)).cuda()
            xs, ys = d_x[perm], d_y[perm]
            tot, cnt = 0.0, 0
            for b0 in range(0, n - batch + 1, batch):
                rate = lr
                if schedule == "cosine":
                    rate = lr * (0.01 + 0.99 * 0.5 * (1.0 + np.cos(np.pi * step / total)))
                bx = xs[b0:b0 + batch].contiguous()
                by = ys[b0:b0 + batch].contiguous()
                _lib.check(lib.hdc_mlp_train_step(self._h, bx.data_ptr(), by.data_ptr(), batch, float(rate),
                                                  ctypes.byref(loss), _stream_ptr(None)), "hdc_mlp_train_step")
                tot += loss.value
                cnt += 1
                step += 1
            self.losses.append(tot / max(cnt, 1))
        return self.losses

    def propose_device(self, d_prev, d_data=None, d_model=None, timeblock=None, stream=None):
        """The device chain (hdc_warmstart_propose): previous solutions on the
        device ([tile][chanblock][8] float64) -> proposed starting gains on the
        device; with the timeblock's data and model also the judge.  Returns
        (d_start, d_use): d_use [chanblock] int32 (1 = proposal kept), None
        without a judge.  Nothing is synchronised with the host."""
        import torch

        d_prev = d_prev.contiguous()
        nt, nc = int(d_prev.shape[0]), int(d_prev.shape[1])
        d_start = torch.empty((nt, nc, 8), dtype=torch.float64, device=d_prev.device)
        if d_data is None:
            _lib.check(_lib.lib().hdc_warmstart_propose(self._h, d_prev.data_ptr(), nt, nc, None, None, 0, 0, 0,
                                                        d_start.data_ptr(), None, _stream_ptr(stream)),
                       "hdc_warmstart_propose")
            return d_start, None
        d_use = torch.empty(nc, dtype=torch.int32, device=d_prev.device)
        _lib.check(_lib.lib().hdc_warmstart_propose(self._h, d_prev.data_ptr(), nt, nc, d_data.data_ptr(),
                                                    d_model.data_ptr(), int(d_data.shape[0]), int(timeblock[0]),
                                                    int(timeblock[1]), d_start.data_ptr(), d_use.data_ptr(),
                                                    _stream_ptr(stream)), "hdc_warmstart_propose")
        return d_start, d_use

    def propose(self, prev_tc: np.ndarray) -> np.ndarray:
        """Host restatement of the proposal (numpy features and frames around
        the device network): gains [tile][chanblock][8] in the gauge of the
        aligned input."""
        import torch

        nt, nc = prev_tc.shape[:2]
        x = torch.from_numpy(features(prev_tc)).cuda()
        y = torch.empty((x.shape[0], OUT_DIM), dtype=torch.float32, device="cuda")
        self.forward_device(x, y)
        torch.cuda.synchronize()
        a, d = _frame(_aligned(prev_tc))
        return _scale_columns(y.cpu().numpy().astype(np.float64).reshape(nt, nc, OUT_DIM), a, d)

    # ---------------------------------------------- persistence
    MAGIC = b"HDCMLP01"

    def save(self, path) -> None:
        """Weights file: magic, layer count, dims, float32 parameters, SHA-256."""
        p = self.get_params()
        body = struct.pack("<I", len(self.dims)) + struct.pack(f"<{len(self.dims)}I", *self.dims) + p.tobytes()
        Path(path).write_bytes(self.MAGIC + body + hashlib.sha256(body).digest())

    @classmethod
    def load(cls, path) -> "WarmStartMLP":
        raw = Path(path).read_bytes()
        if raw[:8] != cls.MAGIC:
            raise ValueError("not a warm-start MLP weights file")
        body, digest = raw[8:-32], raw[-32:]
        if hashlib.sha256(body).digest() != digest:
            raise ValueError("weights file checksum mismatch")
        (nl,) = struct.unpack("<I", body[:4])
        dims = list(struct.unpack(f"<{nl}I", body[4:4 + 4 * nl]))
        m = cls(hidden=dims[1], num_hidden=nl - 2)
        if m.dims != dims:
            raise ValueError(f"unsupported layer widths {dims}")
        m.set_params(np.frombuffer(body[4 + 4 * nl:], np.float32))
        return m


def features_device(d_prev, stream=None):
    """features() on the device (hdc_warmstart_features): [tile][chanblock][8]
    float64 CUDA tensor -> [tile*chanblock][40] float32 CUDA tensor."""
    import torch

    d_prev = d_prev.contiguous()
    nt, nc = int(d_prev.shape[0]), int(d_prev.shape[1])
    x = torch.empty((nt * nc, IN_DIM), dtype=torch.float32, device=d_prev.device)
    _lib.check(_lib.lib().hdc_warmstart_features(d_prev.data_ptr(), nt, nc, x.data_ptr(), _stream_ptr(stream)),
               "hdc_warmstart_features")
    return x


def identity_gains(ntiles: int, nch: int) -> np.ndarray:
    g = np.zeros((ntiles, nch, 8))
    g[..., 0] = 1.0
    g[..., 6] = 1.0
    return g


def judge(d_data, d_model, timeblock, proposal_tc: np.ndarray) -> Tuple[np.ndarray, np.ndarray]:
    """Per chanblock, keep the proposal where its calibration residual is no
    worse than the identity start's (hdc_warmstart_judge, on the device);
    non-finite proposal entries are first replaced by the identity's.
    Returns (start gains, chose_proposal) on the host."""
    import torch

    nt, nch, nbl = (int(x) for x in d_data.shape[:3])
    ntiles = proposal_tc.shape[0]
    ident = identity_gains(ntiles, nch)
    prop = torch.from_numpy(np.ascontiguousarray(np.where(np.isfinite(proposal_tc), proposal_tc, ident),
                                                 np.float64)).cuda()
    start = torch.empty_like(prop)
    use = torch.empty(nch, dtype=torch.int32, device=prop.device)
    _lib.check(_lib.lib().hdc_warmstart_judge(d_data.data_ptr(), d_model.data_ptr(), nt, int(timeblock[0]),
                                              int(timeblock[1]), nch, ntiles, prop.data_ptr(), start.data_ptr(),
                                              use.data_ptr(), _stream_ptr(None)), "hdc_warmstart_judge")
    return start.cpu().numpy(), use.cpu().numpy().astype(bool)


def calibrate_warm(d_data, d_model, timeblock, d_prev, mlp: Optional[WarmStartMLP], max_iterations=50,
                   stop_threshold=1e-8, min_threshold=1e-4):
    """Calibrate one timeblock on the device from the MLP's judged proposal,
    or from identity where there is no previous solution or no network.
    d_prev: the previous timeblock's solutions on the device ([tile]
    [chanblock][8] float64 tensor) or None.  Returns (d_solutions, results,
    d_use, seconds): the solutions stay on the device for the next
    timeblock; seconds is the wall time of proposal, judge and solve."""
    import torch

    nt, nch, nbl = (int(x) for x in d_data.shape[:3])
    ntiles = cal.num_tiles_from_baselines(nbl)
    t0 = time.perf_counter()
    d_use = None
    if d_prev is None or mlp is None:
        dj = torch.zeros((ntiles, nch, 8), dtype=torch.float64, device=d_data.device)
        dj[..., 0] = 1.0
        dj[..., 6] = 1.0
    else:
        dj, d_use = mlp.propose_device(d_prev, d_data, d_model, timeblock)
    res = cal.calibrate_timeblock(d_data, d_model, dj, timeblock, max_iterations, stop_threshold, min_threshold)
    torch.cuda.synchronize()
    return dj, res, d_use, time.perf_counter() - t0


@dataclass
class DriftSky:
    """Seeded synthetic calibration sequence: per-tile gains with a phase slope
    in frequency and a phase that drifts between timeblocks in proportion to
    the slope (a drifting delay), plus small amplitude jitter, over a
    polarised random model (synth.polarised_model)."""

    ntiles: int
    nch: int
    nt_per_block: int
    nblocks: int
    seed: int
    slope_rad_per_mhz: float = 0.5
    chan_mhz: float = 0.04
    drift_per_block: float = 0.15
    snr: Optional[float] = None
    cross_pol: float = 0.3
    amp_jitter: float = 0.0005

    def generate(self, device: bool = False):
        """[(data, model, gains)] per timeblock: numpy arrays, or with
        ``device`` data and model as CUDA tensors drawn on the device (same
        distributions, another random stream; no noise) and gains in numpy."""
        from . import synth

        rng = np.random.default_rng(self.seed)
        gen = None
        if device:
            import torch

            gen = torch.Generator(device="cuda")
            gen.manual_seed(self.seed)
            if self.snr is not None:
                raise ValueError("device generation has no noise")
        nbl = self.ntiles * (self.ntiles - 1) // 2
        f = np.arange(self.nch) * self.chan_mhz
        phi0 = rng.uniform(-np.pi, np.pi, (self.ntiles, 2))
        slope = rng.uniform(-self.slope_rad_per_mhz, self.slope_rad_per_mhz, (self.ntiles, 2))
        amp0 = rng.normal(1.0, 0.1, (self.ntiles, 2))
        leak = rng.normal(0.0, 0.01, (self.ntiles, self.nch, 4))
        blocks = []
        for b in range(self.nblocks):
            g = np.zeros((self.ntiles, self.nch, 8))
            # phase(f, b) = phi0 + slope (f + b drift): the delay behind the
            # slope moves the phase by slope * drift per timeblock
            ph = phi0[:, None, :] + slope[:, None, :] * (f[None, :, None] + b * self.drift_per_block)
            amp = amp0[:, None, :] * (1.0 + self.amp_jitter * rng.normal(size=(self.ntiles, 1, 2)))
            g[..., 0] = amp[..., 0] * np.cos(ph[..., 0])
            g[..., 1] = amp[..., 0] * np.sin(ph[..., 0])
            g[..., 6] = amp[..., 1] * np.cos(ph[..., 1])
            g[..., 7] = amp[..., 1] * np.sin(ph[..., 1])
            g[..., 2:6] = leak
            if device:
                model = synth.polarised_model_device(self.nt_per_block, self.nch, nbl, gen, self.cross_pol)
                data = synth.corrupt_device(model, g)
            else:
                model = synth.polarised_model(self.nt_per_block, self.nch, nbl, rng, self.cross_pol)
                data = synth.corrupt(model, g, rng, self.snr)
            blocks.append((data, model, g))
        return blocks
