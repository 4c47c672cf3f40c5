"""SkyModeller: the host-side mirror of mwa_hyperdrive's ``SkyModeller`` trait
(model/mod.rs:123-204) and ``new_sky_modeller`` (model/mod.rs:215-261) over
libhdc's native modeller.

Visibility buffers are ``[freq][baseline][8]`` (JonesF32 / JonesF64 as 8
reals), device buffers are torch CUDA tensors, host buffers numpy arrays.
Times are given as the local mean sidereal time (the reference computes it
from an Epoch with marlu; precession, if wanted, is applied by passing
precessed tile XYZs through :meth:`SkyModeller.set_tile_xyzs`).
"""

from __future__ import annotations

import ctypes
from typing import Optional, Sequence, Union

import numpy as np

from . import _lib
from .srclist import SkyModelArrays, SourceList, Source

BEAMS = {"none": 0, "analytic": 1, "per_tile": 2, "fee": 3}
FORMS = {"direct": 0, "tensor": 1}
POLS = {"XX_XY_YX_YY": 0, "XX": 1, "YY": 2, "XX_YY": 3, "XX_YY_XY": 4}


def _as_sky(sky: Union[SourceList, SkyModelArrays, Source]) -> SkyModelArrays:
    if isinstance(sky, SkyModelArrays):
        return sky
    if isinstance(sky, SourceList):
        return sky.to_sky_model()
    if isinstance(sky, Source):
        return SkyModelArrays.from_components(sky.components)
    raise TypeError(f"cannot make a sky model from {type(sky)}")


def _stream_ptr(stream) -> ctypes.c_void_p:
    if stream is None:
        try:
            import torch

            return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        except Exception:
            return ctypes.c_void_p(0)
    if isinstance(stream, int):
        return ctypes.c_void_p(stream)
    return ctypes.c_void_p(stream.cuda_stream)


class SkyModeller:
    """GPU sky modeller (SkyModellerGpu equivalent)."""

    def __init__(self, sky, tile_xyzs, freqs, phase_centre, array_latitude_rad: float, pols: str = "XX_XY_YX_YY",
                 beam: str = "none", form: str = "direct", dipole_gains=None, beam_freq_res_hz: float = 1.28e6,
                 fee_beam=None):
        """beam: "none", "analytic" (the dipole-array tile, shared by all
        tiles), "per_tile" (each tile's own dipole amplitudes,
        ``dipole_gains`` [tile][2][16], 0 for a dead dipole; evaluated at the
        nearest multiple of ``beam_freq_res_hz`` of each channel) or "fee"
        (``fee_beam``, a :class:`mwa_hyperdrive_b200.fee.FeeBeam` prepared for
        these tiles and channels, kept alive by this modeller)."""
        self.lib = _lib.lib()
        self.sky = _as_sky(sky)
        self.tile_xyzs = np.ascontiguousarray(tile_xyzs, dtype=np.float64).reshape(-1, 3)
        self.freqs = np.ascontiguousarray(freqs, dtype=np.float64)
        self.num_tiles = self.tile_xyzs.shape[0]
        self.num_baselines = self.num_tiles * (self.num_tiles - 1) // 2
        self.num_freqs = self.freqs.size
        self.phase_centre = tuple(phase_centre)
        self.pols = pols
        self.beam = beam
        self.form = form
        h = ctypes.c_void_p()
        rc = self.lib.hdc_modeller_new(ctypes.byref(self.sky.struct()), POLS[pols], self.tile_xyzs.ctypes.data,
                                       self.num_tiles, self.freqs.ctypes.data, self.num_freqs,
                                       _lib.RADec(*self.phase_centre), float(array_latitude_rad),
                                       BEAMS["none"] if beam == "fee" else BEAMS[beam],
                                       FORMS[form], ctypes.byref(h))
        _lib.check(rc, "hdc_modeller_new")
        self._h = h
        if beam == "per_tile" and dipole_gains is not None:
            self.set_tile_beams(dipole_gains, beam_freq_res_hz)
        if beam == "fee":
            if fee_beam is None:
                raise ValueError('beam="fee" needs fee_beam')
            self.set_fee_beam(fee_beam)

    def set_fee_beam(self, fee_beam) -> None:
        """Use the FEE beam for every tile (its per-tile Jones are evaluated
        per timestep at each component's Az/ZA)."""
        _lib.check(self.lib.hdc_modeller_set_fee_beam(self._h, fee_beam.handle), "set_fee_beam")
        self._fee = fee_beam
        self.beam = "fee"

    def set_tile_beams(self, dipole_gains, beam_freq_res_hz: float = 1.28e6) -> None:
        g = np.ascontiguousarray(dipole_gains, dtype=np.float64).reshape(self.num_tiles, 2, 16)
        _lib.check(self.lib.hdc_modeller_set_tile_beams(self._h, g.ctypes.data, float(beam_freq_res_hz)),
                   "set_tile_beams")
        self.beam = "per_tile"

    def close(self) -> None:
        if getattr(self, "_h", None):
            self.lib.hdc_modeller_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_tile_xyzs(self, tile_xyzs) -> None:
        x = np.ascontiguousarray(tile_xyzs, dtype=np.float64).reshape(self.num_tiles, 3)
        _lib.check(self.lib.hdc_modeller_set_tile_xyzs(self._h, x.ctypes.data), "set_tile_xyzs")
        self.tile_xyzs = x

    def model_timestep_with(self, lst_rad: float, vis_fb, stream=None, return_uvws: bool = True):
        """Accumulate this timestep's cross-correlation model into the device
        tensor ``vis_fb`` ([freq][bl][8], float32 or float64).  Returns the
        baseline UVWs [m] (numpy [bl][3]) if ``return_uvws``."""
        uvws = np.zeros((self.num_baselines, 3)) if return_uvws else None
        up = uvws.ctypes.data if return_uvws else None
        ptr = vis_fb.data_ptr()
        if str(vis_fb.dtype) == "torch.float64":
            rc = self.lib.hdc_modeller_model_timestep_with_f64(self._h, float(lst_rad), ptr, up, _stream_ptr(stream))
        else:
            rc = self.lib.hdc_modeller_model_timestep_with(self._h, float(lst_rad), ptr, up, _stream_ptr(stream))
        _lib.check(rc, "model_timestep_with")
        return uvws

    def model_timestep_with_host(self, lst_rad: float, vis_fb: np.ndarray, stream=None):
        """Trait-style call with a host buffer (copied in, accumulated, copied
        back), as SkyModellerGpu::model_timestep_with does."""
        assert vis_fb.dtype == np.float32 and vis_fb.flags.c_contiguous
        assert vis_fb.shape == (self.num_freqs, self.num_baselines, 8)
        uvws = np.zeros((self.num_baselines, 3))
        rc = self.lib.hdc_modeller_model_timestep_with_host(self._h, float(lst_rad), vis_fb.ctypes.data,
                                                            uvws.ctypes.data, _stream_ptr(stream))
        _lib.check(rc, "model_timestep_with_host")
        return uvws

    def model_timestep(self, lst_rad: float):
        """SkyModeller::model_timestep: a fresh host buffer plus the UVWs."""
        vis = np.zeros((self.num_freqs, self.num_baselines, 8), np.float32)
        uvws = self.model_timestep_with_host(lst_rad, vis)
        return vis, uvws

    def update_with_a_source(self, source, phase_centre) -> None:
        self.sky = _as_sky(source)
        self.phase_centre = tuple(phase_centre)
        rc = self.lib.hdc_modeller_update_with_a_source(self._h, ctypes.byref(self.sky.struct()),
                                                        _lib.RADec(*self.phase_centre))
        _lib.check(rc, "update_with_a_source")

    def model_timestep_autos_with(self, lst_rad: float, vis_ft, stream=None) -> None:
        rc = self.lib.hdc_modeller_model_timestep_autos_with(self._h, float(lst_rad), vis_ft.data_ptr(),
                                                             _stream_ptr(stream))
        _lib.check(rc, "model_timestep_autos_with")


def new_sky_modeller(sky, pols, unflagged_tile_xyzs, unflagged_fine_chan_freqs, phase_centre, array_latitude_rad,
                     beam: str = "none", form: str = "direct") -> SkyModeller:
    """Factory mirroring model/mod.rs:215-261 (the GPU branch)."""
    return SkyModeller(sky, unflagged_tile_xyzs, unflagged_fine_chan_freqs, phase_centre, array_latitude_rad,
                       pols=pols, beam=beam, form=form)


def device_info() -> str:
    buf = ctypes.create_string_buffer(512)
    _lib.check(_lib.lib().hdc_device_info(buf, 512), "hdc_device_info")
    return buf.value.decode()
