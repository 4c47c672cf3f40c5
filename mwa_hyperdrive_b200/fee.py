"""The MWA FEE beam on the device: the host-side mirror of the calls the
reference makes on mwa_hyperbeam 0.11.0 (beam/fee.rs:307-369):
``FEEBeam::gpu_prepare(freqs, delays, gains, norm_to_zenith)`` ->
:class:`FeeBeam`, ``calc_jones_device_pair_inner(az, za, latitude,
iau_order)`` -> :meth:`FeeBeam.calc_jones`, and the unique-tile /
unique-frequency maps of ``BeamGpu`` (beam/mod.rs:355-367).

The coefficients are the contents of the beam file
(mwa_full_embedded_element_pattern.h5) as a dict of arrays (keys
``freqs_hz``, ``modes``, ``num_freq_modes``, ``q``; see ``HdcFeeCoeffs`` in
include/hdc.h); HDF5 is not linked, so reading the file is the caller's.
"""

from __future__ import annotations

import ctypes

import numpy as np

from . import _lib


def _coeff_struct(file: dict):
    keep = {
        "freqs_hz": np.ascontiguousarray(file["freqs_hz"], np.uint32),
        "modes": np.ascontiguousarray(file["modes"], np.int32),
        "num_freq_modes": np.ascontiguousarray(file["num_freq_modes"], np.int32),
        "q": np.ascontiguousarray(file["q"], np.float64),
    }
    nf = keep["freqs_hz"].size
    nmodes = keep["modes"].shape[1]
    if keep["q"].shape != (nf, 2, 16, nmodes, 2):
        raise ValueError(f"q has shape {keep['q'].shape}, expected {(nf, 2, 16, nmodes, 2)}")
    s = _lib.HdcFeeCoeffs(nf, keep["freqs_hz"].ctypes.data, nmodes, keep["modes"].ctypes.data,
                          keep["num_freq_modes"].ctypes.data, keep["q"].ctypes.data)
    return s, keep


class FeeBeam:
    """FEE beam prepared on the current device for ``freqs_hz`` (channels)
    and every tile's ``delays`` [tile][16] (32 marks a dead dipole) and
    ``amps`` [tile][32] (or [tile][16] for both polarisations)."""

    def __init__(self, file: dict, freqs_hz, delays, amps, norm_to_zenith: bool = True):
        self.lib = _lib.lib()
        s, keep = _coeff_struct(file)
        f = np.ascontiguousarray(np.rint(np.asarray(freqs_hz, np.float64)), np.uint32)
        d = np.ascontiguousarray(delays, np.uint32)
        a = np.ascontiguousarray(amps, np.float64)
        if d.ndim != 2 or d.shape[1] != 16 or a.ndim != 2 or a.shape[0] != d.shape[0] or a.shape[1] not in (16, 32):
            raise ValueError("delays must be [tile][16] and amps [tile][16 or 32]")
        self.num_tiles, self.num_freqs = d.shape[0], f.size
        h = ctypes.c_void_p()
        _lib.check(self.lib.hdc_fee_beam_new(ctypes.byref(s), f.ctypes.data, f.size, d.ctypes.data, a.ctypes.data,
                                             d.shape[0], a.shape[1], int(bool(norm_to_zenith)), ctypes.byref(h)),
                   "hdc_fee_beam_new")
        del keep
        self._h = h

    @property
    def handle(self):
        return self._h

    def num_unique_tiles(self) -> int:
        return self.lib.hdc_fee_beam_num_unique_tiles(self._h)

    def num_unique_freqs(self) -> int:
        return self.lib.hdc_fee_beam_num_unique_freqs(self._h)

    def maps(self):
        """(tile_map [tile], freq_map [channel]) as host arrays."""
        t = np.zeros(self.num_tiles, np.int32)
        f = np.zeros(self.num_freqs, np.int32)
        _lib.check(self.lib.hdc_fee_beam_host_maps(self._h, t.ctypes.data, f.ctypes.data), "hdc_fee_beam_host_maps")
        return t, f

    def calc_jones(self, az_rad, za_rad, latitude_rad=None, stream=None):
        """Jones [uniq tile][uniq freq][direction][8] (torch, float64, on the
        device) for device or host direction arrays."""
        import torch

        az = torch.as_tensor(np.asarray(az_rad, np.float64) if not torch.is_tensor(az_rad) else az_rad,
                             dtype=torch.float64, device="cuda").contiguous()
        za = torch.as_tensor(np.asarray(za_rad, np.float64) if not torch.is_tensor(za_rad) else za_rad,
                             dtype=torch.float64, device="cuda").contiguous()
        n = az.numel()
        out = torch.empty((self.num_unique_tiles(), self.num_unique_freqs(), n, 8), dtype=torch.float64,
                          device="cuda")
        lat = None if latitude_rad is None else torch.tensor([float(latitude_rad)], dtype=torch.float64,
                                                             device="cuda")
        st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream if stream is None else stream.cuda_stream)
        _lib.check(self.lib.hdc_fee_calc_jones(self._h, az.data_ptr(), za.data_ptr(), n,
                                               None if lat is None else lat.data_ptr(), 0, out.data_ptr(), st),
                   "hdc_fee_calc_jones")
        self._last = (az, za, lat)  # keep the inputs alive until the stream has used them
        return out

    def close(self) -> None:
        if getattr(self, "_h", None):
            self.lib.hdc_fee_beam_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
