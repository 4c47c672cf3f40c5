"""ctypes binding of libhdc.so (include/hdc.h).

The library is loaded from this package directory; if it is missing or
cannot be loaded the import of any compute entry point fails loudly (there is
no CPU fallback).
"""

from __future__ import annotations

import ctypes
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libhdc.so"

c_int, c_double, c_float, c_void_p, c_char_p = ctypes.c_int, ctypes.c_double, ctypes.c_float, ctypes.c_void_p, ctypes.c_char_p


class HdcError(RuntimeError):
    pass


class RADec(ctypes.Structure):
    _fields_ = [("ra", c_double), ("dec", c_double)]


class XYZ(ctypes.Structure):
    _fields_ = [("x", c_double), ("y", c_double), ("z", c_double)]


class UVW(ctypes.Structure):
    _fields_ = [("u", c_double), ("v", c_double), ("w", c_double)]


class IonoConsts(ctypes.Structure):
    _fields_ = [("alpha", c_double), ("beta", c_double), ("gain", c_double)]


class HdcPeelParams(ctypes.Structure):
    _fields_ = [("num_passes", c_int), ("num_loops", c_int), ("convergence", c_double),
                ("freq_average_factor", c_int), ("beam_kind", c_int), ("array_latitude_rad", c_double),
                ("batch_size", c_int), ("fee_beam", c_void_p)]


class HdcFeeCoeffs(ctypes.Structure):
    _fields_ = [("num_freqs", c_int), ("freqs_hz", c_void_p), ("num_modes", c_int), ("modes", c_void_p),
                ("num_freq_modes", c_void_p), ("q", c_void_p)]


class HdcCalResult(ctypes.Structure):
    _fields_ = [("num_iterations", c_int), ("converged", c_int), ("max_precision", c_double), ("num_failed", c_int)]


class Addresses(ctypes.Structure):
    _fields_ = [
        ("num_freqs", c_int), ("num_vis", c_int), ("num_baselines", c_int),
        ("d_freqs", c_void_p), ("d_shapelet_basis_values", c_void_p),
        ("num_unique_beam_freqs", c_int),
        ("d_tile_map", c_void_p), ("d_freq_map", c_void_p), ("d_tile_index_to_unflagged_tile_index_map", c_void_p),
    ]


class Points(ctypes.Structure):
    _fields_ = [
        ("num_power_laws", c_int), ("power_law_lmns", c_void_p), ("power_law_fds", c_void_p),
        ("power_law_sis", c_void_p),
        ("num_curved_power_laws", c_int), ("curved_power_law_lmns", c_void_p), ("curved_power_law_fds", c_void_p),
        ("curved_power_law_sis", c_void_p), ("curved_power_law_qs", c_void_p),
        ("num_lists", c_int), ("list_lmns", c_void_p), ("list_fds", c_void_p),
    ]


class Gaussians(ctypes.Structure):
    _fields_ = [
        ("num_power_laws", c_int), ("power_law_lmns", c_void_p), ("power_law_fds", c_void_p),
        ("power_law_sis", c_void_p), ("power_law_gps", c_void_p),
        ("num_curved_power_laws", c_int), ("curved_power_law_lmns", c_void_p), ("curved_power_law_fds", c_void_p),
        ("curved_power_law_sis", c_void_p), ("curved_power_law_qs", c_void_p), ("curved_power_law_gps", c_void_p),
        ("num_lists", c_int), ("list_lmns", c_void_p), ("list_fds", c_void_p), ("list_gps", c_void_p),
    ]


class Shapelets(ctypes.Structure):
    _fields_ = [
        ("num_power_laws", c_int), ("power_law_lmns", c_void_p), ("power_law_fds", c_void_p),
        ("power_law_sis", c_void_p), ("power_law_gps", c_void_p), ("power_law_shapelet_uvs", c_void_p),
        ("power_law_shapelet_coeffs", c_void_p), ("power_law_num_shapelet_coeffs", c_void_p),
        ("num_curved_power_laws", c_int), ("curved_power_law_lmns", c_void_p), ("curved_power_law_fds", c_void_p),
        ("curved_power_law_sis", c_void_p), ("curved_power_law_qs", c_void_p), ("curved_power_law_gps", c_void_p),
        ("curved_power_law_shapelet_uvs", c_void_p), ("curved_power_law_shapelet_coeffs", c_void_p),
        ("curved_power_law_num_shapelet_coeffs", c_void_p),
        ("num_lists", c_int), ("list_lmns", c_void_p), ("list_fds", c_void_p), ("list_gps", c_void_p),
        ("list_shapelet_uvs", c_void_p), ("list_shapelet_coeffs", c_void_p), ("list_num_shapelet_coeffs", c_void_p),
    ]


# Every symbol include/hdc.h declares, with its argument and result types.
SIGNATURES = {
    "model_points": (c_char_p, [ctypes.POINTER(Points), ctypes.POINTER(Addresses), c_void_p, c_void_p, c_void_p]),
    "model_points_noalloc": (c_char_p, [ctypes.POINTER(Points), ctypes.POINTER(Addresses), c_void_p, c_void_p,
                                        c_void_p]),
    "model_points_f64out": (c_char_p, [ctypes.POINTER(Points), ctypes.POINTER(Addresses), c_void_p, c_void_p,
                                       c_void_p]),
    "model_points_tc": (c_char_p, [ctypes.POINTER(Points), ctypes.POINTER(Addresses), c_void_p, c_double, RADec,
                                   c_void_p, c_void_p]),
    "model_gaussians": (c_char_p, [ctypes.POINTER(Gaussians), ctypes.POINTER(Addresses), c_void_p, c_void_p,
                                   c_void_p]),
    "model_gaussians_f64out": (c_char_p, [ctypes.POINTER(Gaussians), ctypes.POINTER(Addresses), c_void_p, c_void_p,
                                          c_void_p]),
    "model_shapelets_f64out": (c_char_p, [ctypes.POINTER(Shapelets), ctypes.POINTER(Addresses), c_void_p, c_void_p,
                                          c_void_p]),
    "model_shapelets": (c_char_p, [ctypes.POINTER(Shapelets), ctypes.POINTER(Addresses), c_void_p, c_void_p,
                                   c_void_p]),
    "model_autos": (c_char_p, [c_int, c_int, c_void_p, ctypes.POINTER(Points), ctypes.POINTER(Gaussians),
                               ctypes.POINTER(Shapelets), c_void_p, c_void_p, c_void_p, c_int, c_void_p, c_void_p]),
    "xyzs_to_uvws": (c_char_p, [c_void_p, c_void_p, c_void_p, RADec, c_int, c_int, c_int]),
    "rotate": (c_char_p, [c_void_p, c_int, c_int, c_int, c_void_p, c_void_p, c_void_p]),
    "average": (c_char_p, [c_void_p, c_void_p, c_void_p, c_int, c_int, c_int, c_int]),
    "iono_loop": (c_char_p, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, ctypes.POINTER(IonoConsts), c_int,
                             c_int, c_int, c_void_p, c_void_p, c_double]),
    "subtract_iono": (c_char_p, [c_void_p, c_void_p, IonoConsts, IonoConsts, c_void_p, c_void_p, c_int, c_int,
                                 c_int]),
    "add_model": (c_char_p, [c_void_p, c_void_p, IonoConsts, c_void_p, c_void_p, c_int, c_int, c_int]),
    "hdc_last_error": (c_char_p, []),
    "hdc_device_info": (c_int, [c_char_p, c_int]),
    "hdc_modeller_new": (c_int, [c_void_p, c_int, c_void_p, c_int, c_void_p, c_int, RADec, c_double, c_int, c_int,
                                 ctypes.POINTER(c_void_p)]),
    "hdc_modeller_free": (None, [c_void_p]),
    "hdc_modeller_set_tile_xyzs": (c_int, [c_void_p, c_void_p]),
    "hdc_modeller_set_tile_beams": (c_int, [c_void_p, c_void_p, c_double]),
    "hdc_modeller_set_fee_beam": (c_int, [c_void_p, c_void_p]),
    "hdc_fee_beam_new": (c_int, [ctypes.POINTER(HdcFeeCoeffs), c_void_p, c_int, c_void_p, c_void_p, c_int, c_int,
                                 c_int, ctypes.POINTER(c_void_p)]),
    "hdc_fee_beam_free": (None, [c_void_p]),
    "hdc_fee_beam_num_unique_tiles": (c_int, [c_void_p]),
    "hdc_fee_beam_num_unique_freqs": (c_int, [c_void_p]),
    "hdc_fee_beam_tile_map": (c_void_p, [c_void_p]),
    "hdc_fee_beam_freq_map": (c_void_p, [c_void_p]),
    "hdc_fee_beam_host_maps": (c_int, [c_void_p, c_void_p, c_void_p]),
    "hdc_fee_calc_jones": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_void_p, c_int, c_void_p, c_void_p]),
    "hdc_modeller_model_timestep_with": (c_int, [c_void_p, c_double, c_void_p, c_void_p, c_void_p]),
    "hdc_modeller_model_timestep_with_f64": (c_int, [c_void_p, c_double, c_void_p, c_void_p, c_void_p]),
    "hdc_modeller_model_timestep_with_host": (c_int, [c_void_p, c_double, c_void_p, c_void_p, c_void_p]),
    "hdc_modeller_update_with_a_source": (c_int, [c_void_p, c_void_p, RADec]),
    "hdc_modeller_model_timestep_autos_with": (c_int, [c_void_p, c_double, c_void_p, c_void_p]),
    "hdc_calibrate_timeblock": (c_int, [c_void_p, c_void_p, c_int, c_int, c_int, c_int, c_int, c_void_p, c_int,
                                        c_double, c_double, c_int, ctypes.POINTER(HdcCalResult), c_int, c_void_p]),
    "hdc_calibrate_chanblocks": (c_int, [c_void_p, c_void_p, c_int, c_int, c_int, c_int, c_int, c_void_p, c_int,
                                         c_double, c_double, c_int, c_void_p, c_int, ctypes.POINTER(HdcCalResult),
                                         c_int, c_void_p]),
    "hdc_calibrate_timeblocks": (c_int, [c_void_p, c_void_p, c_int, c_void_p, c_int, c_int, c_int, c_void_p, c_int,
                                         c_double, c_double, c_int, ctypes.POINTER(HdcCalResult), c_int, c_void_p]),
    "hdc_peel_timeblock": (c_int, [c_void_p, c_void_p, c_int, c_int, c_void_p, c_void_p, c_int, c_void_p, c_double,
                                   RADec, c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    "hdc_peel_timeblock_batched": (c_int, [c_void_p, c_void_p, c_int, c_int, c_void_p, c_void_p, c_int, c_void_p,
                                           c_double, RADec, c_int, c_void_p, c_void_p, c_void_p, c_void_p,
                                           c_void_p]),
    "hdc_peel_batched_tuning": (c_int, [ctypes.POINTER(c_int), ctypes.POINTER(c_int), ctypes.POINTER(c_float)]),
    "hdc_calibration_residuals": (c_int, [c_void_p, c_void_p, c_int, c_int, c_int, c_int, c_int, c_void_p, c_void_p,
                                          c_void_p]),
    "hdc_mlp_new": (c_int, [c_int, c_void_p, c_int, ctypes.c_ulonglong, ctypes.POINTER(c_void_p)]),
    "hdc_mlp_free": (None, [c_void_p]),
    "hdc_mlp_num_params": (ctypes.c_longlong, [c_void_p]),
    "hdc_mlp_get_params": (c_int, [c_void_p, c_void_p]),
    "hdc_mlp_set_params": (c_int, [c_void_p, c_void_p]),
    "hdc_mlp_forward": (c_int, [c_void_p, c_void_p, c_int, c_void_p, c_void_p]),
    "hdc_mlp_gradients": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_void_p, c_void_p, c_void_p]),
    "hdc_mlp_train_step": (c_int, [c_void_p, c_void_p, c_void_p, c_int, ctypes.c_float, c_void_p, c_void_p]),
    "hdc_warmstart_features": (c_int, [c_void_p, c_int, c_int, c_void_p, c_void_p]),
    "hdc_warmstart_judge": (c_int, [c_void_p, c_void_p, c_int, c_int, c_int, c_int, c_int, c_void_p, c_void_p,
                                    c_void_p, c_void_p]),
    "hdc_warmstart_propose": (c_int, [c_void_p, c_void_p, c_int, c_int, c_void_p, c_void_p, c_int, c_int, c_int,
                                      c_void_p, c_void_p, c_void_p]),
    "hdc_kernel_launches": (ctypes.c_longlong, []),
    "hdc_kernel_error_string": (c_char_p, [c_int]),
    "hdc_test_stall_next_predict": (c_int, [ctypes.c_ulonglong]),
    "get_gpu_device_info": (c_char_p, [c_int, c_char_p, ctypes.POINTER(c_int), ctypes.POINTER(c_int),
                                       ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(c_int), ctypes.POINTER(c_int)]),
    "hdc_modeller_set_profiling": (c_int, [c_void_p, c_int]),
    "hdc_modeller_profile": (c_int, [c_void_p, c_void_p, c_int]),
    "hdc_probe_fp64_gflops": (c_int, [ctypes.POINTER(c_double)]),
    "hdc_source_brightness": (c_int, [c_void_p, c_void_p, c_int, c_void_p, c_int, c_double, c_double, RADec, c_int,
                                      c_double, c_double, c_void_p]),
    "hdc_source_brightness_fee": (c_int, [c_void_p, c_void_p, c_int, c_void_p, c_int, c_double, c_double, RADec, c_void_p,
                                      c_double, c_double, c_void_p]),
    "hdc_probe_fp32_gflops": (c_int, [ctypes.POINTER(c_double)]),
    "hdc_scale_by_weights": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_int, c_int, c_void_p, c_void_p]),
    "hdc_into_cal_sols": (c_int, [c_void_p, c_int, c_int, c_int, c_void_p, c_int, c_void_p, c_int, c_int, c_void_p,
                                  c_void_p]),
    "hdc_vis_average": (c_int, [c_void_p, c_void_p, c_int, c_int, c_int, c_void_p, c_int, c_void_p, c_void_p, c_int,
                                c_void_p]),
}

# Symbols exported for tests/tools that include/hdc.h does not declare.
EXTRA = {
    "hdc_shapelet_basis": (c_int, [c_void_p]),
}

_lib = None


def lib() -> ctypes.CDLL:
    """Load libhdc.so (raises HdcError if it is missing)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise HdcError(f"{LIB_PATH} is missing: build it with `python -m mwa_hyperdrive_b200.build`")
        l = ctypes.CDLL(str(LIB_PATH))
        for name, (res, args) in {**SIGNATURES, **EXTRA}.items():
            fn = getattr(l, name)
            fn.restype = res
            fn.argtypes = args
        _lib = l
    return _lib


def check(rc: int, what: str = "") -> None:
    if rc != 0:
        msg = lib().hdc_last_error().decode(errors="replace")
        raise HdcError(f"{what} failed (status {rc}): {msg}")


def check_str(res, what: str = "") -> None:
    if res is not None:
        raise HdcError(f"{what} failed: {res.decode(errors='replace')}")
