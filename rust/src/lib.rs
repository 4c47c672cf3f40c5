//! hdc-sys: Rust binding of libhdc (include/hdc.h).
//!
//! `ffi` holds the raw declarations, generated from the C header by
//! `rust/gen_bindings.py` (the role bindgen plays for mwa_hyperdrive's
//! src/gpu headers).  The drop-in layer (`model_points`, `model_gaussians`,
//! `model_shapelets`, `model_autos`, `xyzs_to_uvws`, `rotate`, `average`,
//! `iono_loop`, `subtract_iono`, `add_model`, `get_gpu_device_info`) has the
//! names, struct layouts and argument meaning of mwa_hyperdrive's
//! src/gpu/{model,peel,utils}.h, so `SkyModellerGpu` and `peel_gpu` call it
//! unchanged once `build.rs` links libhdc instead of compiling src/gpu/*.cu.
//!
//! The safe wrappers below cover the native layer's trait-shaped entry
//! points: [`Modeller`] (the `SkyModeller` trait, model/mod.rs:123-204),
//! [`calibrate_timeblock`] (di_calibrate/mod.rs:387-618) and [`FeeBeam`]
//! (the `FEEBeamGpu` calls of beam/fee.rs:307-369).

pub mod ffi;
pub use ffi::*;

use std::ffi::CStr;
use std::fmt;
use std::os::raw::c_int;
use std::ptr::null_mut;

/// A failed libhdc call: the status code and `hdc_last_error()`.
#[derive(Debug, Clone)]
pub struct HdcError {
    pub status: c_int,
    pub message: String,
}

impl fmt::Display for HdcError {
    fn fmt(&self, f: &mut fmt::Formatter) -> fmt::Result {
        write!(f, "libhdc status {}: {}", self.status, self.message)
    }
}

impl std::error::Error for HdcError {}

/// Turn a native-layer status into a Result (the message is read from
/// `hdc_last_error`, which is per host thread).
pub fn check(status: c_int) -> Result<(), HdcError> {
    if status == HDC_OK {
        return Ok(());
    }
    let message = unsafe {
        let p = hdc_last_error();
        if p.is_null() { String::new() } else { CStr::from_ptr(p).to_string_lossy().into_owned() }
    };
    Err(HdcError { status, message })
}

/// Turn a drop-in result (NULL or a static error string) into a Result, as
/// mwa_hyperdrive's `GpuError::Kernel` wrapping does (gpu/mod.rs:73-101).
pub fn check_str(result: *const std::os::raw::c_char) -> Result<(), HdcError> {
    if result.is_null() {
        return Ok(());
    }
    let message = unsafe { CStr::from_ptr(result).to_string_lossy().into_owned() };
    Err(HdcError { status: HDC_ERR_CUDA, message })
}

/// The GPU sky modeller (SkyModellerGpu) over libhdc's native modeller.
pub struct Modeller {
    raw: *mut HdcModeller,
    pub num_freqs: usize,
    pub num_baselines: usize,
}

impl Modeller {
    /// new_sky_modeller (model/mod.rs:215-261) for the unflagged tiles and
    /// channels; `predict_form` is HDC_PREDICT_DIRECT (FP64) or
    /// HDC_PREDICT_TENSOR (tensor-core points, FP32-form Gaussians and
    /// shapelets, within 1e-6 of FP64).
    #[allow(clippy::too_many_arguments)]
    pub fn new(sky: &HdcSkyModel, pols: c_int, tile_xyzs: &[XYZ], freqs_hz: &[f64], phase_centre: RADec,
               array_latitude_rad: f64, beam_kind: c_int, predict_form: c_int) -> Result<Self, HdcError> {
        let mut raw = null_mut();
        check(unsafe {
            hdc_modeller_new(sky, pols, tile_xyzs.as_ptr(), tile_xyzs.len() as c_int, freqs_hz.as_ptr(),
                             freqs_hz.len() as c_int, phase_centre, array_latitude_rad, beam_kind, predict_form,
                             &mut raw)
        })?;
        let n = tile_xyzs.len();
        Ok(Modeller { raw, num_freqs: freqs_hz.len(), num_baselines: n * (n - 1) / 2 })
    }

    /// SkyModeller::model_timestep_with with a host buffer [freq][baseline]
    /// (accumulated into, as the trait does); returns the baseline UVWs.
    pub fn model_timestep_with(&mut self, lst_rad: f64, vis_fb: &mut [JonesF32]) -> Result<Vec<UVW>, HdcError> {
        assert_eq!(vis_fb.len(), self.num_freqs * self.num_baselines);
        let mut uvws = vec![UVW { u: 0.0, v: 0.0, w: 0.0 }; self.num_baselines];
        check(unsafe {
            hdc_modeller_model_timestep_with_host(self.raw, lst_rad, vis_fb.as_mut_ptr(), uvws.as_mut_ptr(),
                                                  null_mut())
        })?;
        Ok(uvws)
    }

    /// The device-buffer form (the reference's peel loop calls this shape):
    /// `d_vis_fb` is a device pointer; asynchronous on `stream`.
    ///
    /// # Safety
    /// `d_vis_fb` must point to num_freqs x num_baselines device JonesF32.
    pub unsafe fn model_timestep_with_device(&mut self, lst_rad: f64, d_vis_fb: *mut JonesF32,
                                             stream: *mut CUstream_st) -> Result<(), HdcError> {
        check(hdc_modeller_model_timestep_with(self.raw, lst_rad, d_vis_fb, null_mut(), stream))
    }

    /// SkyModeller::update_with_a_source (model/mod.rs:174).
    pub fn update_with_a_source(&mut self, source: &HdcSkyModel, phase_centre: RADec) -> Result<(), HdcError> {
        check(unsafe { hdc_modeller_update_with_a_source(self.raw, source, phase_centre) })
    }
}

impl Drop for Modeller {
    fn drop(&mut self) {
        unsafe { hdc_modeller_free(self.raw) }
    }
}

// The reference declares `unsafe impl Send for SkyModellerGpu`
// (model/gpu.rs:140); the native modeller is likewise used from one thread
// at a time.
unsafe impl Send for Modeller {}

/// The MWA FEE beam prepared on the current device (FEEBeam::gpu_prepare,
/// beam/fee.rs:307-320): the caller reads the beam file into `HdcFeeCoeffs`
/// (the `hdf5` crate; complex coefficients from the file's amplitude and
/// phase rows).
pub struct FeeBeam {
    raw: *mut HdcFeeBeam,
    pub num_tiles: usize,
    pub num_freqs: usize,
}

impl FeeBeam {
    /// `delays` [tile][16] (32: a dead dipole), `amps` [tile][32] (X then Y)
    /// or [tile][16]; `freqs_hz` the channels.
    pub fn new(file: &HdcFeeCoeffs, freqs_hz: &[u32], delays: &[[u32; 16]], amps: &[f64], num_amps: usize,
               norm_to_zenith: bool) -> Result<Self, HdcError> {
        assert!(num_amps == 16 || num_amps == 32);
        assert_eq!(amps.len(), delays.len() * num_amps);
        let mut raw = null_mut();
        check(unsafe {
            hdc_fee_beam_new(file, freqs_hz.as_ptr(), freqs_hz.len() as c_int, delays.as_ptr() as *const u32,
                             amps.as_ptr(), delays.len() as c_int, num_amps as c_int, norm_to_zenith as c_int,
                             &mut raw)
        })?;
        Ok(FeeBeam { raw, num_tiles: delays.len(), num_freqs: freqs_hz.len() })
    }

    /// BeamGpu::get_num_unique_tiles / get_num_unique_freqs.
    pub fn num_unique(&self) -> (usize, usize) {
        unsafe {
            (hdc_fee_beam_num_unique_tiles(self.raw) as usize, hdc_fee_beam_num_unique_freqs(self.raw) as usize)
        }
    }

    /// BeamGpu::get_tile_map / get_freq_map: device pointers owned by the beam.
    pub fn device_maps(&self) -> (*const c_int, *const c_int) {
        unsafe { (hdc_fee_beam_tile_map(self.raw), hdc_fee_beam_freq_map(self.raw)) }
    }

    /// BeamGpu::calc_jones_pair (iau_order false): `d_jones` gets
    /// [uniq tile][uniq freq][direction].
    ///
    /// # Safety
    /// `d_az_rad` and `d_za_rad` are device arrays of `n` directions,
    /// `d_latitude_rad` a device pointer to one value (or null), `d_jones`
    /// holds unique tiles x unique frequencies x `n` JonesF64.
    pub unsafe fn calc_jones_pair(&self, d_az_rad: *const f64, d_za_rad: *const f64, n: usize,
                                  d_latitude_rad: *const f64, d_jones: *mut JonesF64,
                                  stream: *mut CUstream_st) -> Result<(), HdcError> {
        check(hdc_fee_calc_jones(self.raw, d_az_rad, d_za_rad, n as c_int, d_latitude_rad, 0, d_jones, stream))
    }

    pub fn as_ptr(&self) -> *const HdcFeeBeam {
        self.raw
    }
}

impl Drop for FeeBeam {
    fn drop(&mut self) {
        unsafe { hdc_fee_beam_free(self.raw) }
    }
}

unsafe impl Send for FeeBeam {}

impl Modeller {
    /// The FEE beam for every tile (HDC_BEAM_FEE); `beam` must outlive the
    /// modeller's use of it.
    pub fn set_fee_beam(&mut self, beam: &FeeBeam) -> Result<(), HdcError> {
        check(unsafe { hdc_modeller_set_fee_beam(self.raw, beam.as_ptr()) })
    }
}

/// calibrate_timeblock (di_calibrate/mod.rs:387-618) on device buffers:
/// `d_di_jones` [tile][chanblock] holds the starting gains in and the
/// solutions out; one result per chanblock.
///
/// # Safety
/// The device pointers must hold the sizes the C declaration documents.
#[allow(clippy::too_many_arguments)]
pub unsafe fn calibrate_timeblock(d_data_tfb: *const JonesF32, d_model_tfb: *const JonesF32, num_timesteps: c_int,
                                  timeblock: (c_int, c_int), num_chanblocks: c_int, num_baselines: c_int,
                                  d_di_jones: *mut JonesF64, max_iterations: c_int, stop_threshold: f64,
                                  min_threshold: f64, pols: c_int, form: c_int,
                                  stream: *mut CUstream_st) -> Result<Vec<HdcCalResult>, HdcError> {
    let mut results = vec![
        HdcCalResult { num_iterations: 0, converged: 0, max_precision: 0.0, num_failed: 0 };
        num_chanblocks as usize
    ];
    check(hdc_calibrate_timeblock(d_data_tfb, d_model_tfb, num_timesteps, timeblock.0, timeblock.1, num_chanblocks,
                                  num_baselines, d_di_jones, max_iterations, stop_threshold, min_threshold, pols,
                                  results.as_mut_ptr(), form, stream))?;
    Ok(results)
}
