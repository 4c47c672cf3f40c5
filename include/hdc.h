/*
 * hdc.h -- C ABI of libhdc, the B200 (sm_100a) sky-model predictor,
 * DI calibration and peeling library.
 *
 * Two layers:
 *
 *  1. Drop-in layer.  The structs and entry points of mwa_hyperdrive's GPU FFI
 *     with the same names, field order and argument meaning, FP64 build
 *     (gpu/types.h, gpu/model.h:33-56, gpu/peel.h:13-35).  A Rust host that
 *     binds those headers with bindgen binds these unchanged.  Like the
 *     reference they return NULL on success or a static error string, run on
 *     the legacy default stream of the current device and accumulate (+=)
 *     into visibility buffers.
 *
 *  2. Native layer (hdc_*).  The SkyModeller trait (model/mod.rs:123-204),
 *     calibrate_timeblock (di_calibrate/mod.rs:387-618) and the peel loop
 *     (params/peel/gpu.rs:25-757) as C entry points with explicit streams.
 *     They return an int status (HDC_OK == 0) and leave a message in
 *     hdc_last_error().
 *
 * Pointers named d_* are device pointers; h_* are host pointers.  Visibility
 * layouts are the reference's: [time][freq][baseline], baselines in
 * upper-triangle order (tile1 < tile2, row-major; math/mod.rs:94-109).
 */
#pragma once

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------------- */
/* Types (gpu/types.h, FP64 build: FLOAT = double, JONES = JonesF64)       */
/* ---------------------------------------------------------------------- */

typedef struct RADec {
    double ra;  /* [rad] */
    double dec; /* [rad] */
} RADec;

typedef struct HADec {
    double ha;
    double dec;
} HADec;

typedef struct XYZ {
    double x, y, z; /* [m] */
} XYZ;

typedef struct UVW {
    double u, v, w; /* [m] */
} UVW;

/* LMN prepared for the RIME: (2 pi l, 2 pi m, 2 pi (n - 1)). */
typedef struct LmnRime {
    double l, m, n;
} LmnRime;

typedef struct GaussianParams {
    double maj, min, pa; /* [rad] */
} GaussianParams;

typedef struct ShapeletCoeff {
    double value;
    unsigned char n1;
    unsigned char n2;
} ShapeletCoeff;

typedef struct ShapeletUV {
    double u, v; /* [m] */
} ShapeletUV;

typedef struct JonesF32 {
    float j00_re, j00_im, j01_re, j01_im, j10_re, j10_im, j11_re, j11_im;
} JonesF32;

typedef struct JonesF64 {
    double j00_re, j00_im, j01_re, j01_im, j10_re, j10_im, j11_re, j11_im;
} JonesF64;

/* gpu/types.h:172-183 */
typedef struct Addresses {
    const int num_freqs;
    const int num_vis;
    const int num_baselines;
    const double *d_freqs;
    const double *d_shapelet_basis_values;
    const int num_unique_beam_freqs;
    const int *d_tile_map;
    const int *d_freq_map;
    const int *d_tile_index_to_unflagged_tile_index_map;
} Addresses;

/* gpu/types.h:187-205 */
typedef struct Points {
    const int num_power_laws;
    const LmnRime *power_law_lmns;
    const JonesF64 *power_law_fds; /* instrumental, at 150 MHz */
    const double *power_law_sis;
    const int num_curved_power_laws;
    const LmnRime *curved_power_law_lmns;
    const JonesF64 *curved_power_law_fds;
    const double *curved_power_law_sis;
    const double *curved_power_law_qs;
    const int num_lists;
    const LmnRime *list_lmns;
    const JonesF64 *list_fds; /* [freq][num_lists] */
} Points;

/* gpu/types.h:210-233 */
typedef struct Gaussians {
    const int num_power_laws;
    const LmnRime *power_law_lmns;
    const JonesF64 *power_law_fds;
    const double *power_law_sis;
    const GaussianParams *power_law_gps;
    const int num_curved_power_laws;
    const LmnRime *curved_power_law_lmns;
    const JonesF64 *curved_power_law_fds;
    const double *curved_power_law_sis;
    const double *curved_power_law_qs;
    const GaussianParams *curved_power_law_gps;
    const int num_lists;
    const LmnRime *list_lmns;
    const JonesF64 *list_fds;
    const GaussianParams *list_gps;
} Gaussians;

/* gpu/types.h:238-267 */
typedef struct Shapelets {
    const int num_power_laws;
    const LmnRime *power_law_lmns;
    const JonesF64 *power_law_fds;
    const double *power_law_sis;
    const GaussianParams *power_law_gps;
    const ShapeletUV *power_law_shapelet_uvs; /* [baseline][num_power_laws] */
    const ShapeletCoeff *power_law_shapelet_coeffs;
    const int *power_law_num_shapelet_coeffs;
    const int num_curved_power_laws;
    const LmnRime *curved_power_law_lmns;
    const JonesF64 *curved_power_law_fds;
    const double *curved_power_law_sis;
    const double *curved_power_law_qs;
    const GaussianParams *curved_power_law_gps;
    const ShapeletUV *curved_power_law_shapelet_uvs;
    const ShapeletCoeff *curved_power_law_shapelet_coeffs;
    const int *curved_power_law_num_shapelet_coeffs;
    const int num_lists;
    const LmnRime *list_lmns;
    const JonesF64 *list_fds;
    const GaussianParams *list_gps;
    const ShapeletUV *list_shapelet_uvs;
    const ShapeletCoeff *list_shapelet_coeffs;
    const int *list_num_shapelet_coeffs;
} Shapelets;

/* gpu/types.h:280-287 */
typedef struct IonoConsts {
    double alpha;
    double beta;
    double gain;
} IonoConsts;

/* ---------------------------------------------------------------------- */
/* Drop-in layer                                                           */
/* ---------------------------------------------------------------------- */

/* Replaces gpu/model.h:33 model_points.  Cross-correlation visibilities of
 * point components for one timestep, accumulated into d_vis_fb [freq][bl].
 * Power-law fluxes are given at 150 MHz (POWER_LAW_FD_REF_FREQ). */
const char *model_points(const Points *comps, const Addresses *a, const UVW *d_uvws, const JonesF64 *d_beam_jones,
                         JonesF32 *d_vis_fb);

/* No counterpart in the reference.  model_points for callers that cannot
 * allocate device memory (hosts that reserve the whole device for their own
 * memory pool, or streaming loops that must not call cudaMalloc because of its
 * implicit device synchronisation).  Same arguments and result as
 * model_points, but its scratch is a fixed array compiled into the library
 * (HDC_NOALLOC_SCRATCH_BYTES per device, held until exit): it needs
 * 64 B per component + 64 B per (channel, component), each of its three
 * tables rounded up to 256 B (LMN 32 B and envelope 32 B per component, flux
 * 64 B per channel and component), and larger problems are rejected with an
 * error.  Kernel errors are read back and cleared as in model_points.  Every
 * call on a device shares that array, so calls whose kernels overlap on the
 * GPU race and must be serialised.  The first call on a device looks up the
 * array's device address and should come before any stream capture. */
#define HDC_NOALLOC_SCRATCH_BYTES (16u * 1024u * 1024u)
const char *model_points_noalloc(const Points *comps, const Addresses *a, const UVW *d_uvws,
                                 const JonesF64 *d_beam_jones, JonesF32 *d_vis_fb);

/* model_points with FP64 output (d_vis_fb JonesF64 [freq][bl], accumulated):
 * the 1e-10 parity mode.  No counterpart in the reference, whose output
 * precision is fixed at compile time (gpu/types.h:13-21). */
const char *model_points_f64out(const Points *comps, const Addresses *a, const UVW *d_uvws,
                                const JonesF64 *d_beam_jones, JonesF64 *d_vis_fb);

/* model_points on the tensor cores (tcgen05 integer digit planes; results
 * within 1e-6 of the FP64 predict).  No counterpart in the reference.  Takes
 * the per-tile XYZs (d_tile_xyzs [tile], metres, the tile order of the
 * baselines), the LST and the phase centre instead of per-baseline UVWs: the
 * predict factors per tile because uvw_pq = R (xyz_p - xyz_q).  The beam is
 * d_beam_jones NULL (none) or the reference's layout [uniq_tile][uniq_freq]
 * [component] with Addresses' tile and frequency maps: when every tile maps
 * to one row it is applied as W = B S B^H per component, otherwise per tile
 * (the block form over twice the components, about twice the tensor-core
 * work).  Any number of tiles (blocks of 128 x 64 tiles). */
const char *model_points_tc(const Points *comps, const Addresses *a, const XYZ *d_tile_xyzs, double lst_rad,
                            RADec phase_centre, const JonesF64 *d_beam_jones, JonesF32 *d_vis_fb);

/* Replaces gpu/model.h:40 model_gaussians. */
const char *model_gaussians(const Gaussians *comps, const Addresses *a, const UVW *d_uvws,
                            const JonesF64 *d_beam_jones, JonesF32 *d_vis_fb);

/* model_gaussians with FP64 output (see model_points_f64out). */
const char *model_gaussians_f64out(const Gaussians *comps, const Addresses *a, const UVW *d_uvws,
                                   const JonesF64 *d_beam_jones, JonesF64 *d_vis_fb);

/* Replaces gpu/model.h:47 model_shapelets. */
const char *model_shapelets(const Shapelets *comps, const Addresses *a, const UVW *d_uvws,
                            const JonesF64 *d_beam_jones, JonesF32 *d_vis_fb);

/* model_shapelets with FP64 output (see model_points_f64out). */
const char *model_shapelets_f64out(const Shapelets *comps, const Addresses *a, const UVW *d_uvws,
                                   const JonesF64 *d_beam_jones, JonesF64 *d_vis_fb);

/* Replaces gpu/model.h:53 model_autos.  vis_fb is [freq][tile]. */
const char *model_autos(int num_tiles, int num_freqs, const double *freqs, const Points *points,
                        const Gaussians *gaussians, const Shapelets *shapelets, const JonesF64 *beam_jones,
                        const int *tile_map, const int *freq_map, int num_fee_freqs,
                        const int *tile_index_to_unflagged_tile_index_map, JonesF32 *vis_fb);

/* Replaces gpu/peel.h:13 xyzs_to_uvws: d_xyzs [t][tile], d_lmsts [t],
 * d_uvws [t][bl]. */
const char *xyzs_to_uvws(const XYZ *d_xyzs, const double *d_lmsts, UVW *d_uvws, RADec pointing_centre, int num_tiles,
                         int num_baselines, int num_timesteps);

/* Replaces gpu/peel.h:16 rotate (in place, [t][f][bl]). */
const char *rotate(JonesF32 *vis_fb, const int num_timesteps, const int num_baselines, const int num_freqs,
                   const UVW *uvws_from, const UVW *uvws_to, const double *lambdas);

/* Replaces gpu/peel.h:19 average (time and freq_average_factor channels). */
const char *average(const JonesF32 *d_high_res_vis, const float *d_high_res_weights, JonesF32 *d_low_res_vis,
                    const int num_timesteps, const int num_baselines, const int num_freqs,
                    const int freq_average_factor);

/* Replaces gpu/peel.h:23 iono_loop.  *iono_consts is read and updated. */
const char *iono_loop(const JonesF32 *d_vis_residual, const float *d_vis_weights, const JonesF32 *d_vis_model,
                      JonesF32 *d_vis_model_rotated, JonesF64 *d_iono_fits, IonoConsts *iono_consts,
                      const int num_baselines, const int num_freqs, const int num_iterations, const UVW *d_uvws,
                      const double *d_lambdas_m, const double convergence);

/* Replaces gpu/peel.h:29 subtract_iono. */
const char *subtract_iono(JonesF32 *d_vis_residual, const JonesF32 *d_vis_model, const IonoConsts iono_consts,
                          const IonoConsts old_iono_consts, const UVW *d_uvws, const double *d_lambdas_m,
                          const int num_timesteps, const int num_baselines, const int num_freqs);

/* Replaces gpu/peel.cu:737 add_model.  The argument order is the one of the
 * reference's definition (peel.cu:737-740: ..., num_timesteps, num_freqs,
 * num_baselines), which is also how params/peel/gpu.rs:465-475 calls it;
 * gpu/peel.h:33 declares the last two the other way round. */
const char *add_model(JonesF32 *d_vis_residual, const JonesF32 *d_vis_model, const IonoConsts iono_consts,
                      const double *d_lambdas_m, const UVW *d_uvws, const int num_timesteps, const int num_freqs,
                      const int num_baselines);

/* Replaces gpu/utils.h:28 get_gpu_device_info (called by gpu/utils.rs:35-60
 * for the MODELLER string of the calibration solutions): makes `device`
 * current and reports its name, compute capability, global memory [bytes] and
 * the CUDA driver and runtime versions (1000 * major + 10 * minor).  NULL on
 * success, else a static error string. */
const char *get_gpu_device_info(int device, char name[256], int *device_major, int *device_minor,
                                size_t *total_global_mem, int *driver_version, int *runtime_version);

/* Drop-in error reporting.  The drop-in model_* calls read their kernels'
 * error word after the launch (a synchronous read on the legacy default
 * stream) and return one of these static strings instead of NULL when a
 * kernel reported a problem; the word is cleared first, so the next call
 * starts clean.  A kernel whose bounded wait ran out leaves the visibilities
 * of its baselines unchanged. */

/* ---------------------------------------------------------------------- */
/* Native layer                                                            */
/* ---------------------------------------------------------------------- */

#define HDC_OK 0
#define HDC_ERR_ARG 1
#define HDC_ERR_CUDA 2
#define HDC_ERR_ALLOC 3
#define HDC_ERR_TIMEOUT 4
#define HDC_ERR_UNSUPPORTED 5

/* A cudaStream_t without requiring the CUDA headers. NULL = legacy default. */
typedef struct CUstream_st *hdcStream_t;

/* Message for the last non-OK status on this thread ("" if none). */
const char *hdc_last_error(void);

/* Library and device description, e.g. for the solutions' MODELLER string
 * (di_calibrate/mod.rs:258-260; gpu/utils.cu:43-68). */
int hdc_device_info(char *buf, int buf_len);

/* Component type and flux-model codes of HdcSkyModel. */
#define HDC_POINT 0
#define HDC_GAUSSIAN 1
#define HDC_SHAPELET 2
#define HDC_FLUX_LIST 0
#define HDC_FLUX_POWER_LAW 1
#define HDC_FLUX_CURVED_POWER_LAW 2

/* A sky model as a struct of arrays over components (host memory), in the
 * reference's modelling order (srclist/types/components/mod.rs:169-272).
 * fds holds 5 doubles per entry (freq [Hz], I, Q, U, V) [Jy]; a component's
 * entries are fds[fd_start .. fd_start + fd_count).  (Curved) power laws have
 * one entry, the reference flux density.  Shapelet coefficients are
 * coeff_*[coeff_start .. coeff_start + coeff_count). */
typedef struct HdcSkyModel {
    int num_components;
    const int *comp_type;
    const double *ra;
    const double *dec;
    const double *maj;
    const double *min;
    const double *pa;
    const int *flux_type;
    const double *si;
    const double *q;
    const int *fd_start;
    const int *fd_count;
    const double *fds;
    const int *coeff_start;
    const int *coeff_count;
    const int *coeff_n1;
    const int *coeff_n2;
    const double *coeff_value;
} HdcSkyModel;

/* Beam used by the native modeller. */
#define HDC_BEAM_NONE 0          /* identity Jones (beam/mod.rs:255-388 NoBeam) */
#define HDC_BEAM_ANALYTIC_DIPOLE 1 /* 4x4 dipole tile over a ground plane, shared by all tiles */
#define HDC_BEAM_ANALYTIC_PER_TILE 2 /* the same tile with each tile's own dipole gains (hdc_modeller_set_tile_beams) */
#define HDC_BEAM_FEE 3               /* the MWA FEE beam per tile (hdc_modeller_set_fee_beam) */

/* Veto brightness of every source of a source list (srclist/veto.rs:58-129),
 * on the device: per coarse frequency h_freqs [Hz], the sum over a source's
 * components of the beam-attenuated flux density |(J I J^H)_XX| +
 * |(J I J^H)_YY| (I the component's instrumental flux at that frequency, J
 * the beam response at its Az/El for lst_rad and latitude_rad; beam_kind
 * HDC_BEAM_NONE or HDC_BEAM_ANALYTIC_DIPOLE).  h_brightness[s] is the
 * smallest of those sums over the frequencies, or -1 when one of the
 * source's components lies below min_elevation_rad or farther than
 * source_dist_cutoff_rad from the phase centre.  h_comp_source[c] is the
 * source index of component c of sky.  The caller sorts, thresholds and
 * keeps the top N as veto_sources does (Python: srclist_io.veto_sources). */
int hdc_source_brightness(const HdcSkyModel *sky, const int *h_comp_source, int num_sources, const double *h_freqs,
                          int num_freqs, double lst_rad, double latitude_rad, RADec phase_centre, int beam_kind,
                          double source_dist_cutoff_rad, double min_elevation_rad, double *h_brightness);

/* Precision form of the point-source predict. */
#define HDC_PREDICT_DIRECT 0     /* FP64 direct per-baseline kernel (the plain form) */
#define HDC_PREDICT_TENSOR 1     /* factored tcgen05 contraction (points only) */

/* Polarisations (context/mod.rs:26): 0 XX_XY_YX_YY, 1 XX, 2 YY, 3 XX_YY,
 * 4 XX_YY_XY. */

typedef struct HdcModeller HdcModeller;

/* new_sky_modeller / SkyModellerGpu::new (model/mod.rs:215-261,
 * model/gpu.rs:150-520) for the unflagged tiles and channels.  The tile XYZs
 * are used for every timestep unless hdc_modeller_set_tile_xyzs replaces them
 * (e.g. with precessed positions). */
int hdc_modeller_new(const HdcSkyModel *sky, int pols, const XYZ *h_unflagged_tile_xyzs, int num_tiles,
                     const double *h_freqs, int num_freqs, RADec phase_centre, double array_latitude_rad,
                     int beam_kind, int predict_form, HdcModeller **out);
void hdc_modeller_free(HdcModeller *m);

int hdc_modeller_set_tile_xyzs(HdcModeller *m, const XYZ *h_tile_xyzs);

/* Per-tile beams (BeamGpu::calc_jones_pair, beam/mod.rs:342-367): switch the
 * modeller to HDC_BEAM_ANALYTIC_PER_TILE with the amplitude of every dipole
 * of every tile, h_dipole_gains [tile][2][16] (X dipoles then Y dipoles,
 * row-major over the 4 x 4 grid from the south-west corner, 0 for a dead
 * dipole; a tile with all 16 at 1 has the HDC_BEAM_ANALYTIC_DIPOLE beam).
 * Tiles with equal gains share one beam (the reference's unique tiles); the
 * beam is evaluated per timestep at the nearest multiple of freq_res_hz of
 * each channel (1.28e6: the MWA coarse channels, the frequency resolution of
 * the reference's FEE beam), in the reference's [uniq_tile][uniq_freq]
 * [component] layout.  The direct form applies B_p S B_q^H per baseline; the
 * tensor form uses its block form (twice the components). */
int hdc_modeller_set_tile_beams(HdcModeller *m, const double *h_dipole_gains, double freq_res_hz);

/* ---------------------------------------------------------------------- */
/* MWA FEE beam on the device                                             */
/* ---------------------------------------------------------------------- */
/* The reference takes its per-tile beam Jones from mwa_hyperbeam 0.11.0's
 * FEE model (beam/fee.rs:307-369: FEEBeam::gpu_prepare(freqs, delays, gains,
 * norm_to_zenith = true), then calc_jones_device_pair_inner(az, za, latitude,
 * iau_order = false) into [uniq tile][uniq freq][direction], with the tile
 * and frequency maps and unique counts of beam/mod.rs:342-367).  The model
 * is the spherical-wave expansion of each dipole's embedded element pattern
 * (Sokolowski et al. 2017, PASA 34, e062).  HDF5 is not linked: the caller
 * reads the beam file (mwa_full_embedded_element_pattern.h5) and passes its
 * arrays here. */
typedef struct HdcFeeCoeffs {
    int num_freqs;                 /* frequencies of the file */
    const uint32_t *freqs_hz;      /* [num_freqs] */
    int num_modes;                 /* columns of the file's "modes" data set */
    const int32_t *modes;          /* [3][num_modes]: s (1 or 2), m, n of each column */
    const int32_t *num_freq_modes; /* [num_freqs]: columns of that frequency's data sets (the first ones of modes) */
    const double *q;               /* [num_freqs][2: X, Y][16 dipoles][num_modes][2]: complex coefficient (re, im)
                                      of each column; the file holds amplitude and phase [deg] */
} HdcFeeCoeffs;

typedef struct HdcFeeBeam HdcFeeBeam;

/* FEEBeam::gpu_prepare: each tile's dipole delays h_delays [num_tiles][16]
 * (steps of 435 ps; 32 marks a dead dipole, whose amplitudes become 0) and
 * amplitudes h_amps [num_tiles][num_amps] (num_amps 32: X dipoles then Y;
 * 16: the same for both), each of h_freqs_hz [num_freqs] taken at the file's
 * closest frequency.  Tiles with equal delays and amplitudes share one beam,
 * as do channels with the same closest frequency.  The dipole sums of every
 * unique (tile, frequency) are formed on the host and uploaded; with
 * norm_to_zenith each Jones element is divided by the magnitude of the
 * zenith-pointed (all delays 0, amplitudes 1) beam's element at zenith. */
int hdc_fee_beam_new(const HdcFeeCoeffs *file, const uint32_t *h_freqs_hz, int num_freqs, const uint32_t *h_delays,
                     const double *h_amps, int num_tiles, int num_amps, int norm_to_zenith, HdcFeeBeam **out);
void hdc_fee_beam_free(HdcFeeBeam *b);
/* BeamGpu::get_num_unique_tiles / get_num_unique_freqs / get_tile_map /
 * get_freq_map (beam/mod.rs:355-367); the maps are device pointers owned by
 * the beam ([num_tiles] and [num_freqs]). */
int hdc_fee_beam_num_unique_tiles(const HdcFeeBeam *b);
int hdc_fee_beam_num_unique_freqs(const HdcFeeBeam *b);
const int *hdc_fee_beam_tile_map(const HdcFeeBeam *b);
const int *hdc_fee_beam_freq_map(const HdcFeeBeam *b);
/* Host copies of the two maps (h_tile_map [num_tiles], h_freq_map
 * [num_freqs]; either may be NULL).  No counterpart in the reference. */
int hdc_fee_beam_host_maps(const HdcFeeBeam *b, int *h_tile_map, int *h_freq_map);
/* calc_jones_device_pair_inner (beam/fee.rs:330-349): for directions
 * d_az_rad, d_za_rad [num_directions] write d_jones [uniq tile][uniq freq]
 * [num_directions].  d_latitude_rad (a device pointer to one value, or NULL)
 * applies the parallactic-angle rotation; iau_order must be 0 (the order the
 * reference asks for).  Asynchronous on stream. */
int hdc_fee_calc_jones(const HdcFeeBeam *b, const double *d_az_rad, const double *d_za_rad, int num_directions,
                       const double *d_latitude_rad, int iau_order, JonesF64 *d_jones, hdcStream_t stream);
/* Use an FEE beam for every tile of the modeller (HDC_BEAM_FEE): its
 * per-tile Jones are evaluated per timestep at each component's Az/ZA, with
 * the parallactic rotation at the modeller's latitude.  The beam must have
 * been prepared for the modeller's channel frequencies and tile count, and
 * must stay alive while the modeller uses it. */
int hdc_modeller_set_fee_beam(HdcModeller *m, const HdcFeeBeam *b);
/* hdc_source_brightness with the FEE beam, as veto_sources evaluates it
 * (srclist/veto.rs:99-104: calc_jones with no tile, i.e. the observation's
 * ideal delays and unit gains, beam/fee.rs:287-292): beam is prepared for
 * one tile with those delays and gains and for the num_freqs frequencies
 * h_freqs. */
int hdc_source_brightness_fee(const HdcSkyModel *sky, const int *h_comp_source, int num_sources,
                              const double *h_freqs, int num_freqs, double lst_rad, double latitude_rad,
                              RADec phase_centre, const HdcFeeBeam *beam, double source_dist_cutoff_rad,
                              double min_elevation_rad, double *h_brightness);

/* SkyModeller::model_timestep_with at a given LMST (the device-level form the
 * reference's peel loop calls, model/gpu.rs:1152-1166): d_vis_fb [freq][bl]
 * is accumulated into (not cleared); h_uvws_out [bl] may be NULL. */
int hdc_modeller_model_timestep_with(HdcModeller *m, double lst_rad, JonesF32 *d_vis_fb, UVW *h_uvws_out,
                                     hdcStream_t stream);

/* As above with an FP64 visibility buffer (no f32 demotion; parity mode). */
int hdc_modeller_model_timestep_with_f64(HdcModeller *m, double lst_rad, JonesF64 *d_vis_fb, UVW *h_uvws_out,
                                         hdcStream_t stream);

/* SkyModeller::model_timestep_with with host buffers, as the trait is called
 * (model/gpu.rs:1476-1496): copies h_vis_fb in, accumulates, copies back. */
int hdc_modeller_model_timestep_with_host(HdcModeller *m, double lst_rad, JonesF32 *h_vis_fb, UVW *h_uvws_out,
                                          hdcStream_t stream);

/* SkyModeller::update_with_a_source (model/mod.rs:174): replace the sky model
 * and the phase centre. */
int hdc_modeller_update_with_a_source(HdcModeller *m, const HdcSkyModel *source, RADec phase_centre);

/* SkyModeller::model_timestep_autos_with (model/mod.rs:199): d_vis_fb is
 * [freq][tile], accumulated. */
int hdc_modeller_model_timestep_autos_with(HdcModeller *m, double lst_rad, JonesF32 *d_vis_fb, hdcStream_t stream);

/* Diagnostics.  Number of kernels libhdc has launched in this process. */
long long hdc_kernel_launches(void);

/* The static message for a kernel error word (bit 0: a bounded wait ran out,
 * HDC_ERR_TIMEOUT; bit 1: an index outside a table, HDC_ERR_ARG), NULL for 0.
 * Native calls return the status and leave the message in hdc_last_error();
 * a modeller's device calls are asynchronous, so its kernels' errors are
 * reported by its next call (the host-buffer call synchronises and reports
 * its own). */
const char *hdc_kernel_error_string(int word);

/* Failure-path testing (no counterpart in the reference): the next direct
 * predict kernel launched in this process issues none of its component-table
 * copies and gives each bounded wait wait_ns nanoseconds, so its first wait
 * runs out with nothing in flight; the call then reports HDC_ERR_TIMEOUT (or
 * the drop-in timeout string) and leaves its visibilities unchanged.  One
 * launch only; the library stays usable. */
int hdc_test_stall_next_predict(unsigned long long wait_ns);

/* Per-kernel-class device time of a modeller's last calls, measured with
 * CUDA events on the launching stream when profiling is enabled.
 * out_ms[0..3] = points, Gaussians, shapelets, geometry/beam prep [ms],
 * accumulated since the last reset. */
int hdc_modeller_set_profiling(HdcModeller *m, int enable);
int hdc_modeller_profile(HdcModeller *m, double *out_ms, int reset);

/* Achievable FP64 FMA rate of the current device [GFLOP/s], measured by a
 * register-resident FMA-chain kernel over all SMs (the FP64 roofline
 * denominator; a measurement, not a datasheet value). */
int hdc_probe_fp64_gflops(double *out_gflops);
/* The same for FP32 FMAs (the chosen form's direct kernels are FP32-bound). */
int hdc_probe_fp32_gflops(double *out_gflops);

/* Per-chanblock calibration outcome (di_calibrate/mod.rs:620-632). */
typedef struct HdcCalResult {
    int num_iterations;
    int converged;
    double max_precision;
    int num_failed;
} HdcCalResult;

#define HDC_CAL_PLAIN 0         /* stream data and model every iteration */
#define HDC_CAL_COLLAPSED 1     /* sum the timeblock's timesteps once into per-baseline covariances (FP64) */
#define HDC_CAL_COLLAPSED_F32 2 /* the same with covariances stored in FP32 (half the bytes per iteration) */

/* calibrate_timeblock (di_calibrate/mod.rs:387-618): calibrate every
 * chanblock of one timeblock, then re-calibrate failed chanblocks from
 * neighbour-interpolated starts until no more converge.  d_data_tfb and
 * d_model_tfb are [num_timesteps][num_chanblocks][num_baselines] (pre-weighted
 * as CalVis::scale_by_weights leaves them); the timeblock is timesteps
 * [timeblock_start, timeblock_end).  d_di_jones is this timeblock's
 * [tile][chanblock] slice of the solutions (model -> data, not inverted): the
 * initial guesses in, the solutions out (NaN where failed).  h_results gets
 * one entry per chanblock.  Up to 256 tiles. */
int hdc_calibrate_timeblock(const JonesF32 *d_data_tfb, const JonesF32 *d_model_tfb, int num_timesteps,
                            int timeblock_start, int timeblock_end, int num_chanblocks, int num_baselines,
                            JonesF64 *d_di_jones, int max_iterations, double stop_threshold, double min_threshold,
                            int pols, HdcCalResult *h_results, int form, hdcStream_t stream);

/* One pass of calibrate_timeblock without its retry of failed chanblocks:
 * every chanblock when h_chanblock_list is NULL, else only the num_listed
 * chanblocks it names (from their starts in d_di_jones; only their entries
 * of h_results are written).  The building block of a calibration whose
 * chanblocks are spread over several GPUs (mwa_hyperdrive_b200/shard.py):
 * each rank runs its chanblocks' first pass, the ranks exchange results,
 * and each re-runs its failed chanblocks from the neighbour-interpolated
 * starts (di_calibrate/mod.rs:473-614) formed over the whole band. */
int hdc_calibrate_chanblocks(const JonesF32 *d_data_tfb, const JonesF32 *d_model_tfb, int num_timesteps,
                             int timeblock_start, int timeblock_end, int num_chanblocks, int num_baselines,
                             JonesF64 *d_di_jones, int max_iterations, double stop_threshold, double min_threshold,
                             int pols, const int *h_chanblock_list, int num_listed, HdcCalResult *h_results, int form,
                             hdcStream_t stream);

/* All timeblocks (calibrate_timeblocks, di_calibrate/mod.rs:272-361): every
 * timeblock k = [h_timeblock_bounds[2k], h_timeblock_bounds[2k+1]) starts
 * from identity; the first pass of all timeblocks runs as one CUDA graph
 * (identity start, collapse, persistent MitchCal kernel per timeblock), then
 * failed chanblocks are retried per timeblock as in hdc_calibrate_timeblock.
 * d_di_jones [timeblock][tile][chanblock] gets the solutions, h_results
 * [timeblock][chanblock] the results. */
int hdc_calibrate_timeblocks(const JonesF32 *d_data_tfb, const JonesF32 *d_model_tfb, int num_timesteps,
                             const int *h_timeblock_bounds, int num_timeblocks, int num_chanblocks,
                             int num_baselines, JonesF64 *d_di_jones, int max_iterations, double stop_threshold,
                             double min_threshold, int pols, HdcCalResult *h_results, int form, hdcStream_t stream);

/* Per-chanblock calibration residual sum_{t,bl} ||D - G_p M G_q^H||_F^2 for
 * the gains d_di_jones [tile][chanblock] over timesteps
 * [timeblock_start, timeblock_end); h_residuals [num_chanblocks].  Used to
 * judge a proposed starting point for the solver against identity. */
int hdc_calibration_residuals(const JonesF32 *d_data_tfb, const JonesF32 *d_model_tfb, int num_timesteps,
                              int timeblock_start, int timeblock_end, int num_chanblocks, int num_baselines,
                              const JonesF64 *d_di_jones, double *h_residuals, hdcStream_t stream);

/* Learned warm start (no counterpart in the reference): a multilayer
 * perceptron trained and evaluated by this library's own FP32 kernels.
 * dims[0..num_layers] are the layer widths; hidden layers use ReLU, the
 * output layer is linear; if residual_offset >= 0 the output adds the input
 * slice starting there (width dims[num_layers]).  Parameters are laid out
 * per layer as W [out][in] then b [out]. */
typedef struct HdcMlp HdcMlp;
int hdc_mlp_new(int num_layers, const int *dims, int residual_offset, unsigned long long seed, HdcMlp **out);
void hdc_mlp_free(HdcMlp *m);
long long hdc_mlp_num_params(HdcMlp *m);
int hdc_mlp_get_params(HdcMlp *m, float *h_out);
int hdc_mlp_set_params(HdcMlp *m, const float *h_in);
/* d_x [batch][dims[0]] -> d_y [batch][dims[num_layers]] (device pointers) */
int hdc_mlp_forward(HdcMlp *m, const float *d_x, int batch, float *d_y, hdcStream_t stream);
/* Mean-squared-error loss and its gradient with respect to every parameter
 * (h_grads [num_params], may be NULL; h_loss may be NULL). */
int hdc_mlp_gradients(HdcMlp *m, const float *d_x, const float *d_target, int batch, float *h_grads,
                      double *h_loss, hdcStream_t stream);
/* One Adam step (beta1 0.9, beta2 0.999, eps 1e-8) on the MSE loss. */
int hdc_mlp_train_step(HdcMlp *m, const float *d_x, const float *d_target, int batch, float lr, double *h_loss,
                       hdcStream_t stream);

/* Warm-start chain on the device, one stream, no host synchronisation.
 * d_prev_tc [tile][chanblock] are the previous timeblock's solutions (NaN
 * where failed).  hdc_warmstart_features writes the network inputs d_x
 * [tile*chanblock][40] (FP32): per (tile, chanblock) the gauge-aligned
 * solutions at chanblocks c-2..c+2 in the frame of the centre's XX and YY
 * gains, band edges extrapolated through the centre.
 * hdc_warmstart_propose runs features, the network (40 inputs, 8 outputs)
 * and the mapping back to gains; with d_data_tfb and d_model_tfb non-NULL it
 * then judges every chanblock's proposal by its calibration residual over
 * the timeblock against the identity start and writes the chosen start to
 * d_start_tc [tile][chanblock] (d_use [chanblock], may be NULL: 1 where the
 * proposal was kept); with both NULL d_start_tc gets the proposal itself.
 * No counterpart in the reference (its solver starts from identity,
 * di_calibrate/mod.rs:283-287). */
int hdc_warmstart_features(const JonesF64 *d_prev_tc, int num_tiles, int num_chanblocks, float *d_x,
                           hdcStream_t stream);
/* The judge alone: per chanblock keep d_proposal_tc where its residual is
 * finite and no larger than the identity start's, else identity, into
 * d_start_tc (a different buffer); d_use as above. */
int hdc_warmstart_judge(const JonesF32 *d_data_tfb, const JonesF32 *d_model_tfb, int num_timesteps,
                        int timeblock_start, int timeblock_end, int num_chanblocks, int num_tiles,
                        const JonesF64 *d_proposal_tc, JonesF64 *d_start_tc, int *d_use, hdcStream_t stream);
int hdc_warmstart_propose(HdcMlp *mlp, const JonesF64 *d_prev_tc, int num_tiles, int num_chanblocks,
                          const JonesF32 *d_data_tfb, const JonesF32 *d_model_tfb, int num_timesteps,
                          int timeblock_start, int timeblock_end, JonesF64 *d_start_tc, int *d_use,
                          hdcStream_t stream);

/* Peel loop controls (PeelLoopParams and PeelWeightParams' consumers,
 * params/peel/mod.rs:207-224).  num_passes is the number of passes over all
 * sources, num_loops the iono-fit iterations per source.  (The reference's
 * peel_gpu destructures PeelLoopParams::get() with the two swapped,
 * gpu.rs:41; pass them swapped to reproduce that.) */
typedef struct HdcPeelParams {
    int num_passes;
    int num_loops;
    double convergence;
    int freq_average_factor; /* high-res channels per low-res channel */
    int beam_kind;           /* HDC_BEAM_* for the per-source models */
    double array_latitude_rad;
    int batch_size;          /* batched form: sources per sub-batch in list order (0: all in one) */
    const HdcFeeBeam *fee_beam; /* beam_kind HDC_BEAM_FEE: the beam, prepared for these tiles and channels */
} HdcPeelParams;

/* peel_gpu (params/peel/gpu.rs:25-757): peel num_sources sources from the
 * residual visibilities d_resid_tfb [t][f][bl] (in place, phase centre
 * `phase_centre`), weights d_weights_tfb [t][f][bl] (>= 0).  Source i is
 * h_sources[i] (its components) at weighted position h_source_positions[i];
 * h_iono_consts[i] holds its (alpha, beta, gain), read and updated.  Low-res
 * channel wavelengths use the mean frequency of each channel group; the
 * low-res UVWs use average_lmst (the timeblock's median LMST). */
int hdc_peel_timeblock(JonesF32 *d_resid_tfb, const float *d_weights_tfb, int num_timesteps, int num_freqs,
                       const double *h_freqs, const XYZ *h_tile_xyzs, int num_tiles, const double *h_lmsts,
                       double average_lmst, RADec phase_centre, int num_sources, const HdcSkyModel *h_sources,
                       const RADec *h_source_positions, IonoConsts *h_iono_consts, const HdcPeelParams *params,
                       hdcStream_t stream);

/* The same timeblock peeled with every source's fit of a pass batched
 * (this project's chosen form; no counterpart in the reference): one
 * accumulation sweep over the high-resolution residual for all sources of a
 * sub-batch, all their iono fits in one launch per iteration, one sweep
 * applying their updates.  Sources of one sub-batch see the residual as it
 * was when the sub-batch started (Jacobi) instead of each other's updates;
 * sub-batches follow one another in list order (the reference's
 * Gauss-Seidel order between them; params->batch_size sources each, 0 for
 * one sub-batch of all).  With one source, or sub-batches of one, this is
 * the reference's sequence.  Needs num_sources x (timesteps x channels x
 * baselines) JonesF32 of device memory for the source models unless every
 * source is one point at its own position. */
int hdc_peel_timeblock_batched(JonesF32 *d_resid_tfb, const float *d_weights_tfb, int num_timesteps, int num_freqs,
                               const double *h_freqs, const XYZ *h_tile_xyzs, int num_tiles, const double *h_lmsts,
                               double average_lmst, RADec phase_centre, int num_sources, const HdcSkyModel *h_sources,
                               const RADec *h_source_positions, IonoConsts *h_iono_consts, const HdcPeelParams *params,
                               hdcStream_t stream);

/* The accumulation-sweep launch shape the batched peel's autotuner chose for
 * the last new problem shape (low-resolution bins and sources per CTA;
 * sources 0: the variant staging 16 baselines' residual in shared memory for
 * every source) and its measured time. */
int hdc_peel_batched_tuning(int *block_bins, int *block_sources, float *ms);

/* ---- Visibility preparation before DI calibration ---------------------- */

/* CalVis::scale_by_weights (params/di_calibration.rs:578-625), in place on
 * the device: data and model [timestep][chanblock][baseline] are multiplied
 * by f64(weight) x d_baseline_weights[baseline] (NULL: 1) in FP64 and stored
 * back as FP32; where that product is <= 0 both become 0 (flagged). */
int hdc_scale_by_weights(JonesF32 *d_data_tfb, JonesF32 *d_model_tfb, const float *d_weights_tfb,
                         int num_timesteps, int num_chanblocks, int num_baselines, const double *d_baseline_weights,
                         hdcStream_t stream);

/* vis_average (averaging/mod.rs:537-600) on the device: all num_timesteps of
 * d_from_tfb / d_weights_from_tfb [timestep][freq][baseline] averaged into
 * d_to_fb / d_weights_to_fb [chanblock][baseline].  The channels split into
 * num_chanblocks + num_flagged chunks of ceil(num_freqs / (num_chanblocks +
 * num_flagged)) channels; chunks listed in h_flagged_chanblocks are skipped
 * and the others fill the outputs in order.  Each output is the FP64
 * weight-weighted mean of its samples with weight > 0 and their weight sum,
 * or, where no weight is > 0, the plain mean and minus the sum of |weight|
 * (vis_average_weights_non_zero, averaging/mod.rs:606-648); results are the
 * reference's bit for bit.  At most 8000 flagged of at most 65536 chunks
 * (the reference's u16 chanblock indices); h_flagged_chanblocks in any
 * order.  Asynchronous on stream; allocates nothing. */
int hdc_vis_average(const JonesF32 *d_from_tfb, const float *d_weights_from_tfb, int num_timesteps, int num_freqs,
                    int num_baselines, const int *h_flagged_chanblocks, int num_flagged, JonesF32 *d_to_fb,
                    float *d_weights_to_fb, int num_chanblocks, hdcStream_t stream);

/* into_cal_sols (di_calibrate/mod.rs:89-176) on the device: the solver's
 * model->data gains d_di_jones [timeblock][unflagged tile][unflagged
 * chanblock] become the data->model solutions d_out [timeblock][tile]
 * [chanblock] of all num_unflagged + num_flagged tiles and chanblocks: each
 * Jones matrix inverted (marlu Jones::inv; for pols XX or YY only that
 * entry, inverted as a complex number, the others 0), NaN for flagged tiles
 * and chanblocks.  Flag lists in any order, at most 1024 tiles and 8000
 * chanblocks.  Asynchronous on stream; allocates nothing. */
int hdc_into_cal_sols(const JonesF64 *d_di_jones, int num_timeblocks, int num_unflagged_tiles,
                      int num_unflagged_chanblocks, const int *h_flagged_tiles, int num_flagged_tiles,
                      const int *h_flagged_chanblocks, int num_flagged_chanblocks, int pols, JonesF64 *d_out,
                      hdcStream_t stream);

#ifdef __cplusplus
} /* extern "C" */
#endif
