// Native modeller state (host side).
#pragma once

#include <vector>

#include "predict.cuh"

namespace hdc {

struct TypeTables {
    int nc = 0;
    double4* d_lmn = nullptr;    // [nc]
    JonesF64* d_S = nullptr;     // [nf][nc] instrumental flux
    JonesF64* d_W = nullptr;     // [nf][nc] B S B^H (beam set)
    double4* d_gp = nullptr;     // [nc]
    double2* d_radec = nullptr;  // [nc]
    ShapeletCoeff* d_coeffs = nullptr;
    int* d_cstart = nullptr;
    int* d_ccount = nullptr;
    double2* d_suv_tile = nullptr;  // [nc][ntiles]
    float* d_sdense = nullptr;      // [nc][SDN][SDN] signed dense coefficients, or NULL
    JonesF64* d_B = nullptr;        // per-tile beams: [uniq tile][uniq freq][nc] at the current timestep
    JonesF32* d_B32 = nullptr;      // the same in FP32 (points in the tensor form: its producers' reads)
    void release();
};

// Per-tile analytic beams (hdc_modeller_set_tile_beams): the dipole gains of
// every distinct tile, the unique row of each tile, the beam frequencies and
// the unique column of each channel.
struct TileBeams {
    int n_uniq_tile = 0, n_uniq_freq = 0;
    double* d_gains = nullptr;      // [uniq tile][2][16]
    int* d_tile_map = nullptr;      // [tile]
    double* d_freqs = nullptr;      // [uniq freq] Hz
    int* d_freq_map = nullptr;      // [channel]
    const HdcFeeBeam* fee = nullptr;  // HDC_BEAM_FEE: the caller's beam (the maps above are copies of its maps)
    void release();
};

// The FEE beam's per-timestep evaluation for the modeller (csrc/fee.cu):
// Jones [uniq tile][uniq freq][n] of the directions d_radec at the LST, with
// the parallactic rotation at latitude lat.
int fee_launch_radec(const HdcFeeBeam* b, const double2* d_radec, int n, double lst, double lat, JonesF64* d_out,
                     cudaStream_t s);
int fee_num_tiles(const HdcFeeBeam* b);
int fee_num_freqs(const HdcFeeBeam* b);
int fee_device(const HdcFeeBeam* b);
// A peel loop's per-source modeller (direct FP64 form) with the loop's beam:
// params->beam_kind, or the FEE beam params->fee_beam.
int peel_modeller_new(const HdcSkyModel* sky, const XYZ* h_xyzs, int num_tiles, const double* h_freqs, int num_freqs,
                      RADec phase_centre, const HdcPeelParams* params, HdcModeller** out);

struct TensorState;

struct Modeller {
    int device = 0;
    int pols = 0, ntiles = 0, nbl = 0, nf = 0, beam_kind = 0, form = 0;
    RADec pc{0, 0};
    double lat = 0;
    std::vector<double> freqs;
    std::vector<XYZ> xyzs;
    double* d_freqs = nullptr;
    XYZ* d_xyzs = nullptr;
    UVW* d_uvws = nullptr;
    const double* d_sbf = nullptr;
    // This modeller's kernel error word, its pinned host copy and the event
    // after the last copy: each call queues a copy of the word behind its
    // kernels; a call that finds an earlier copy completed and set reports it
    // (calls on the device are asynchronous, so an error surfaces at the next
    // call, or at the end of the host-buffer call, which synchronises).
    int* d_err = nullptr;
    int* h_err = nullptr;
    cudaEvent_t err_ev = nullptr;
    int queue_error_check(cudaStream_t s);
    int take_error(bool wait);
    TypeTables t[3];
    TileBeams tb;  // set when beam_kind == HDC_BEAM_ANALYTIC_PER_TILE or HDC_BEAM_FEE
    JonesF32* d_host_vis = nullptr;
    size_t host_vis_bytes = 0;
    JonesF32* d_host_model = nullptr;  // host-buffer call: Gaussians + shapelets staged here
    size_t host_model_bytes = 0;
    TensorState* tc = nullptr;

    // Optional CUDA-event timing of each kernel class on the launching stream:
    // class 0..2 = the per-type predict kernels, 3 = geometry/beam prep.
    bool profiling = false;
    struct EvPair {
        cudaEvent_t a, b;
        int cls;
    };
    std::vector<EvPair> ev_pending, ev_free;
    double prof_ms[4] = {0, 0, 0, 0};
    void prof_begin(int cls, cudaStream_t s, EvPair& e);
    void prof_end(cudaStream_t s, EvPair& e);
    void prof_collect();

    int build_tables(const HdcSkyModel* sky);
    bool tile_beams() const { return beam_kind == HDC_BEAM_ANALYTIC_PER_TILE || beam_kind == HDC_BEAM_FEE; }
    int set_tile_beams(const double* h_gains, double freq_res_hz);
    int set_fee_beam(const HdcFeeBeam* b);
    int alloc_tile_beam_tables();
    int geometry(double lst, cudaStream_t s);
    const JonesF64* weights(int ty) const;
    DirectParams direct_params(int ty, void* vis) const;
    int model(double lst, void* d_vis, bool out64, UVW* h_uvws, cudaStream_t s);
    // the predict kernels of channels [f0, f0 + nfc) after geometry(); d_vis
    // is the whole [nf][nbl] visibility array.  Classes (types bit-set: 1
    // points, 2 Gaussians, 4 shapelets) are added in the reference's order,
    // or Gaussians, shapelets, points in the tensor form; the pol mask
    // follows when mask is set.
    int model_channels(double lst, void* d_vis, bool out64, int f0, int nfc, cudaStream_t s, int types = 7,
                       bool mask = true);
    // host-buffer predict: upload, predict and download of channel chunks
    // overlap on three streams
    static constexpr int PIPE_CHUNKS = 5;
    cudaStream_t pipe_s[3] = {nullptr, nullptr, nullptr};
    cudaEvent_t pipe_ev[2 * PIPE_CHUNKS + 2] = {};
    int model_host_pipelined(double lst, JonesF32* h_vis, UVW* h_uvws, cudaStream_t s);
    // the same for the tensor form with a shared beam: Gaussians and
    // shapelets over all channels into d_host_model while the buffer
    // uploads, then the points chunk by chunk, each chunk downloaded as soon
    // as its points are in
    int model_host_points_last(double lst, JonesF32* h_vis, UVW* h_uvws, cudaStream_t s);
    // rc, after waiting for the pipeline's streams when rc reports an error
    int host_call_drained(int rc);
    // model_timestep_with over baseline UVWs the caller computed (as the
    // reference's peel loop passes its own d_uvws, model/gpu.rs:1152-1166);
    // direct FP64 kernels, JonesF32 output.
    int model_uvws(double lst, const UVW* d_uvws_ext, JonesF32* d_vis, cudaStream_t s);
    int autos(double lst, JonesF32* d_vis, cudaStream_t s);
    int tensor_setup();
    void* tensor_workspace(bool out64);
    TensorSync* tensor_sync();  // the tensor predict's second stream (NULL: none)
    void tensor_release();
    ~Modeller();
};

}  // namespace hdc
