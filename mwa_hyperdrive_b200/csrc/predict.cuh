// Direct FP64 predictor kernels (shared by the drop-in entry points and the
// native modeller).
#pragma once

#include "common.cuh"

namespace hdc {

// Per-type component tables consumed by the direct kernel.  Component order
// is the modelling order; for the drop-in layer it is power laws, curved
// power laws, lists (gpu/types.h:187-267), which is also the beam-direction
// order of d_beam_jones.
constexpr int SDN = SDN_TABLE;  // orders 0..5 in the dense shapelet form

struct DirectParams {
    int nbl, nf, ntiles, nc;
    const double* freqs;  // [nf] Hz
    const UVW* uvws;      // [nbl] m
    const double4* lmn;   // [nc] (l, m, n - 1, 0), dimensionless (turn units)
    const JonesF64* flux; // [nf][nc]: B S B^H when the beam is shared (or none), S when per tile
    const double4* gp;    // [nc] Gaussian: (C maj^2, C min^2, sin pa, cos pa); shapelet: (maj K, -min K, sin pa, cos pa)
    // per-tile beam, reference layout [uniq_tile][uniq_freq][nc]
    const JonesF64* beam;
    const int* tile_map;
    const int* unflagged_map;
    const int* freq_map;
    int n_uniq_freq;
    int n_uniq_tile;  // rows of beam (the chosen form's per-tile kernel stages them; 0: not known)
    // shapelets
    const double* sbf;  // [SBF_N][SBF_L]
    const float* sbf32; // the same table in FP32 (chosen form), or NULL
    // chosen form, orders below SDN: the table as FP32 (value, next - value)
    // pairs, position-major [SBF_L][SDN / 2] float4, and per component a dense SDN x SDN coefficient
    // matrix [nc][n1][n2] with the sign of i^(n1+n2) folded in; NULL when
    // some coefficient's order is SDN or more
    const float4* sbfp;
    const float* sdense;
    const ShapeletCoeff* coeffs;
    const int* coeff_start;
    const int* coeff_count;
    const ShapeletUV* suv_bl;  // [nbl][nc] m, or NULL
    const double2* suv_tile;   // [nc][ntiles] m, or NULL (then suv = tile1 - tile2)
    void* vis;                 // [nf][nbl] JonesF32 or JonesF64, accumulated
    int* err;
    // Limit of each bounded wait on the staged tables [ns] (0: the default
    // 2 s).  stall != 0 (set only through hdc_test_stall_next_predict) issues
    // none of the table copies, so that the first wait runs out with nothing
    // in flight.
    unsigned long long wait_ns;
    int stall;
};

// Static message for a kernel error word (KERR_* bits), NULL for 0.
const char* kernel_error_string(int word);
// Status code of a kernel error word for the native layer (HDC_OK for 0).
int kernel_error_status(int word);

// Launch the direct kernel for component type ty (0 point, 1 Gaussian,
// 2 shapelet).  tile_beam selects per-tile beam Jones; out64 an FP64 output;
// fast the FP32 form (errors ~1e-7 of the visibility; shared beam only).
cudaError_t launch_direct(int ty, bool tile_beam, bool out64, const DirectParams& p, cudaStream_t s,
                          bool fast = false);

// Per-tile beams for the tensor-core predict: beam [n_uniq_tile]
// [n_uniq_freq][nc] (the reference's layout), the unique row of every tile
// (any unflagged-tile map already applied) and the unique column of every
// channel of the launch.
struct TensorBeam {
    const JonesF64* beam;
    const JonesF32* beam32;  // the same table in FP32 (the producers' reads), or NULL
    const int* tile_map;
    const int* freq_map;
    int n_uniq_tile;
    int n_uniq_freq;
};

// A second stream and its events, with which the tensor predict of a shared
// beam writes the next chunk's table while the Gram kernel of the current
// chunk runs (two tables in the workspace).  One per caller: not shared
// between concurrent calls.
struct TensorSync {
    cudaStream_t ts = nullptr;
    cudaEvent_t start = nullptr, table_done[2] = {nullptr, nullptr}, gram_done[2] = {nullptr, nullptr};
};
int tensor_sync_init(TensorSync& t);
void tensor_sync_free(TensorSync& t);

// The tensor-core point predict of one timestep (csrc/tensor.cu): d_W is
// B S B^H [nf][nc] with a beam shared by all tiles (beam NULL), or S [nf][nc]
// with per-tile beams.  ws: tensor_workspace_bytes(nf, nbl, ntiles, nc,
// per-tile beams, out64, sync != NULL) bytes; sync NULL runs every kernel
// on s in turn.
size_t tensor_workspace_bytes(int nf, int nbl, int ntiles, int nc, bool tile_beam, bool out64, bool two_tables);
// Per-chunk output of the table form (shared beam, nc <= tensor_single_pass()
// components, JonesF32 output): after the Gram products of channels
// [f0, f0 + nch) the chunk's visibilities become vis + model + planes (model:
// [nf][nbl], added before the planes), and done(ctx, f0, nch) is called to
// queue the chunk's further work on s; no whole-array combine follows.
struct TensorChunkOut {
    const JonesF32* model;
    int (*done)(void* ctx, int f0, int nch);
    void* ctx;
};
int tensor_single_pass();
int launch_tensor_points(int nf, int nbl, int ntiles, int nc, const double* d_freqs, const XYZ* d_xyzs, double ha,
                         double dec, const double4* d_lmn, const JonesF64* d_W, const TensorBeam* beam, void* d_vis,
                         bool out64, void* ws, int* d_err, cudaStream_t s, TensorSync* sync,
                         const TensorChunkOut* chunk_out = nullptr);

struct AutosParams {
    int ntiles, nf;
    int nc_total;
    // up to 3 type tables concatenated by the caller into one [nf][nc] flux
    // table (S) and a beam table [uniq_tile][uniq_freq][nc] (NULL: identity)
    const JonesF64* flux;
    const JonesF64* beam;
    const int* tile_map;
    const int* unflagged_map;
    const int* freq_map;
    int n_uniq_freq;
    int n_uniq_tile;  // rows of beam (the chosen form's per-tile kernel stages them; 0: not known)
    JonesF32* vis;  // [nf][ntiles]
};
cudaError_t launch_autos(const AutosParams& p, cudaStream_t s);

// mask_pols over a [n] JonesF32 buffer (model/mod.rs:264-285)
cudaError_t launch_mask_pols(JonesF32* vis, size_t n, int pols, cudaStream_t s);

}  // namespace hdc
