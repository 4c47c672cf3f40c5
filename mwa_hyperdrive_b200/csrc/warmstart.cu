// Learned warm start for DI calibration, device side (this project's
// addition; mwa_hyperdrive's solver starts every timeblock from identity,
// di_calibrate/mod.rs:283-287).  The whole chain from the previous
// timeblock's solutions to the judged starting gains runs on one stream
// with no host synchronisation:
//
//   1. align_frame_kernel: per chanblock, rotate all solutions by the phase
//      that makes tile 0's XX real and positive (the solutions' free phase);
//      non-finite solutions become identity; the frame of each (tile,
//      chanblock) is its aligned XX and YY gains (1 where either is
//      non-finite or below 1e-6 in modulus).
//   2. features_kernel: for each (tile, chanblock) the aligned solutions at
//      chanblocks c-2 .. c+2 right-multiplied by diag(1/a, 1/d), a and d the
//      centre's frame; neighbours beyond the band edge continue the line
//      through the centre and the mirrored in-band neighbour (2 N_0 - N_-j).
//      40 FP32 inputs per (tile, chanblock).
//   3. the network's forward pass (hdc_mlp_forward, same stream).
//   4. denorm_kernel: proposal = output diag(a, d); non-finite entries are
//      replaced by the identity's.
//   5. judge (calibrate.cu): per chanblock, the proposal is kept where its
//      calibration residual over the timeblock is finite and no larger than
//      the identity start's; otherwise that chanblock starts from identity.
//
// The host-side restatement of steps 1, 2 and 4 (numpy, used to build
// training sets) is mwa_hyperdrive_b200/warmstart.py; the tests hold the two
// to each other.

#include "common.cuh"

namespace hdc {

int mlp_io_dims(HdcMlp* m, int* in, int* out);
int launch_judge(const JonesF32* d_data, const JonesF32* d_model, int t0, int t1, int nchan, int nbl, int ntiles,
                 const JonesF64* d_prop, JonesF64* d_start, int* d_use, cudaStream_t s);

namespace ws {

constexpr int NB = 2;               // neighbouring chanblocks on each side
constexpr int IN = 8 * (2 * NB + 1);
constexpr int OUT = 8;

__device__ __forceinline__ bool finite8(const double* v) {
    bool ok = true;
#pragma unroll
    for (int k = 0; k < 8; k++) ok = ok && isfinite(v[k]);
    return ok;
}

// aligned [tile][chanblock][8], frame [tile][chanblock] = (a re, a im, d re, d im)
__global__ void align_frame_kernel(const JonesF64* __restrict__ prev, int ntiles, int nchan,
                                   double* __restrict__ aligned, double4* __restrict__ frame) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ntiles * nchan) return;
    const int c = i % nchan;
    const JonesF64 r = prev[c];  // tile 0, this chanblock
    const double ax = hypot(r.j00_re, r.j00_im);
    cplx ph = {1.0, 0.0};
    if (ax > 0.0) {  // false for NaN
        const double m = fmax(ax, 1e-300);
        ph = {r.j00_re / m, -r.j00_im / m};
    }
    const double* s = reinterpret_cast<const double*>(prev + i);
    double v[8];
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const double re = s[2 * k], im = s[2 * k + 1];
        v[2 * k] = re * ph.re - im * ph.im;
        v[2 * k + 1] = re * ph.im + im * ph.re;
    }
    if (!finite8(v)) {
#pragma unroll
        for (int k = 0; k < 8; k++) v[k] = (k == 0 || k == 6) ? 1.0 : 0.0;
    }
#pragma unroll
    for (int k = 0; k < 8; k++) aligned[(size_t)i * 8 + k] = v[k];
    const bool ok = isfinite(v[0]) && isfinite(v[1]) && isfinite(v[6]) && isfinite(v[7]) &&
                    hypot(v[0], v[1]) > 1e-6 && hypot(v[6], v[7]) > 1e-6;
    frame[i] = ok ? make_double4(v[0], v[1], v[6], v[7]) : make_double4(1.0, 0.0, 1.0, 0.0);
}

__device__ __forceinline__ cplx crecip(double re, double im) {
    const double d = re * re + im * im;
    return {re / d, -im / d};
}

// J diag(ca, cd): columns 0 (xx, yx) times ca, column 1 (xy, yy) times cd
__device__ __forceinline__ void scale_cols(const double* p, cplx ca, cplx cd, double* o) {
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const cplx f = (k == 0 || k == 2) ? ca : cd;
        const double re = p[2 * k], im = p[2 * k + 1];
        o[2 * k] = re * f.re - im * f.im;
        o[2 * k + 1] = re * f.im + im * f.re;
    }
}

// one thread per (tile, chanblock, neighbour j in 0..4)
__global__ void features_kernel(const double* __restrict__ aligned, const double4* __restrict__ frame, int ntiles,
                                int nchan, float* __restrict__ x) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= ntiles * nchan * (2 * NB + 1)) return;
    const int j = g % (2 * NB + 1);
    const int i = g / (2 * NB + 1);
    const int tile = i / nchan, c = i % nchan;
    const double4 fr = frame[i];
    const cplx ia = crecip(fr.x, fr.y), id = crecip(fr.z, fr.w);
    const double* row = aligned + (size_t)tile * nchan * 8;
    const int raw = c + j - NB;
    double n[8];
    if (raw >= 0 && raw < nchan) {
        scale_cols(row + (size_t)raw * 8, ia, id, n);
    } else {
        const int mir = min(max(2 * c - raw, 0), nchan - 1);
        double cen[8], m[8];
        scale_cols(row + (size_t)c * 8, ia, id, cen);
        scale_cols(row + (size_t)mir * 8, ia, id, m);
#pragma unroll
        for (int k = 0; k < 8; k++) n[k] = 2.0 * cen[k] - m[k];
    }
    float* o = x + (size_t)i * IN + 8 * j;
#pragma unroll
    for (int k = 0; k < 8; k++) o[k] = (float)n[k];
}

// proposal [tile][chanblock] = y diag(a, d), non-finite entries -> identity's
__global__ void denorm_kernel(const float* __restrict__ y, const double4* __restrict__ frame, int n,
                              JonesF64* __restrict__ prop) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double4 fr = frame[i];
    double v[8], o[8];
#pragma unroll
    for (int k = 0; k < 8; k++) v[k] = (double)y[(size_t)i * OUT + k];
    scale_cols(v, cplx{fr.x, fr.y}, cplx{fr.z, fr.w}, o);
#pragma unroll
    for (int k = 0; k < 8; k++)
        if (!isfinite(o[k])) o[k] = (k == 0 || k == 6) ? 1.0 : 0.0;
    double* d = reinterpret_cast<double*>(prop + i);
#pragma unroll
    for (int k = 0; k < 8; k++) d[k] = o[k];
}

// stream-ordered scratch for one call
struct Scratch {
    cudaStream_t s;
    void* p = nullptr;
    explicit Scratch(cudaStream_t st) : s(st) {}
    ~Scratch() {
        if (p) cudaFreeAsync(p, s);
    }
};

int features(const JonesF64* d_prev, int ntiles, int nchan, float* d_x, double* d_aligned, double4* d_frame,
             cudaStream_t s) {
    const int n = ntiles * nchan;
    align_frame_kernel<<<(n + 255) / 256, 256, 0, s>>>(d_prev, ntiles, nchan, d_aligned, d_frame);
    const int nf = n * (2 * NB + 1);
    features_kernel<<<(nf + 255) / 256, 256, 0, s>>>(d_aligned, d_frame, ntiles, nchan, d_x);
    count_launches(2);
    HDC_CUDA_RET_INT(cudaGetLastError());
    return HDC_OK;
}

}  // namespace ws
}  // namespace hdc

using namespace hdc;

extern "C" int hdc_warmstart_features(const JonesF64* d_prev_tc, int num_tiles, int num_chanblocks, float* d_x,
                                      hdcStream_t stream) {
    if (!d_prev_tc || !d_x || num_tiles < 2 || num_chanblocks < 1) {
        set_error("hdc_warmstart_features: invalid arguments");
        return HDC_ERR_ARG;
    }
    cudaStream_t s = (cudaStream_t)stream;
    const size_t n = (size_t)num_tiles * num_chanblocks;
    ws::Scratch sc(s);
    HDC_CUDA_RET_INT(pool_malloc_async(&sc.p, n * (8 * sizeof(double) + sizeof(double4)), s));
    double* aligned = static_cast<double*>(sc.p);
    double4* frame = reinterpret_cast<double4*>(aligned + n * 8);
    return ws::features(d_prev_tc, num_tiles, num_chanblocks, d_x, aligned, frame, s);
}

extern "C" int hdc_warmstart_judge(const JonesF32* d_data_tfb, const JonesF32* d_model_tfb, int num_timesteps,
                                   int timeblock_start, int timeblock_end, int num_chanblocks, int num_tiles,
                                   const JonesF64* d_proposal_tc, JonesF64* d_start_tc, int* d_use,
                                   hdcStream_t stream) {
    if (!d_data_tfb || !d_model_tfb || !d_proposal_tc || !d_start_tc || d_proposal_tc == d_start_tc ||
        num_tiles < 2 || num_tiles > 256 || num_chanblocks < 1 || timeblock_start < 0 ||
        timeblock_end > num_timesteps || timeblock_start >= timeblock_end) {
        set_error("hdc_warmstart_judge: invalid arguments");
        return HDC_ERR_ARG;
    }
    return launch_judge(d_data_tfb, d_model_tfb, timeblock_start, timeblock_end, num_chanblocks,
                        num_tiles * (num_tiles - 1) / 2, num_tiles, d_proposal_tc, d_start_tc, d_use,
                        (cudaStream_t)stream);
}

extern "C" int hdc_warmstart_propose(HdcMlp* mlp, const JonesF64* d_prev_tc, int num_tiles, int num_chanblocks,
                                     const JonesF32* d_data_tfb, const JonesF32* d_model_tfb, int num_timesteps,
                                     int timeblock_start, int timeblock_end, JonesF64* d_start_tc, int* d_use,
                                     hdcStream_t stream) {
    int din = 0, dout = 0;
    if (!mlp || !d_prev_tc || !d_start_tc || num_tiles < 2 || num_tiles > 256 || num_chanblocks < 1 ||
        mlp_io_dims(mlp, &din, &dout) != HDC_OK || din != ws::IN || dout != ws::OUT) {
        set_error("hdc_warmstart_propose: invalid arguments (network must map %d inputs to %d outputs)", ws::IN,
                  ws::OUT);
        return HDC_ERR_ARG;
    }
    const bool judge = d_data_tfb && d_model_tfb;
    if (judge && (timeblock_start < 0 || timeblock_end > num_timesteps || timeblock_start >= timeblock_end)) {
        set_error("hdc_warmstart_propose: invalid timeblock");
        return HDC_ERR_ARG;
    }
    cudaStream_t s = (cudaStream_t)stream;
    const size_t n = (size_t)num_tiles * num_chanblocks;
    ws::Scratch sc(s);
    const size_t bytes = n * (8 * sizeof(double) + sizeof(double4) + sizeof(float) * (ws::IN + ws::OUT)) +
                         (judge ? n * sizeof(JonesF64) : 0);
    HDC_CUDA_RET_INT(pool_malloc_async(&sc.p, bytes, s));
    double* aligned = static_cast<double*>(sc.p);
    double4* frame = reinterpret_cast<double4*>(aligned + n * 8);
    float* x = reinterpret_cast<float*>(frame + n);
    float* y = x + n * ws::IN;
    JonesF64* prop = judge ? reinterpret_cast<JonesF64*>(y + n * ws::OUT) : d_start_tc;
    int rc = ws::features(d_prev_tc, num_tiles, num_chanblocks, x, aligned, frame, s);
    if (rc) return rc;
    rc = hdc_mlp_forward(mlp, x, (int)n, y, stream);
    if (rc) return rc;
    ws::denorm_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(y, frame, (int)n, prop);
    count_launches(1);
    HDC_CUDA_RET_INT(cudaGetLastError());
    if (!judge) return HDC_OK;
    const int nbl = num_tiles * (num_tiles - 1) / 2;
    return launch_judge(d_data_tfb, d_model_tfb, timeblock_start, timeblock_end, num_chanblocks, nbl, num_tiles,
                        prop, d_start_tc, d_use, s);
}
