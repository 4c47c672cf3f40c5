// Visibility preparation before DI calibration, on the device:
//
// * hdc_scale_by_weights -- CalVis::scale_by_weights
//   (params/di_calibration.rs:578-625): data and model are multiplied by
//   their visibility weight (times an optional per-baseline weight) in FP64
//   and stored back as FP32; a weight <= 0 zeroes both (flagged).
// * hdc_vis_average -- vis_average and vis_average_weights_non_zero
//   (averaging/mod.rs:537-648): one time chunk of visibilities and weights
//   [time][channel][baseline] averaged into [chanblock][baseline]; channel
//   chunks of ceil(channels / (chanblocks + flagged)) channels, the flagged
//   chunks skipped; per output the weight-weighted FP64 mean of the samples
//   with positive weight and their weight sum, or, if none is positive, the
//   plain mean and minus the sum of |weight|.
//
// Both stream their inputs once (HBM-bound); sums run in the reference's order (time outer, channel
// inner) so the FP32 results are the reference's bit for bit.

#include <vector>

#include "common.cuh"
#include "flagtable.cuh"

namespace hdc {
namespace vp {

__global__ void scale_kernel(JonesF32* __restrict__ data, JonesF32* __restrict__ model,
                             const float* __restrict__ weights, const double* __restrict__ bl_weights, size_t n,
                             int nbl) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double w = (double)weights[i] * (bl_weights ? bl_weights[i % nbl] : 1.0);
    float4* d = reinterpret_cast<float4*>(data + i);
    float4* m = reinterpret_cast<float4*>(model + i);
    if (w <= 0.0) {
        const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
        d[0] = z, d[1] = z, m[0] = z, m[1] = z;
        return;
    }
    auto sc = [w](float4 v) {
        return make_float4((float)((double)v.x * w), (float)((double)v.y * w), (float)((double)v.z * w),
                           (float)((double)v.w * w));
    };
    const float4 d0 = d[0], d1 = d[1], m0 = m[0], m1 = m[1];
    d[0] = sc(d0), d[1] = sc(d1), m[0] = sc(m0), m[1] = sc(m1);
}

// The flagged chanblocks travel in the launch's parameters (FlagTable, no
// device table) as g[k] = flagged[k] - k over the ascending flagged indices,
// so output o takes chunk o + #{k : g[k] <= o}.
constexpr int FLAG_CAP_SMALL = 256;
constexpr int FLAG_CAP = 8000;  // 16 KB of launch parameters (the limit is 32764 bytes)

// Two threads per (output chanblock, baseline): each sums one half of the
// Jones matrix ([XX, XY] or [YX, YY], one float4) and both read the weight
// (one transaction).  The
// (time, channel) samples are taken in batches of PF whose loads are all
// issued before the first is summed, so each thread keeps PF loads in flight;
// the sums still run in (time, channel) order.
constexpr int PF = 4;
constexpr int AVG_THREADS = 256;

template <int CAP>
__global__ void __launch_bounds__(AVG_THREADS) average_kernel(const JonesF32* __restrict__ from,
                                                              const float* __restrict__ wfrom, int nt, int nf,
                                                              int nbl, int avg_freq,
                                                              const __grid_constant__ FlagTable<CAP> tab, int nout,
                                                              JonesF32* __restrict__ to, float* __restrict__ wto) {
    const size_t tid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const size_t g = tid >> 1;
    const int half = (int)(tid & 1);
    if (g >= (size_t)nout * nbl) return;
    const int bl = (int)(g % nbl), o = (int)(g / nbl);
    const int f0 = (o + flag_count_le(tab, o)) * avg_freq, f1 = min(f0 + avg_freq, nf);
    const int navg = f1 - f0, total = nt * navg;
    double ws[4] = {0, 0, 0, 0}, s[4] = {0, 0, 0, 0};
    double wsum = 0.0, fsum = 0.0;
    bool all_flagged = true;
    int t = 0, f = f0;  // (time, channel) of the next sample to load
    for (int k0 = 0; k0 < total; k0 += PF) {
        float4 a[PF];
        float w[PF];
#pragma unroll
        for (int j = 0; j < PF; j++) {
            if (k0 + j < total) {
                const size_t i = ((size_t)t * nf + f) * nbl + bl;
                a[j] = __ldcs(reinterpret_cast<const float4*>(from + i) + half);
                w[j] = __ldcs(wfrom + i);
                if (++f == f1) f = f0, t++;
            }
        }
#pragma unroll
        for (int j = 0; j < PF; j++) {
            if (k0 + j < total) {
                const double v[4] = {a[j].x, a[j].y, a[j].z, a[j].w};
                const double wa = fabs((double)w[j]);
#pragma unroll
                for (int k = 0; k < 4; k++) s[k] += v[k];
                if (w[j] > 0.f) {
                    all_flagged = false;
#pragma unroll
                    for (int k = 0; k < 4; k++)
                        ws[k] = __dadd_rn(ws[k], __dmul_rn(v[k], wa));  // no FMA: rounds as the reference
                    wsum += wa;
                } else {
                    fsum += wa;
                }
            }
        }
    }
    float r[4];
    float wr;
    if (all_flagged || wsum <= 0.0) {
        const double len = (double)total;
#pragma unroll
        for (int k = 0; k < 4; k++) r[k] = (float)(s[k] / len);
        wr = (float)-fsum;
    } else {
#pragma unroll
        for (int k = 0; k < 4; k++) r[k] = (float)(ws[k] / wsum);
        wr = (float)wsum;
    }
    __stcs(reinterpret_cast<float4*>(to + g) + half, make_float4(r[0], r[1], r[2], r[3]));
    if (half == 0) __stcs(wto + g, wr);
}

}  // namespace vp
}  // namespace hdc

using namespace hdc;

extern "C" int hdc_scale_by_weights(JonesF32* d_data_tfb, JonesF32* d_model_tfb, const float* d_weights_tfb,
                                    int num_timesteps, int num_chanblocks, int num_baselines,
                                    const double* d_baseline_weights, hdcStream_t stream) {
    if (!d_data_tfb || !d_model_tfb || !d_weights_tfb || num_timesteps < 0 || num_chanblocks < 0 ||
        num_baselines < 1) {
        set_error("hdc_scale_by_weights: invalid arguments");
        return HDC_ERR_ARG;
    }
    const size_t n = (size_t)num_timesteps * num_chanblocks * num_baselines;
    if (n == 0) return HDC_OK;
    vp::scale_kernel<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(
        d_data_tfb, d_model_tfb, d_weights_tfb, d_baseline_weights, n, num_baselines);
    count_launches(1);
    HDC_CUDA_RET_INT(cudaGetLastError());
    return HDC_OK;
}

extern "C" int hdc_vis_average(const JonesF32* d_from_tfb, const float* d_weights_from_tfb, int num_timesteps,
                               int num_freqs, int num_baselines, const int* h_flagged_chanblocks, int num_flagged,
                               JonesF32* d_to_fb, float* d_weights_to_fb, int num_chanblocks, hdcStream_t stream) {
    if (!d_from_tfb || !d_weights_from_tfb || !d_to_fb || !d_weights_to_fb || num_timesteps < 1 || num_freqs < 1 ||
        num_baselines < 1 || num_chanblocks < 1 || num_flagged < 0 || (num_flagged > 0 && !h_flagged_chanblocks)) {
        set_error("hdc_vis_average: invalid arguments");
        return HDC_ERR_ARG;
    }
    const long long nchunks = (long long)num_chanblocks + num_flagged;
    if (num_flagged > vp::FLAG_CAP || nchunks > 65536) {
        set_error("hdc_vis_average: at most %d flagged of at most 65536 chanblocks (u16 indices)", vp::FLAG_CAP);
        return HDC_ERR_ARG;
    }
    const int avg_freq = (int)((num_freqs + nchunks - 1) / nchunks);
    if ((nchunks - 1) * avg_freq >= num_freqs) {
        set_error("hdc_vis_average: %d channels do not make %lld chunks", num_freqs, nchunks);
        return HDC_ERR_ARG;
    }
    bool ok;
    const std::vector<int> fl = sorted_flags(h_flagged_chanblocks, num_flagged, (int)nchunks, &ok);
    if (!ok) {
        set_error("hdc_vis_average: a flagged chanblock is out of range or repeated");
        return HDC_ERR_ARG;
    }
    cudaStream_t s = (cudaStream_t)stream;
    const size_t n = 2 * (size_t)num_chanblocks * num_baselines;
    const unsigned blocks = (unsigned)((n + vp::AVG_THREADS - 1) / vp::AVG_THREADS);
    auto launch = [&](auto& tab) {
        tab.n = num_flagged;
        for (int k = 0; k < num_flagged; k++) tab.v[k] = (unsigned short)(fl[k] - k);
        vp::average_kernel<<<blocks, vp::AVG_THREADS, 0, s>>>(d_from_tfb, d_weights_from_tfb, num_timesteps,
                                                              num_freqs, num_baselines, avg_freq, tab,
                                                              num_chanblocks, d_to_fb, d_weights_to_fb);
    };
    if (num_flagged <= vp::FLAG_CAP_SMALL) {
        FlagTable<vp::FLAG_CAP_SMALL> tab;
        launch(tab);
    } else {
        static thread_local FlagTable<vp::FLAG_CAP> tab;  // 16 KB: off the stack
        launch(tab);
    }
    count_launches(1);
    HDC_CUDA_RET_INT(cudaGetLastError());
    return HDC_OK;
}
