// Native peel loop: peel_gpu of mwa_hyperdrive (params/peel/gpu.rs:25-757)
// over libhdc's kernels, on one stream.
//
// Per pass and per source (Gauss-Seidel over sources, as the reference):
//   uvws_to   = xyzs_to_uvws(source position)
//   rotate the residual to the source (uvws_from -> uvws_to)
//   model     = the source predicted at its own phase centre with uvws_to
//   resid_src = residual + model * iono(old consts)         (add_model)
//   model_rot = model * iono(old consts)                    (add_model into 0)
//   average both to low resolution (time and channel groups)
//   iono_loop from (0, 0, 1) on the low-resolution data at the source's
//     low-resolution UVWs -> (da, db, dg)
//   consts    = (a + da, b + db, g * dg), reverted if |a| or |b| > 1e-3 or
//               g < 0 or g > 1.5 (gpu.rs:541-627)
//   residual += model * iono(old) - model * iono(consts)    (subtract_iono)
//   uvws_from <- uvws_to
// then rotate back to the phase centre.  The only host round trip per
// source is the read of the fitted constants.

#include <cmath>
#include <memory>
#include <vector>

#include "modeller.cuh"

namespace hdc {
cudaError_t k_xyzs_to_uvws(const XYZ* xyzs, const double* lmsts, UVW* uvws, RADec pc, int ntiles, int nbl, int nt,
                           cudaStream_t s);
cudaError_t k_rotate(JonesF32* vis, int nt, int nbl, int nf, const UVW* from, const UVW* to, const double* lambdas,
                     cudaStream_t s);
cudaError_t k_average(const JonesF32* hi, const float* w, JonesF32* lo, int nt, int nbl, int nf, int favg,
                      cudaStream_t s);
cudaError_t k_subtract_iono(JonesF32* resid, const JonesF32* model, IonoConsts c, IonoConsts old, const UVW* uvws,
                            const double* lambdas, int nt, int nbl, int nf, cudaStream_t s);
cudaError_t k_add_model(JonesF32* resid, const JonesF32* model, IonoConsts c, const double* lambdas, const UVW* uvws,
                        int nt, int nf, int nbl, cudaStream_t s);
cudaError_t k_weights_average(const float* w, float* lo, int nt, int nbl, int nf, int favg, cudaStream_t s);
const char* iono_loop_on(const JonesF32* d_resid, const float* d_w, const JonesF32* d_model, JonesF32* d_model_rot,
                         JonesF64* d_fits, IonoConsts* consts, int nbl, int nf, int niter, const UVW* d_uvws,
                         const double* d_lambdas, double convergence, cudaStream_t s);
}  // namespace hdc

using namespace hdc;

namespace {

struct DevBuf {
    void* p = nullptr;
    ~DevBuf() {
        if (p) cudaFree(p);
    }
    template <class T>
    T* as() {
        return reinterpret_cast<T*>(p);
    }
};

}  // namespace

#define PEEL_CK(call)                                                        \
    do {                                                                     \
        cudaError_t e_ = (call);                                             \
        if (e_ != cudaSuccess) {                                             \
            set_error("hdc_peel_timeblock: %s: %s", #call, cudaGetErrorString(e_)); \
            return HDC_ERR_CUDA;                                             \
        }                                                                    \
    } while (0)

extern "C" int hdc_peel_timeblock(JonesF32* d_resid_tfb, const float* d_weights_tfb, int num_timesteps, int num_freqs,
                                  const double* h_freqs, const XYZ* h_tile_xyzs, int num_tiles, const double* h_lmsts,
                                  double average_lmst, RADec phase_centre, int num_sources,
                                  const HdcSkyModel* h_sources, const RADec* h_source_positions,
                                  IonoConsts* h_iono_consts, const HdcPeelParams* params, hdcStream_t stream) {
    cudaStream_t s = (cudaStream_t)stream;
    if (!d_resid_tfb || !d_weights_tfb || !h_freqs || !h_tile_xyzs || !h_lmsts || !params || num_tiles < 2 ||
        num_timesteps < 1 || num_freqs < 1 || num_sources < 0 || (num_sources > 0 && (!h_sources || !h_iono_consts ||
                                                                                      !h_source_positions))) {
        set_error("hdc_peel_timeblock: invalid arguments");
        return HDC_ERR_ARG;
    }
    const int favg = params->freq_average_factor;
    if (favg < 1 || num_freqs % favg != 0) {
        set_error("hdc_peel_timeblock: %d channels are not a multiple of the averaging factor %d", num_freqs, favg);
        return HDC_ERR_ARG;
    }
    if (num_sources == 0) return HDC_OK;
    const int nt = num_timesteps, nf = num_freqs, nbl = num_tiles * (num_tiles - 1) / 2, nlo = nf / favg;
    const size_t nvis = (size_t)nt * nf * nbl;

    // host-side tables
    std::vector<double> lam(nf), lam_lo(nlo);
    for (int f = 0; f < nf; f++) lam[f] = VEL_C / h_freqs[f];
    std::vector<double> freqs_lo(nlo, 0.0);
    for (int k = 0; k < nlo; k++) {
        double sum = 0.0;
        for (int f = k * favg; f < (k + 1) * favg; f++) sum += h_freqs[f];
        freqs_lo[k] = sum / favg;
        lam_lo[k] = VEL_C / freqs_lo[k];
    }
    std::vector<XYZ> xyz_t((size_t)nt * num_tiles);
    for (int t = 0; t < nt; t++)
        for (int i = 0; i < num_tiles; i++) xyz_t[(size_t)t * num_tiles + i] = h_tile_xyzs[i];

    DevBuf b_lam, b_lam_lo, b_lmst, b_avg_lmst, b_xyz_t, b_from, b_to, b_uv_lo, b_model, b_resid_src, b_model_rot,
        b_resid_lo, b_model_lo, b_model_lo_rot, b_w_lo, b_fits;
    PEEL_CK(cudaMalloc(&b_lam.p, sizeof(double) * nf));
    PEEL_CK(cudaMalloc(&b_lam_lo.p, sizeof(double) * nlo));
    PEEL_CK(cudaMalloc(&b_lmst.p, sizeof(double) * nt));
    PEEL_CK(cudaMalloc(&b_avg_lmst.p, sizeof(double)));
    PEEL_CK(cudaMalloc(&b_xyz_t.p, sizeof(XYZ) * xyz_t.size()));
    PEEL_CK(cudaMalloc(&b_from.p, sizeof(UVW) * (size_t)nt * nbl));
    PEEL_CK(cudaMalloc(&b_to.p, sizeof(UVW) * (size_t)nt * nbl));
    PEEL_CK(cudaMalloc(&b_uv_lo.p, sizeof(UVW) * nbl));
    PEEL_CK(cudaMalloc(&b_model.p, sizeof(JonesF32) * nvis));
    PEEL_CK(cudaMalloc(&b_resid_src.p, sizeof(JonesF32) * nvis));
    PEEL_CK(cudaMalloc(&b_model_rot.p, sizeof(JonesF32) * nvis));
    PEEL_CK(cudaMalloc(&b_resid_lo.p, sizeof(JonesF32) * (size_t)nlo * nbl));
    PEEL_CK(cudaMalloc(&b_model_lo.p, sizeof(JonesF32) * (size_t)nlo * nbl));
    PEEL_CK(cudaMalloc(&b_model_lo_rot.p, sizeof(JonesF32) * (size_t)nlo * nbl));
    PEEL_CK(cudaMalloc(&b_w_lo.p, sizeof(float) * (size_t)nlo * nbl));
    PEEL_CK(cudaMalloc(&b_fits.p, sizeof(JonesF64) * (size_t)nlo * nbl + 256));
    PEEL_CK(cudaMemcpyAsync(b_lam.p, lam.data(), sizeof(double) * nf, cudaMemcpyHostToDevice, s));
    PEEL_CK(cudaMemcpyAsync(b_lam_lo.p, lam_lo.data(), sizeof(double) * nlo, cudaMemcpyHostToDevice, s));
    PEEL_CK(cudaMemcpyAsync(b_lmst.p, h_lmsts, sizeof(double) * nt, cudaMemcpyHostToDevice, s));
    PEEL_CK(cudaMemcpyAsync(b_avg_lmst.p, &average_lmst, sizeof(double), cudaMemcpyHostToDevice, s));
    PEEL_CK(cudaMemcpyAsync(b_xyz_t.p, xyz_t.data(), sizeof(XYZ) * xyz_t.size(), cudaMemcpyHostToDevice, s));
    PEEL_CK(k_weights_average(d_weights_tfb, b_w_lo.as<float>(), nt, nbl, nf, favg, s));

    // one modeller per source, phase centre at the source (update_with_a_source
    // with the source's weighted position, gpu.rs:442)
    std::vector<std::unique_ptr<Modeller>> models;
    for (int i = 0; i < num_sources; i++) {
        HdcModeller* hm = nullptr;
        int rc = peel_modeller_new(&h_sources[i], h_tile_xyzs, num_tiles, h_freqs, num_freqs, h_source_positions[i],
                                   params, &hm);
        if (rc) return rc;
        models.emplace_back(reinterpret_cast<Modeller*>(hm));
    }

    UVW* from = b_from.as<UVW>();
    UVW* to = b_to.as<UVW>();
    const XYZ* dxyz = b_xyz_t.as<XYZ>();
    const double* dlam = b_lam.as<double>();
    for (int pass = 0; pass < params->num_passes; pass++) {
        PEEL_CK(k_xyzs_to_uvws(dxyz, b_lmst.as<double>(), from, phase_centre, num_tiles, nbl, nt, s));
        for (int i = 0; i < num_sources; i++) {
            const IonoConsts old = h_iono_consts[i];
            const RADec sp = h_source_positions[i];
            PEEL_CK(k_xyzs_to_uvws(dxyz, b_lmst.as<double>(), to, sp, num_tiles, nbl, nt, s));
            PEEL_CK(k_rotate(d_resid_tfb, nt, nbl, nf, from, to, dlam, s));
            PEEL_CK(cudaMemsetAsync(b_model.p, 0, sizeof(JonesF32) * nvis, s));
            for (int t = 0; t < nt; t++) {
                int rc = models[i]->model_uvws(h_lmsts[t], to + (size_t)t * nbl,
                                               b_model.as<JonesF32>() + (size_t)t * nf * nbl, s);
                if (rc) return rc;
            }
            PEEL_CK(cudaMemcpyAsync(b_resid_src.p, d_resid_tfb, sizeof(JonesF32) * nvis, cudaMemcpyDeviceToDevice, s));
            PEEL_CK(k_add_model(b_resid_src.as<JonesF32>(), b_model.as<JonesF32>(), old, dlam, to, nt, nf, nbl, s));
            PEEL_CK(cudaMemsetAsync(b_model_rot.p, 0, sizeof(JonesF32) * nvis, s));
            PEEL_CK(k_add_model(b_model_rot.as<JonesF32>(), b_model.as<JonesF32>(), old, dlam, to, nt, nf, nbl, s));
            PEEL_CK(k_average(b_resid_src.as<JonesF32>(), d_weights_tfb, b_resid_lo.as<JonesF32>(), nt, nbl, nf, favg, s));
            PEEL_CK(k_average(b_model_rot.as<JonesF32>(), d_weights_tfb, b_model_lo.as<JonesF32>(), nt, nbl, nf, favg, s));
            PEEL_CK(k_xyzs_to_uvws(dxyz, b_avg_lmst.as<double>(), b_uv_lo.as<UVW>(), sp, num_tiles, nbl, 1, s));
            IonoConsts g = {0.0, 0.0, 1.0};
            const char* err = iono_loop_on(b_resid_lo.as<JonesF32>(), b_w_lo.as<float>(), b_model_lo.as<JonesF32>(),
                                           b_model_lo_rot.as<JonesF32>(), b_fits.as<JonesF64>(), &g, nbl, nlo,
                                           params->num_loops, b_uv_lo.as<UVW>(), b_lam_lo.as<double>(),
                                           params->convergence, s);
            if (err) {
                set_error("hdc_peel_timeblock: %s", err);
                return HDC_ERR_CUDA;
            }
            IonoConsts c = {old.alpha + g.alpha, old.beta + g.beta, old.gain * g.gain};
            const bool issue = std::fabs(c.alpha) > 1e-3 || std::fabs(c.beta) > 1e-3 || c.gain < 0.0 || c.gain > 1.5;
            if (issue) c = old;
            h_iono_consts[i] = c;
            PEEL_CK(k_subtract_iono(d_resid_tfb, b_model.as<JonesF32>(), c, old, to, dlam, nt, nbl, nf, s));
            std::swap(from, to);
        }
        PEEL_CK(k_xyzs_to_uvws(dxyz, b_lmst.as<double>(), to, phase_centre, num_tiles, nbl, nt, s));
        PEEL_CK(k_rotate(d_resid_tfb, nt, nbl, nf, from, to, dlam, s));
    }
    PEEL_CK(cudaStreamSynchronize(s));
    return HDC_OK;
}
