// Native sky modeller: the SkyModeller trait (model/mod.rs:123-204) over the
// direct FP64 kernels (and the tensor-core point path), with all per-timestep
// geometry, beam and flux work on the device.
//
// Construction (SkyModellerGpu::new / update_source_list,
// model/gpu.rs:150-861; ComponentList::new, components/mod.rs:181-272):
// components are split by type in the given order; per type the device holds
//   lmn   [nc]      (l, m, n - 1) in turn units (the reference's LmnRime / 2 pi)
//   S     [nf][nc]  instrumental flux per channel (list fluxes tabulated on the
//                   host with estimate_at_freq, power laws extrapolated on the
//                   device from the catalogue reference frequency, as the CPU
//                   modeller does)
//   gp    [nc]      envelope parameters
// Per timestep (model_timestep_with, model/cpu.rs:787-812): baseline UVWs from
// the tile XYZs at the phase centre's hour angle (tile UVW differences, as
// marlu's xyzs_to_cross_uvws), per-tile shapelet UVs at each shapelet's own
// hour angle (components/mod.rs:279-298), the beam-weighted flux
// W = B S B^H when a beam is set, then the per-type direct kernels.

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "modeller.cuh"
#include "predict.cuh"

namespace hdc {

// ---------------------------------------------------------------------------
// Host restatement of the flux-density models (srclist/types/flux_density/
// mod.rs:158-275) used to tabulate list-type fluxes.
// ---------------------------------------------------------------------------
struct Stokes {
    double freq, i, q, u, v;
};

static Stokes fd_entry(const HdcSkyModel* s, int idx) {
    const double* p = s->fds + 5 * (size_t)idx;
    return Stokes{p[0], p[1], p[2], p[3], p[4]};
}
static Stokes scale(Stokes a, double r) { return Stokes{a.freq, a.i * r, a.q * r, a.u * r, a.v * r}; }
static double signum_rs(double x) { return std::isnan(x) ? NAN : (std::signbit(x) ? -1.0 : 1.0); }

Stokes estimate_list(const HdcSkyModel* s, int c, double freq) {
    const int start = s->fd_start[c], count = s->fd_count[c];
    double si;
    Stokes smaller;
    if (count == 1) {
        si = -0.8;  // DEFAULT_SPEC_INDEX (constants.rs)
        smaller = fd_entry(s, start);
    } else {
        Stokes a = fd_entry(s, start), b = fd_entry(s, start + 1);
        for (int w = 0; w + 1 < count; w++) {
            const Stokes w0 = fd_entry(s, start + w), w1 = fd_entry(s, start + w + 1);
            a = w0;
            b = w1;
            if (std::fabs(w0.freq - freq) < 1e-3) return w0;
            if (std::fabs(w1.freq - freq) < 1e-3) return w1;
            if (freq < w1.freq) break;
        }
        if (signum_rs(a.i) != signum_rs(b.i)) {
            const double run = b.freq - a.freq, df = freq - a.freq;
            return Stokes{freq, a.i + (b.i - a.i) / run * df, a.q + (b.q - a.q) / run * df,
                          a.u + (b.u - a.u) / run * df, a.v + (b.v - a.v) / run * df};
        }
        si = std::log(b.i / a.i) / std::log(b.freq / a.freq);
        smaller = (b.freq < freq) ? b : a;
    }
    Stokes out = smaller;
    out.freq = freq;
    return scale(out, std::pow(freq / smaller.freq, si));
}

static JonesF64 inst_stokes(const Stokes& f) {
    return JonesF64{f.i - f.q, 0.0, f.u, -f.v, f.u, f.v, f.i + f.q, 0.0};
}

// ---------------------------------------------------------------------------
// Device kernels
// ---------------------------------------------------------------------------
struct FluxComp {
    int flux_type;  // 1 power law, 2 curved power law (lists are host-tabulated)
    double freq, i, q, u, v, si, cq;
};

__global__ void flux_kernel(const FluxComp* comps, int nc, const double* freqs, int nf, JonesF64* S) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const int f = blockIdx.y;
    if (c >= nc) return;
    const FluxComp k = comps[c];
    if (k.flux_type == 0) return;
    const double nu = freqs[f];
    const double ratio = pow(nu / k.freq, k.si);
    double i = k.i * ratio, q = k.q * ratio, u = k.u * ratio, v = k.v * ratio;
    if (k.flux_type == 2) {
        const double lr = log(nu / k.freq);
        const double curved = exp(k.cq * (lr * lr));
        i *= curved;
        q *= curved;
        u *= curved;
        v *= curved;
    }
    S[(size_t)f * nc + c] = JonesF64{i - q, 0.0, u, -v, u, v, i + q, 0.0};
}

// Baseline UVWs (m) as tile-UVW differences at one hour angle / declination.
__global__ void baseline_uvw_kernel(const XYZ* xyzs, int ntiles, int nbl, double s_ha, double c_ha, double s_dec,
                                    double c_dec, UVW* uvws) {
    const int bl = blockIdx.x * blockDim.x + threadIdx.x;
    if (bl >= nbl) return;
    int t1, t2;
    baseline_to_tiles(bl, ntiles, t1, t2);
    const XYZ a = xyzs[t1], b = xyzs[t2];
    const double u1 = s_ha * a.x + c_ha * a.y;
    const double v1 = -s_dec * c_ha * a.x + s_dec * s_ha * a.y + c_dec * a.z;
    const double w1 = c_dec * c_ha * a.x - c_dec * s_ha * a.y + s_dec * a.z;
    const double u2 = s_ha * b.x + c_ha * b.y;
    const double v2 = -s_dec * c_ha * b.x + s_dec * s_ha * b.y + c_dec * b.z;
    const double w2 = c_dec * c_ha * b.x - c_dec * s_ha * b.y + s_dec * b.z;
    uvws[bl] = UVW{u1 - u2, v1 - v2, w1 - w2};
}

// Per (shapelet component, tile) UV [m] at the component's hour angle.
__global__ void shapelet_tile_uv_kernel(const double2* radec, int nc, const XYZ* xyzs, int ntiles, double lst,
                                        double2* out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nc * ntiles) return;
    const int c = i / ntiles, t = i % ntiles;
    const double2 rd = radec[c];
    double s_ha, c_ha, s_dec, c_dec;
    sincos(lst - rd.x, &s_ha, &c_ha);
    sincos(rd.y, &s_dec, &c_dec);
    const XYZ a = xyzs[t];
    out[i] = make_double2(s_ha * a.x + c_ha * a.y, -s_dec * c_ha * a.x + s_dec * s_ha * a.y + c_dec * a.z);
}

// Analytic 4x4 dipole-array tile over a ground plane (a model of this
// project; mwa_hyperdrive has no analytic beam): for direction (az, za),
// J = A R(az)^T diag(cos za, 1) R(az), A = AFx(l) AFy(m) GP(za) / |GP(0)|,
// l = sin za sin az, m = sin za cos az, AFx(l) = (cos(k 0.55 l) + cos(k 1.65 l))/2
// (1.1 m dipole spacing), GP = 1 - exp(-2 i k h cos za), h = 0.278 m.
__device__ J2 analytic_beam(double az, double el, double freq) {
    if (el <= 0.0) return jzero();
    const double za = FRAC_PI_2 - el;
    const double k = TAU * freq / VEL_C;
    double sza, cza, saz, caz;
    sincos(za, &sza, &cza);
    sincos(az, &saz, &caz);
    const double l = sza * saz, m = sza * caz;
    const double afx = 0.5 * (cos(k * 0.55 * l) + cos(k * 1.65 * l));
    const double afy = 0.5 * (cos(k * 0.55 * m) + cos(k * 1.65 * m));
    const double h = 0.278;
    double sp, cp;
    sincos(2.0 * k * h * cza, &sp, &cp);
    const double gp0 = 2.0 * fabs(sin(k * h));
    const double a = afx * afy / gp0;
    const cplx amp = cplx{1.0 - cp, sp} * a;
    const double p00 = cza * saz * saz + caz * caz;
    const double p01 = (cza - 1.0) * saz * caz;
    const double p11 = cza * caz * caz + saz * saz;
    return J2{amp * p00, amp * p01, amp * p01, amp * p11};
}

// The same tile with its own dipole amplitudes g [2][16] (X dipoles, then Y;
// dipole d at east (d % 4 - 1.5) 1.1 m, north (d / 4 - 1.5) 1.1 m):
// J = diag(ax, ay) R(az)^T diag(cos za, 1) R(az), ax = AF(g_x) GP / |GP(0)|,
// AF(g) = (1/16) sum_d g_d exp(i k (x_d l + y_d m)).  With every g_d = 1,
// AF = AFx(l) AFy(m) and J is analytic_beam's.
__device__ J2 analytic_beam_tile(double az, double el, double freq, const double* g) {
    if (el <= 0.0) return jzero();
    const double za = FRAC_PI_2 - el;
    const double k = TAU * freq / VEL_C;
    double sza, cza, saz, caz;
    sincos(za, &sza, &cza);
    sincos(az, &saz, &caz);
    const double l = sza * saz, m = sza * caz;
    cplx ex[4], ey[4];
    for (int i = 0; i < 4; i++) {
        const double x = (i - 1.5) * 1.1;
        double s, c;
        sincos(k * x * l, &s, &c);
        ex[i] = cplx{c, s};
        sincos(k * x * m, &s, &c);
        ey[i] = cplx{c, s};
    }
    cplx afx = {0.0, 0.0}, afy = {0.0, 0.0};
    for (int d = 0; d < 16; d++) {
        const cplx e = ex[d & 3] * ey[d >> 2];
        afx = afx + e * g[d];
        afy = afy + e * g[16 + d];
    }
    const double h = 0.278;
    double sp, cp;
    sincos(2.0 * k * h * cza, &sp, &cp);
    const double gp0 = 2.0 * fabs(sin(k * h));
    const cplx gp = cplx{1.0 - cp, sp} * (1.0 / (16.0 * gp0));
    const cplx ax = afx * gp, ay = afy * gp;
    const double p00 = cza * saz * saz + caz * caz;
    const double p01 = (cza - 1.0) * saz * caz;
    const double p11 = cza * caz * caz + saz * saz;
    return J2{ax * p00, ax * p01, ay * p01, ay * p11};
}

// W[f][c] = B S B^H for a beam shared by all tiles (model/cpu.rs:187-230,
// 336-337 with B1 == B2).
__global__ void beam_weight_kernel(const double2* radec, int nc, const double* freqs, int nf, double lst, double lat,
                                   const JonesF64* S, JonesF64* W) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const int f = blockIdx.y;
    if (c >= nc) return;
    const double2 rd = radec[c];
    double az, el;
    hadec_to_azel(lst - rd.x, rd.y, lat, az, el);
    const J2 b = analytic_beam(az, el, freqs[f]);
    const J2 s = load_j(S[(size_t)f * nc + c]);
    W[(size_t)f * nc + c] = store_j((b * s) * herm(b));
}

// FP32 copy of a per-tile beam table (n Jones matrices).
__global__ void jones_to_f32_kernel(const JonesF64* __restrict__ in, size_t n, JonesF32* __restrict__ out) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double4* a = reinterpret_cast<const double4*>(in + i);
    const double4 x = a[0], y = a[1];
    float4* o = reinterpret_cast<float4*>(out + i);
    o[0] = make_float4((float)x.x, (float)x.y, (float)x.z, (float)x.w);
    o[1] = make_float4((float)y.x, (float)y.y, (float)y.z, (float)y.w);
}

// Per-tile beams B [uniq tile][uniq freq][nc] of one component type at this
// timestep.
__global__ void tile_beam_kernel(const double2* radec, int nc, const double* ufreqs, int nuf, const double* gains,
                                 double lst, double lat, JonesF64* B) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const int uf = blockIdx.y, u = blockIdx.z;
    if (c >= nc) return;
    const double2 rd = radec[c];
    double az, el;
    hadec_to_azel(lst - rd.x, rd.y, lat, az, el);
    B[((size_t)u * nuf + uf) * nc + c] = store_j(analytic_beam_tile(az, el, ufreqs[uf], gains + 32 * u));
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
template <class T>
static cudaError_t dalloc(T** p, size_t n) {
    *p = nullptr;
    if (n == 0) return cudaSuccess;
    return cudaMalloc((void**)p, sizeof(T) * n);
}
template <class T>
static void dfree(T*& p) {
    if (p) cudaFree((void*)p);
    p = nullptr;
}

void TileBeams::release() {
    dfree(d_gains);
    dfree(d_tile_map);
    dfree(d_freqs);
    dfree(d_freq_map);
    fee = nullptr;
    n_uniq_tile = n_uniq_freq = 0;
}

void TypeTables::release() {
    dfree(d_B);
    dfree(d_B32);
    dfree(d_lmn);
    dfree(d_S);
    dfree(d_W);
    dfree(d_gp);
    dfree(d_radec);
    dfree(d_coeffs);
    dfree(d_cstart);
    dfree(d_ccount);
    dfree(d_suv_tile);
    dfree(d_sdense);
    nc = 0;
}

static void lmn_turns(double ra, double dec, double pc_ra, double pc_dec, double out[3]) {
    // marlu RADec::to_lmn; prepare_for_rime's 2 pi is applied in the kernel's
    // turn-based phase instead.
    const double d_ra = ra - pc_ra;
    const double s_d_ra = std::sin(d_ra), c_d_ra = std::cos(d_ra);
    const double s_dec = std::sin(dec), c_dec = std::cos(dec);
    const double pc_s = std::sin(pc_dec), pc_c = std::cos(pc_dec);
    out[0] = c_dec * s_d_ra;
    out[1] = s_dec * pc_c - c_dec * pc_s * c_d_ra;
    out[2] = (s_dec * pc_s + c_dec * pc_c * c_d_ra) - 1.0;
}

int Modeller::build_tables(const HdcSkyModel* sky) {
    for (int ty = 0; ty < 3; ty++) t[ty].release();
    std::vector<int> idx[3];
    for (int c = 0; c < sky->num_components; c++) {
        const int ty = sky->comp_type[c];
        if (ty < 0 || ty > 2) {
            set_error("component %d has unknown type %d", c, ty);
            return HDC_ERR_ARG;
        }
        const int ft = sky->flux_type[c];
        if (ft < 0 || ft > 2 || sky->fd_count[c] < 1) {
            set_error("component %d has an invalid flux model", c);
            return HDC_ERR_ARG;
        }
        idx[ty].push_back(c);
    }
    std::vector<double> hfreqs(freqs);
    for (int ty = 0; ty < 3; ty++) {
        TypeTables& tt = t[ty];
        const int nc = (int)idx[ty].size();
        tt.nc = nc;
        if (nc == 0) continue;
        std::vector<double4> lmn(nc), gp(nc);
        std::vector<double2> radec(nc);
        std::vector<JonesF64> S((size_t)nf * nc);
        std::vector<FluxComp> fc(nc);
        std::vector<ShapeletCoeff> coeffs;
        std::vector<int> cstart(nc), ccount(nc);
        for (int k = 0; k < nc; k++) {
            const int c = idx[ty][k];
            double l3[3];
            lmn_turns(sky->ra[c], sky->dec[c], pc.ra, pc.dec, l3);
            lmn[k] = make_double4(l3[0], l3[1], l3[2], 0.0);
            radec[k] = make_double2(sky->ra[c], sky->dec[c]);
            if (ty >= 1) {
                const double sp = std::sin(sky->pa[c]), cp = std::cos(sky->pa[c]);
                if (ty == 1)
                    gp[k] = make_double4(GAUSSIAN_EXP_CONST * (sky->maj[c] * sky->maj[c]),
                                         GAUSSIAN_EXP_CONST * (sky->min[c] * sky->min[c]), sp, cp);
                else
                    gp[k] = make_double4(sky->maj[c] * SHAPELET_CONST, -sky->min[c] * SHAPELET_CONST, sp, cp);
            }
            const int ft = sky->flux_type[c];
            FluxComp f = {};
            f.flux_type = ft;
            if (ft == HDC_FLUX_LIST) {
                for (int fi = 0; fi < nf; fi++) S[(size_t)fi * nc + k] = inst_stokes(estimate_list(sky, c, hfreqs[fi]));
            } else {
                const Stokes r = fd_entry(sky, sky->fd_start[c]);
                f.freq = r.freq;
                f.i = r.i;
                f.q = r.q;
                f.u = r.u;
                f.v = r.v;
                f.si = sky->si[c];
                f.cq = (ft == HDC_FLUX_CURVED_POWER_LAW) ? sky->q[c] : 0.0;
            }
            fc[k] = f;
            if (ty == 2) {
                cstart[k] = (int)coeffs.size();
                ccount[k] = sky->coeff_count[c];
                for (int q = 0; q < sky->coeff_count[c]; q++) {
                    const int ci = sky->coeff_start[c] + q;
                    const int n1 = sky->coeff_n1[ci], n2 = sky->coeff_n2[ci];
                    if (n1 < 0 || n1 >= SBF_N || n2 < 0 || n2 >= SBF_N) {
                        set_error("shapelet coefficient order (%d, %d) outside 0..%d", n1, n2, SBF_N - 1);
                        return HDC_ERR_ARG;
                    }
                    ShapeletCoeff sc;
                    std::memset(&sc, 0, sizeof(sc));
                    sc.value = sky->coeff_value[ci];
                    sc.n1 = (unsigned char)n1;
                    sc.n2 = (unsigned char)n2;
                    coeffs.push_back(sc);
                }
            }
        }
        HDC_CUDA_RET_INT(dalloc(&tt.d_lmn, nc));
        HDC_CUDA_RET_INT(dalloc(&tt.d_S, (size_t)nf * nc));
        HDC_CUDA_RET_INT(dalloc(&tt.d_gp, nc));
        HDC_CUDA_RET_INT(dalloc(&tt.d_radec, nc));
        HDC_CUDA_RET_INT(cudaMemcpy(tt.d_lmn, lmn.data(), sizeof(double4) * nc, cudaMemcpyHostToDevice));
        HDC_CUDA_RET_INT(cudaMemcpy(tt.d_gp, gp.data(), sizeof(double4) * nc, cudaMemcpyHostToDevice));
        HDC_CUDA_RET_INT(cudaMemcpy(tt.d_radec, radec.data(), sizeof(double2) * nc, cudaMemcpyHostToDevice));
        HDC_CUDA_RET_INT(cudaMemcpy(tt.d_S, S.data(), sizeof(JonesF64) * S.size(), cudaMemcpyHostToDevice));
        FluxComp* d_fc = nullptr;
        HDC_CUDA_RET_INT(dalloc(&d_fc, nc));
        HDC_CUDA_RET_INT(cudaMemcpy(d_fc, fc.data(), sizeof(FluxComp) * nc, cudaMemcpyHostToDevice));
        dim3 g((nc + 127) / 128, nf);
        flux_kernel<<<g, 128>>>(d_fc, nc, d_freqs, nf, tt.d_S);
        count_launches(1);
        cudaError_t e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaDeviceSynchronize();
        cudaFree(d_fc);
        HDC_CUDA_RET_INT(e);
        if (beam_kind == HDC_BEAM_ANALYTIC_DIPOLE) HDC_CUDA_RET_INT(dalloc(&tt.d_W, (size_t)nf * nc));
        if (ty == 2) {
            HDC_CUDA_RET_INT(dalloc(&tt.d_coeffs, coeffs.size() + 1));
            if (!coeffs.empty())
                HDC_CUDA_RET_INT(cudaMemcpy(tt.d_coeffs, coeffs.data(), sizeof(ShapeletCoeff) * coeffs.size(),
                                            cudaMemcpyHostToDevice));
            HDC_CUDA_RET_INT(dalloc(&tt.d_cstart, nc));
            HDC_CUDA_RET_INT(dalloc(&tt.d_ccount, nc));
            HDC_CUDA_RET_INT(cudaMemcpy(tt.d_cstart, cstart.data(), sizeof(int) * nc, cudaMemcpyHostToDevice));
            HDC_CUDA_RET_INT(cudaMemcpy(tt.d_ccount, ccount.data(), sizeof(int) * nc, cudaMemcpyHostToDevice));
            HDC_CUDA_RET_INT(dalloc(&tt.d_suv_tile, (size_t)nc * ntiles));
            // dense form: sum of value * sign(i^(n1+n2)) per (n1, n2); the
            // real part takes even n1 + n2, the imaginary part odd
            bool dense = true;
            for (const ShapeletCoeff& sc : coeffs) dense = dense && sc.n1 < SDN && sc.n2 < SDN;
            if (dense) {
                std::vector<double> dm((size_t)nc * SDN * SDN, 0.0);
                for (int k = 0; k < nc; k++)
                    for (int q = 0; q < ccount[k]; q++) {
                        const ShapeletCoeff& sc = coeffs[cstart[k] + q];
                        const double sgn = ((sc.n1 + sc.n2) & 3) < 2 ? 1.0 : -1.0;
                        dm[((size_t)k * SDN + sc.n1) * SDN + sc.n2] += sgn * sc.value;
                    }
                std::vector<float> df(dm.begin(), dm.end());
                HDC_CUDA_RET_INT(dalloc(&tt.d_sdense, df.size()));
                HDC_CUDA_RET_INT(cudaMemcpy(tt.d_sdense, df.data(), sizeof(float) * df.size(), cudaMemcpyHostToDevice));
            }
        }
    }
    if (tile_beams()) return alloc_tile_beam_tables();
    return HDC_OK;
}

int Modeller::alloc_tile_beam_tables() {
    for (int ty = 0; ty < 3; ty++) {
        dfree(t[ty].d_B);
        dfree(t[ty].d_B32);
        if (t[ty].nc == 0) continue;
        HDC_CUDA_RET_INT(dalloc(&t[ty].d_B, (size_t)tb.n_uniq_tile * tb.n_uniq_freq * t[ty].nc));
        if (ty == 0 && form == HDC_PREDICT_TENSOR)
            HDC_CUDA_RET_INT(dalloc(&t[ty].d_B32, (size_t)tb.n_uniq_tile * tb.n_uniq_freq * t[ty].nc));
    }
    return HDC_OK;
}

int Modeller::set_tile_beams(const double* h_gains, double freq_res_hz) {
    if (!h_gains || !(freq_res_hz > 0.0)) {
        set_error("hdc_modeller_set_tile_beams: invalid arguments");
        return HDC_ERR_ARG;
    }
    // unique tiles by their 32 gains, in order of first appearance
    std::vector<int> tmap(ntiles);
    std::vector<double> ugains;
    for (int p = 0; p < ntiles; p++) {
        const double* g = h_gains + 32 * (size_t)p;
        int found = -1;
        for (size_t u = 0; u < ugains.size() / 32 && found < 0; u++)
            if (std::equal(g, g + 32, ugains.begin() + 32 * u)) found = (int)u;
        if (found < 0) {
            found = (int)(ugains.size() / 32);
            ugains.insert(ugains.end(), g, g + 32);
        }
        tmap[p] = found;
    }
    // unique beam frequencies: each channel at the nearest multiple of the resolution
    std::vector<long long> bins(nf);
    for (int f = 0; f < nf; f++) bins[f] = std::llround(freqs[f] / freq_res_hz);
    std::vector<long long> ub(bins);
    std::sort(ub.begin(), ub.end());
    ub.erase(std::unique(ub.begin(), ub.end()), ub.end());
    std::vector<int> fmap(nf);
    std::vector<double> ufreq(ub.size());
    for (size_t i = 0; i < ub.size(); i++) ufreq[i] = (double)ub[i] * freq_res_hz;
    for (int f = 0; f < nf; f++) fmap[f] = (int)(std::lower_bound(ub.begin(), ub.end(), bins[f]) - ub.begin());
    cudaDeviceSynchronize();
    tb.release();
    tb.n_uniq_tile = (int)(ugains.size() / 32);
    tb.n_uniq_freq = (int)ub.size();
    HDC_CUDA_RET_INT(dalloc(&tb.d_gains, ugains.size()));
    HDC_CUDA_RET_INT(dalloc(&tb.d_tile_map, ntiles));
    HDC_CUDA_RET_INT(dalloc(&tb.d_freqs, ufreq.size()));
    HDC_CUDA_RET_INT(dalloc(&tb.d_freq_map, nf));
    HDC_CUDA_RET_INT(cudaMemcpy(tb.d_gains, ugains.data(), sizeof(double) * ugains.size(), cudaMemcpyHostToDevice));
    HDC_CUDA_RET_INT(cudaMemcpy(tb.d_tile_map, tmap.data(), sizeof(int) * ntiles, cudaMemcpyHostToDevice));
    HDC_CUDA_RET_INT(cudaMemcpy(tb.d_freqs, ufreq.data(), sizeof(double) * ufreq.size(), cudaMemcpyHostToDevice));
    HDC_CUDA_RET_INT(cudaMemcpy(tb.d_freq_map, fmap.data(), sizeof(int) * nf, cudaMemcpyHostToDevice));
    for (int ty = 0; ty < 3; ty++) dfree(t[ty].d_W);
    beam_kind = HDC_BEAM_ANALYTIC_PER_TILE;
    return alloc_tile_beam_tables();
}

int Modeller::set_fee_beam(const HdcFeeBeam* b) {
    if (!b || fee_num_tiles(b) != ntiles || fee_num_freqs(b) != nf || fee_device(b) != device) {
        set_error("hdc_modeller_set_fee_beam: the beam was not prepared for this modeller's %d tiles and %d channels "
                  "on device %d", ntiles, nf, device);
        return HDC_ERR_ARG;
    }
    cudaDeviceSynchronize();
    tb.release();
    tb.n_uniq_tile = hdc_fee_beam_num_unique_tiles(b);
    tb.n_uniq_freq = hdc_fee_beam_num_unique_freqs(b);
    HDC_CUDA_RET_INT(dalloc(&tb.d_tile_map, ntiles));
    HDC_CUDA_RET_INT(dalloc(&tb.d_freq_map, nf));
    HDC_CUDA_RET_INT(cudaMemcpy(tb.d_tile_map, hdc_fee_beam_tile_map(b), sizeof(int) * ntiles,
                                cudaMemcpyDeviceToDevice));
    HDC_CUDA_RET_INT(cudaMemcpy(tb.d_freq_map, hdc_fee_beam_freq_map(b), sizeof(int) * nf, cudaMemcpyDeviceToDevice));
    tb.fee = b;
    for (int ty = 0; ty < 3; ty++) dfree(t[ty].d_W);
    beam_kind = HDC_BEAM_FEE;
    return alloc_tile_beam_tables();
}

int Modeller::geometry(double lst, cudaStream_t s) {
    const double ha = lst - pc.ra;
    const double s_ha = std::sin(ha), c_ha = std::cos(ha);
    const double s_dec = std::sin(pc.dec), c_dec = std::cos(pc.dec);
    baseline_uvw_kernel<<<(nbl + 255) / 256, 256, 0, s>>>(d_xyzs, ntiles, nbl, s_ha, c_ha, s_dec, c_dec, d_uvws);
    count_launches(1);
    HDC_CUDA_RET_INT(cudaGetLastError());
    if (t[2].nc > 0) {
        const int n = t[2].nc * ntiles;
        shapelet_tile_uv_kernel<<<(n + 255) / 256, 256, 0, s>>>(t[2].d_radec, t[2].nc, d_xyzs, ntiles, lst,
                                                                 t[2].d_suv_tile);
        count_launches(1);
        HDC_CUDA_RET_INT(cudaGetLastError());
    }
    if (tile_beams()) {
        for (int ty = 0; ty < 3; ty++) {
            if (t[ty].nc == 0 || tb.n_uniq_tile == 0) continue;
            if (tb.fee) {
                const int rc = fee_launch_radec(tb.fee, t[ty].d_radec, t[ty].nc, lst, lat, t[ty].d_B, s);
                if (rc) return rc;
                continue;
            }
            dim3 g((t[ty].nc + 127) / 128, tb.n_uniq_freq, tb.n_uniq_tile);
            tile_beam_kernel<<<g, 128, 0, s>>>(t[ty].d_radec, t[ty].nc, tb.d_freqs, tb.n_uniq_freq, tb.d_gains, lst,
                                                lat, t[ty].d_B);
            count_launches(1);
            HDC_CUDA_RET_INT(cudaGetLastError());
        }
        // the points' table in FP32 for the tensor form's producers
        if (t[0].d_B32) {
            const size_t n = (size_t)tb.n_uniq_tile * tb.n_uniq_freq * t[0].nc;
            jones_to_f32_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(t[0].d_B, n, t[0].d_B32);
            count_launches(1);
            HDC_CUDA_RET_INT(cudaGetLastError());
        }
    } else if (beam_kind != HDC_BEAM_NONE) {
        for (int ty = 0; ty < 3; ty++) {
            if (t[ty].nc == 0) continue;
            dim3 g((t[ty].nc + 127) / 128, nf);
            beam_weight_kernel<<<g, 128, 0, s>>>(t[ty].d_radec, t[ty].nc, d_freqs, nf, lst, lat, t[ty].d_S, t[ty].d_W);
            count_launches(1);
            HDC_CUDA_RET_INT(cudaGetLastError());
        }
    }
    return HDC_OK;
}

// B S B^H for a beam shared by all tiles; S when there is no beam or a beam
// per tile (applied per baseline)
const JonesF64* Modeller::weights(int ty) const {
    return beam_kind == HDC_BEAM_ANALYTIC_DIPOLE ? t[ty].d_W : t[ty].d_S;
}

DirectParams Modeller::direct_params(int ty, void* vis) const {
    DirectParams p = {};
    p.nbl = nbl;
    p.nf = nf;
    p.ntiles = ntiles;
    p.nc = t[ty].nc;
    p.freqs = d_freqs;
    p.uvws = d_uvws;
    p.lmn = t[ty].d_lmn;
    p.flux = weights(ty);
    p.gp = t[ty].d_gp;
    p.sbf = d_sbf;
    p.sbf32 = form == HDC_PREDICT_TENSOR ? device_shapelet_basis_f32() : nullptr;
    p.sbfp = form == HDC_PREDICT_TENSOR ? device_shapelet_basis_pairs() : nullptr;
    p.sdense = form == HDC_PREDICT_TENSOR ? t[ty].d_sdense : nullptr;
    p.coeffs = t[ty].d_coeffs;
    p.coeff_start = t[ty].d_cstart;
    p.coeff_count = t[ty].d_ccount;
    p.suv_bl = nullptr;
    p.suv_tile = t[ty].d_suv_tile;
    if (tile_beams()) {
        p.beam = t[ty].d_B;
        p.tile_map = tb.d_tile_map;
        p.unflagged_map = nullptr;
        p.freq_map = tb.d_freq_map;
        p.n_uniq_freq = tb.n_uniq_freq;
        p.n_uniq_tile = tb.n_uniq_tile;
    }
    p.vis = vis;
    p.err = d_err;
    return p;
}

void Modeller::prof_begin(int cls, cudaStream_t s, EvPair& e) {
    if (!profiling) return;
    if (!ev_free.empty()) {
        e = ev_free.back();
        ev_free.pop_back();
    } else {
        cudaEventCreate(&e.a);
        cudaEventCreate(&e.b);
    }
    e.cls = cls;
    cudaEventRecord(e.a, s);
}

void Modeller::prof_end(cudaStream_t s, EvPair& e) {
    if (!profiling) return;
    cudaEventRecord(e.b, s);
    ev_pending.push_back(e);
}

void Modeller::prof_collect() {
    for (EvPair& e : ev_pending) {
        float ms = 0.f;
        cudaEventSynchronize(e.b);
        if (cudaEventElapsedTime(&ms, e.a, e.b) == cudaSuccess) prof_ms[e.cls] += ms;
        ev_free.push_back(e);
    }
    ev_pending.clear();
}

int Modeller::model_channels(double lst, void* d_vis, bool out64, int f0, int nfc, cudaStream_t s, int types,
                             bool mask) {
    EvPair e{};
    const size_t vis_off = (size_t)f0 * nbl * (out64 ? sizeof(JonesF64) : sizeof(JonesF32));
    void* vis = static_cast<char*>(d_vis) + vis_off;
    // the reference's order (points, Gaussians, shapelets: the FP32 sums
    // round as its do); the tensor form adds Gaussians, shapelets, then
    // points, as its host-buffer call does (that call stages the first two and
    // adds the points chunk by chunk)
    static constexpr int REF_ORDER[3] = {0, 1, 2}, TENSOR_ORDER[3] = {1, 2, 0};
    const int* order = form == HDC_PREDICT_TENSOR ? TENSOR_ORDER : REF_ORDER;
    for (int k = 0; k < 3; k++) {
        const int ty = order[k];
        if (t[ty].nc == 0 || !(types & (1 << ty))) continue;
        prof_begin(ty, s, e);
        if (ty == 0 && form == HDC_PREDICT_TENSOR) {
            // the workspace holds planes for all nf channels; a chunk of nfc
            // channels uses its start (chunks of one call run in order on s)
            void* ws = tensor_workspace(out64);
            if (!ws) return HDC_ERR_ALLOC;
            TensorBeam tbm = {t[0].d_B, t[0].d_B32, tb.d_tile_map, tb.d_freq_map + f0, tb.n_uniq_tile,
                              tb.n_uniq_freq};
            const int rc = launch_tensor_points(nfc, nbl, ntiles, t[0].nc, d_freqs + f0, d_xyzs, lst - pc.ra, pc.dec,
                                                t[0].d_lmn, weights(0) + (size_t)f0 * t[0].nc,
                                                tile_beams() ? &tbm : nullptr, vis, out64, ws, d_err, s, tensor_sync());
            if (rc) return rc;
        } else {
            // the chosen (tensor) form keeps Gaussians and shapelets in the
            // direct kernel, in its FP32 form with a shared beam (FP64 with
            // per-tile beams)
            DirectParams p = direct_params(ty, vis);
            p.nf = nfc;
            p.freqs = d_freqs + f0;
            p.flux = p.flux + (size_t)f0 * p.nc;
            if (tile_beams()) p.freq_map = tb.d_freq_map + f0;
            HDC_CUDA_RET_INT(launch_direct(ty, tile_beams(), out64, p, s, form == HDC_PREDICT_TENSOR));
        }
        prof_end(s, e);
    }
    if (!out64 && mask) HDC_CUDA_RET_INT(launch_mask_pols((JonesF32*)vis, (size_t)nfc * nbl, pols, s));
    return HDC_OK;
}

int Modeller::queue_error_check(cudaStream_t s) {
    HDC_CUDA_RET_INT(cudaMemcpyAsync(h_err, d_err, sizeof(int), cudaMemcpyDeviceToHost, s));
    HDC_CUDA_RET_INT(cudaEventRecord(err_ev, s));
    return HDC_OK;
}

// Report the kernel error word as of the last queued copy.  wait: block until
// that copy has landed; otherwise look only if it already has.
int Modeller::take_error(bool wait) {
    cudaError_t q = wait ? cudaEventSynchronize(err_ev) : cudaEventQuery(err_ev);
    if (q == cudaErrorNotReady) return HDC_OK;
    if (q != cudaSuccess) {
        hdc::set_error("modeller: %s", cudaGetErrorString(q));
        return HDC_ERR_CUDA;
    }
    const int w = *(volatile int*)h_err;
    if (!w) return HDC_OK;
    // clear both copies before reporting, so that the next call starts clean
    HDC_CUDA_RET_INT(cudaMemset(d_err, 0, sizeof(int)));
    *(volatile int*)h_err = 0;
    hdc::set_error("modeller: %s", kernel_error_string(w));
    return kernel_error_status(w);
}

int Modeller::model(double lst, void* d_vis, bool out64, UVW* h_uvws, cudaStream_t s) {
    int rc0 = take_error(false);
    if (rc0) return rc0;
    EvPair e{};
    prof_begin(3, s, e);
    int rc = geometry(lst, s);
    if (rc) return rc;
    prof_end(s, e);
    rc = model_channels(lst, d_vis, out64, 0, nf, s);
    if (rc) return rc;
    rc = queue_error_check(s);
    if (rc) return rc;
    if (h_uvws) {
        HDC_CUDA_RET_INT(cudaMemcpyAsync(h_uvws, d_uvws, sizeof(UVW) * nbl, cudaMemcpyDeviceToHost, s));
        HDC_CUDA_RET_INT(cudaStreamSynchronize(s));
        return take_error(true);
    }
    return HDC_OK;
}

int Modeller::model_uvws(double lst, const UVW* d_uvws_ext, JonesF32* d_vis, cudaStream_t s) {
    int rc = take_error(false);
    if (rc) return rc;
    rc = geometry(lst, s);
    if (rc) return rc;
    for (int ty = 0; ty < 3; ty++) {
        if (t[ty].nc == 0) continue;
        DirectParams p = direct_params(ty, d_vis);
        p.uvws = d_uvws_ext;
        HDC_CUDA_RET_INT(launch_direct(ty, tile_beams(), false, p, s));
    }
    return queue_error_check(s);
}

int Modeller::autos(double lst, JonesF32* d_vis, cudaStream_t s) {
    int rc = take_error(false);
    if (rc) return rc;
    rc = geometry(lst, s);
    if (rc) return rc;
    for (int ty = 0; ty < 3; ty++) {
        if (t[ty].nc == 0) continue;
        AutosParams p = {};
        p.ntiles = ntiles;
        p.nf = nf;
        p.nc_total = t[ty].nc;
        p.flux = weights(ty);  // with a shared beam, B S B^H is already the auto term
        p.beam = nullptr;
        if (tile_beams()) {
            p.beam = t[ty].d_B;
            p.tile_map = tb.d_tile_map;
            p.unflagged_map = nullptr;
            p.freq_map = tb.d_freq_map;
            p.n_uniq_freq = tb.n_uniq_freq;
        }
        p.vis = d_vis;
        HDC_CUDA_RET_INT(launch_autos(p, s));
    }
    return HDC_OK;
}

Modeller::~Modeller() {
    tb.release();
    if (err_ev) cudaEventDestroy(err_ev);
    if (h_err) cudaFreeHost(h_err);
    dfree(d_err);
    for (int i = 0; i < 3; i++)
        if (pipe_s[i]) cudaStreamDestroy(pipe_s[i]);
    for (auto& ev : pipe_ev)
        if (ev) cudaEventDestroy(ev);
    for (int ty = 0; ty < 3; ty++) t[ty].release();
    dfree(d_freqs);
    dfree(d_xyzs);
    dfree(d_uvws);
    dfree(d_host_vis);
    dfree(d_host_model);
    tensor_release();
    for (EvPair& e : ev_pending) ev_free.push_back(e);
    for (EvPair& e : ev_free) {
        cudaEventDestroy(e.a);
        cudaEventDestroy(e.b);
    }
}

}  // namespace hdc

using hdc::Modeller;

namespace hdc {
// Per (component, coarse frequency): the veto's tests and brightness
// (srclist/veto.rs:58-129).  A component below the elevation limit or
// farther than the cutoff from the phase centre marks its source vetoed;
// otherwise its beam-attenuated flux |(J I J^H)_XX| + |(J I J^H)_YY| (I the
// instrumental flux, J the beam; veto.rs:193-207) is added to its source's
// total at that frequency.
__global__ void veto_kernel(const double2* radec, const int* comp_source, int nc, const double* freqs, int nf,
                            double lst, double lat, double pc_ra, double pc_dec, int beam_kind, double cutoff,
                            double min_el, const JonesF64* S, const JonesF64* B, const int* bmap, double* src_fd,
                            int* src_vetoed) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const int f = blockIdx.y;
    if (c >= nc) return;
    const double2 rd = radec[c];
    const int src = comp_source[c];
    double az, el;
    hadec_to_azel(lst - rd.x, rd.y, lat, az, el);
    // angular separation from the phase centre (haversine)
    const double sd = sin(0.5 * (rd.y - pc_dec)), sr = sin(0.5 * (rd.x - pc_ra));
    const double hav = sd * sd + cos(rd.y) * cos(pc_dec) * sr * sr;
    const double sep = 2.0 * asin(sqrt(fmin(1.0, fmax(0.0, hav))));
    if (el < min_el || sep > cutoff) {
        if (f == 0) atomicOr(src_vetoed + src, 1);
        return;
    }
    J2 s = load_j(S[(size_t)f * nc + c]);
    if (beam_kind == HDC_BEAM_ANALYTIC_DIPOLE) {
        const J2 b = analytic_beam(az, el, freqs[f]);
        s = b * (s * herm(b));
    } else if (beam_kind == HDC_BEAM_FEE) {
        // the FEE table [unique frequency][component] of the one beam
        const J2 b = load_j(B[(size_t)bmap[f] * nc + c]);
        s = b * (s * herm(b));
    }
    atomicAdd(src_fd + (size_t)src * nf + f, hypot(s.a.re, s.a.im) + hypot(s.d.re, s.d.im));
}
}  // namespace hdc

namespace hdc {
// hdc_source_brightness and hdc_source_brightness_fee: fee is the FEE beam
// when beam_kind is HDC_BEAM_FEE.
static int source_brightness(const HdcSkyModel* sky, const int* h_comp_source, int num_sources, const double* h_freqs,
                             int num_freqs, double lst_rad, double latitude_rad, RADec phase_centre, int beam_kind,
                             const HdcFeeBeam* fee, double source_dist_cutoff_rad, double min_elevation_rad,
                             double* h_brightness) {
    if (!sky || !h_comp_source || !h_freqs || !h_brightness || num_sources < 1 || num_freqs < 1 ||
        (beam_kind != HDC_BEAM_NONE && beam_kind != HDC_BEAM_ANALYTIC_DIPOLE && beam_kind != HDC_BEAM_FEE)) {
        set_error("hdc_source_brightness: invalid arguments");
        return HDC_ERR_ARG;
    }
    int dev = 0;
    HDC_CUDA_RET_INT(cudaGetDevice(&dev));
    if (beam_kind == HDC_BEAM_FEE &&
        (!fee || fee_num_freqs(fee) != num_freqs || hdc_fee_beam_num_unique_tiles(fee) != 1 || fee_device(fee) != dev)) {
        set_error("hdc_source_brightness_fee: the beam must be prepared on the current device for one tile (the "
                  "ideal delays, unit gains) and the %d frequencies given", num_freqs);
        return HDC_ERR_ARG;
    }
    const int nc = sky->num_components, nf = num_freqs;
    for (int c = 0; c < nc; c++)
        if (h_comp_source[c] < 0 || h_comp_source[c] >= num_sources) {
            set_error("hdc_source_brightness: component %d names source %d of %d", c, h_comp_source[c], num_sources);
            return HDC_ERR_ARG;
        }
    // instrumental flux per (frequency, component): lists on the host, power
    // laws on the device, as the modeller tabulates them
    std::vector<JonesF64> S((size_t)nf * std::max(nc, 1));
    std::vector<FluxComp> fc(std::max(nc, 1));
    std::vector<double2> radec(std::max(nc, 1));
    for (int c = 0; c < nc; c++) {
        const int ft = sky->flux_type[c];
        if (ft < 0 || ft > 2 || sky->fd_count[c] < 1) {
            set_error("hdc_source_brightness: component %d has an invalid flux model", c);
            return HDC_ERR_ARG;
        }
        radec[c] = make_double2(sky->ra[c], sky->dec[c]);
        FluxComp f = {};
        f.flux_type = ft;
        if (ft == HDC_FLUX_LIST) {
            for (int fi = 0; fi < nf; fi++) S[(size_t)fi * nc + c] = inst_stokes(estimate_list(sky, c, h_freqs[fi]));
        } else {
            const Stokes r = fd_entry(sky, sky->fd_start[c]);
            f.freq = r.freq;
            f.i = r.i;
            f.q = r.q;
            f.u = r.u;
            f.v = r.v;
            f.si = sky->si[c];
            f.cq = (ft == HDC_FLUX_CURVED_POWER_LAW) ? sky->q[c] : 0.0;
        }
        fc[c] = f;
    }
    std::vector<double> fd((size_t)num_sources * nf, 0.0);
    std::vector<int> vetoed(num_sources, 0);
    if (nc > 0) {
        JonesF64* d_S = nullptr;
        FluxComp* d_fc = nullptr;
        double2* d_radec = nullptr;
        int *d_src = nullptr, *d_vet = nullptr;
        double *d_freqs = nullptr, *d_fd = nullptr;
        JonesF64* d_B = nullptr;
        int* d_bmap = nullptr;
        auto release = [&]() {
            dfree(d_B);
            dfree(d_bmap);
            dfree(d_S);
            dfree(d_fc);
            dfree(d_radec);
            dfree(d_src);
            dfree(d_vet);
            dfree(d_freqs);
            dfree(d_fd);
        };
        cudaError_t e = dalloc(&d_S, S.size());
        if (e == cudaSuccess) e = dalloc(&d_fc, (size_t)nc);
        if (e == cudaSuccess) e = dalloc(&d_radec, (size_t)nc);
        if (e == cudaSuccess) e = dalloc(&d_src, (size_t)nc);
        if (e == cudaSuccess) e = dalloc(&d_vet, (size_t)num_sources);
        if (e == cudaSuccess) e = dalloc(&d_freqs, (size_t)nf);
        if (e == cudaSuccess) e = dalloc(&d_fd, fd.size());
        if (e == cudaSuccess) e = cudaMemcpy(d_S, S.data(), sizeof(JonesF64) * S.size(), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(d_fc, fc.data(), sizeof(FluxComp) * nc, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(d_radec, radec.data(), sizeof(double2) * nc, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(d_src, h_comp_source, sizeof(int) * nc, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(d_freqs, h_freqs, sizeof(double) * nf, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemset(d_vet, 0, sizeof(int) * num_sources);
        if (e == cudaSuccess) e = cudaMemset(d_fd, 0, sizeof(double) * fd.size());
        int rc_fee = HDC_OK;
        if (e == cudaSuccess && beam_kind == HDC_BEAM_FEE) {
            // the beam's Jones at every component for each unique frequency
            // (on the legacy stream, ahead of the veto kernel)
            e = dalloc(&d_B, (size_t)hdc_fee_beam_num_unique_freqs(fee) * nc);
            if (e == cudaSuccess) e = dalloc(&d_bmap, (size_t)nf);
            if (e == cudaSuccess)
                e = cudaMemcpy(d_bmap, hdc_fee_beam_freq_map(fee), sizeof(int) * nf, cudaMemcpyDeviceToDevice);
            if (e == cudaSuccess) rc_fee = fee_launch_radec(fee, d_radec, nc, lst_rad, latitude_rad, d_B, 0);
        }
        if (e == cudaSuccess && rc_fee == HDC_OK) {
            const dim3 g((nc + 127) / 128, nf);
            flux_kernel<<<g, 128>>>(d_fc, nc, d_freqs, nf, d_S);
            veto_kernel<<<g, 128>>>(d_radec, d_src, nc, d_freqs, nf, lst_rad, latitude_rad, phase_centre.ra,
                                    phase_centre.dec, beam_kind, source_dist_cutoff_rad, min_elevation_rad, d_S,
                                    d_B, d_bmap, d_fd, d_vet);
            count_launches(2);
            e = cudaGetLastError();
        }
        if (rc_fee != HDC_OK) {
            release();
            return rc_fee;
        }
        if (e == cudaSuccess) e = cudaMemcpy(fd.data(), d_fd, sizeof(double) * fd.size(), cudaMemcpyDeviceToHost);
        if (e == cudaSuccess)
            e = cudaMemcpy(vetoed.data(), d_vet, sizeof(int) * num_sources, cudaMemcpyDeviceToHost);
        release();
        if (e != cudaSuccess) {
            set_error("hdc_source_brightness: %s", cudaGetErrorString(e));
            return HDC_ERR_CUDA;
        }
    }
    for (int s = 0; s < num_sources; s++) {
        double m = INFINITY;
        for (int f = 0; f < nf; f++) m = std::min(m, fd[(size_t)s * nf + f]);
        h_brightness[s] = vetoed[s] ? -1.0 : m;
    }
    return HDC_OK;
}
}  // namespace hdc

extern "C" int hdc_source_brightness(const HdcSkyModel* sky, const int* h_comp_source, int num_sources,
                                     const double* h_freqs, int num_freqs, double lst_rad, double latitude_rad,
                                     RADec phase_centre, int beam_kind, double source_dist_cutoff_rad,
                                     double min_elevation_rad, double* h_brightness) {
    if (beam_kind == HDC_BEAM_FEE) {
        hdc::set_error("hdc_source_brightness: the FEE beam goes through hdc_source_brightness_fee");
        return HDC_ERR_ARG;
    }
    return hdc::source_brightness(sky, h_comp_source, num_sources, h_freqs, num_freqs, lst_rad, latitude_rad,
                                  phase_centre, beam_kind, nullptr, source_dist_cutoff_rad, min_elevation_rad,
                                  h_brightness);
}

extern "C" int hdc_source_brightness_fee(const HdcSkyModel* sky, const int* h_comp_source, int num_sources,
                                         const double* h_freqs, int num_freqs, double lst_rad, double latitude_rad,
                                         RADec phase_centre, const HdcFeeBeam* beam, double source_dist_cutoff_rad,
                                         double min_elevation_rad, double* h_brightness) {
    return hdc::source_brightness(sky, h_comp_source, num_sources, h_freqs, num_freqs, lst_rad, latitude_rad,
                                  phase_centre, HDC_BEAM_FEE, beam, source_dist_cutoff_rad, min_elevation_rad,
                                  h_brightness);
}

extern "C" int hdc_modeller_new(const HdcSkyModel* sky, int pols, const XYZ* h_xyzs, int num_tiles,
                                const double* h_freqs, int num_freqs, RADec phase_centre, double array_latitude_rad,
                                int beam_kind, int predict_form, HdcModeller** out) {
    if (!sky || !h_xyzs || !h_freqs || !out || num_tiles < 2 || num_freqs < 1) {
        hdc::set_error("hdc_modeller_new: invalid arguments");
        return HDC_ERR_ARG;
    }
    if (pols < 0 || pols > 4 || beam_kind < 0 || beam_kind > 2 || predict_form < 0 || predict_form > 1) {
        hdc::set_error("hdc_modeller_new: invalid pols/beam/form code");
        return HDC_ERR_ARG;
    }
    Modeller* m = new Modeller();
    cudaGetDevice(&m->device);
    m->pols = pols;
    m->ntiles = num_tiles;
    m->nbl = num_tiles * (num_tiles - 1) / 2;
    m->nf = num_freqs;
    m->pc = phase_centre;
    m->lat = array_latitude_rad;
    m->beam_kind = beam_kind;
    m->form = predict_form;
    m->freqs.assign(h_freqs, h_freqs + num_freqs);
    m->xyzs.assign(h_xyzs, h_xyzs + num_tiles);
    int rc = HDC_OK;
    auto fail = [&](int r) {
        delete m;
        return r;
    };
    if (cudaMalloc(&m->d_freqs, sizeof(double) * num_freqs) != cudaSuccess ||
        cudaMalloc(&m->d_xyzs, sizeof(XYZ) * num_tiles) != cudaSuccess ||
        cudaMalloc(&m->d_uvws, sizeof(UVW) * m->nbl) != cudaSuccess) {
        cudaGetLastError();
        hdc::set_error("hdc_modeller_new: device allocation failed");
        return fail(HDC_ERR_ALLOC);
    }
    cudaMemcpy(m->d_freqs, h_freqs, sizeof(double) * num_freqs, cudaMemcpyHostToDevice);
    cudaMemcpy(m->d_xyzs, h_xyzs, sizeof(XYZ) * num_tiles, cudaMemcpyHostToDevice);
    m->d_sbf = hdc::device_shapelet_basis();
    if (!m->d_sbf) {
        hdc::set_error("hdc_modeller_new: device tables unavailable");
        return fail(HDC_ERR_ALLOC);
    }
    if (cudaMalloc(&m->d_err, sizeof(int)) != cudaSuccess ||
        cudaHostAlloc(&m->h_err, sizeof(int), cudaHostAllocDefault) != cudaSuccess ||
        cudaEventCreateWithFlags(&m->err_ev, cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        hdc::set_error("hdc_modeller_new: device allocation failed");
        return fail(HDC_ERR_ALLOC);
    }
    cudaMemset(m->d_err, 0, sizeof(int));
    *m->h_err = 0;
    cudaEventRecord(m->err_ev, 0);
    rc = m->build_tables(sky);
    if (rc) return fail(rc);
    if (beam_kind == HDC_BEAM_ANALYTIC_PER_TILE) {
        // every dipole at unit gain until hdc_modeller_set_tile_beams
        std::vector<double> ones((size_t)32 * num_tiles, 1.0);
        rc = m->set_tile_beams(ones.data(), 1.28e6);
        if (rc) return fail(rc);
    }
    if (predict_form == HDC_PREDICT_TENSOR) {
        rc = m->tensor_setup();
        if (rc) return fail(rc);
    }
    *out = reinterpret_cast<HdcModeller*>(m);
    return HDC_OK;
}

namespace hdc {
int peel_modeller_new(const HdcSkyModel* sky, const XYZ* h_xyzs, int num_tiles, const double* h_freqs, int num_freqs,
                      RADec phase_centre, const HdcPeelParams* params, HdcModeller** out) {
    const bool fee = params->beam_kind == HDC_BEAM_FEE;
    if (fee && !params->fee_beam) {
        set_error("peel: beam_kind HDC_BEAM_FEE needs fee_beam");
        return HDC_ERR_ARG;
    }
    int rc = hdc_modeller_new(sky, 0, h_xyzs, num_tiles, h_freqs, num_freqs, phase_centre, params->array_latitude_rad,
                              fee ? HDC_BEAM_NONE : params->beam_kind, HDC_PREDICT_DIRECT, out);
    if (rc || !fee) return rc;
    rc = hdc_modeller_set_fee_beam(*out, params->fee_beam);
    if (rc) {
        hdc_modeller_free(*out);
        *out = nullptr;
    }
    return rc;
}
}  // namespace hdc

extern "C" int hdc_modeller_set_tile_beams(HdcModeller* hm, const double* h_dipole_gains, double freq_res_hz) {
    Modeller* m = reinterpret_cast<Modeller*>(hm);
    if (!m) return HDC_ERR_ARG;
    return m->set_tile_beams(h_dipole_gains, freq_res_hz);
}

extern "C" int hdc_modeller_set_fee_beam(HdcModeller* hm, const HdcFeeBeam* b) {
    Modeller* m = reinterpret_cast<Modeller*>(hm);
    if (!m) return HDC_ERR_ARG;
    return m->set_fee_beam(b);
}

extern "C" void hdc_modeller_free(HdcModeller* m) { delete reinterpret_cast<Modeller*>(m); }

extern "C" int hdc_modeller_set_tile_xyzs(HdcModeller* hm, const XYZ* h_xyzs) {
    Modeller* m = reinterpret_cast<Modeller*>(hm);
    if (!m || !h_xyzs) return HDC_ERR_ARG;
    m->xyzs.assign(h_xyzs, h_xyzs + m->ntiles);
    HDC_CUDA_RET_INT(cudaMemcpy(m->d_xyzs, h_xyzs, sizeof(XYZ) * m->ntiles, cudaMemcpyHostToDevice));
    return HDC_OK;
}

extern "C" int hdc_modeller_model_timestep_with(HdcModeller* hm, double lst, JonesF32* d_vis, UVW* h_uvws,
                                                hdcStream_t stream) {
    Modeller* m = reinterpret_cast<Modeller*>(hm);
    if (!m || !d_vis) {
        hdc::set_error("hdc_modeller_model_timestep_with: invalid arguments");
        return HDC_ERR_ARG;
    }
    return m->model(lst, d_vis, false, h_uvws, (cudaStream_t)stream);
}

extern "C" int hdc_modeller_model_timestep_with_f64(HdcModeller* hm, double lst, JonesF64* d_vis, UVW* h_uvws,
                                                    hdcStream_t stream) {
    Modeller* m = reinterpret_cast<Modeller*>(hm);
    if (!m || !d_vis) {
        hdc::set_error("hdc_modeller_model_timestep_with_f64: invalid arguments");
        return HDC_ERR_ARG;
    }
    return m->model(lst, d_vis, true, h_uvws, (cudaStream_t)stream);
}

extern "C" int hdc_modeller_model_timestep_with_host(HdcModeller* hm, double lst, JonesF32* h_vis, UVW* h_uvws,
                                                     hdcStream_t stream) {
    Modeller* m = reinterpret_cast<Modeller*>(hm);
    if (!m || !h_vis) {
        hdc::set_error("hdc_modeller_model_timestep_with_host: invalid arguments");
        return HDC_ERR_ARG;
    }
    cudaStream_t s = (cudaStream_t)stream;
    const size_t bytes = sizeof(JonesF32) * (size_t)m->nf * m->nbl;
    if (m->host_vis_bytes < bytes) {
        if (m->d_host_vis) cudaFree(m->d_host_vis);
        m->d_host_vis = nullptr;
        m->host_vis_bytes = 0;
        HDC_CUDA_RET_INT(cudaMalloc(&m->d_host_vis, bytes));
        m->host_vis_bytes = bytes;
    }
    if (m->form == HDC_PREDICT_TENSOR && !m->tile_beams() && m->t[0].nc > 0 &&
        m->t[0].nc <= hdc::tensor_single_pass() && (m->t[1].nc > 0 || m->t[2].nc > 0)) {
        if (m->host_model_bytes < bytes) {
            if (m->d_host_model) cudaFree(m->d_host_model);
            m->d_host_model = nullptr;
            m->host_model_bytes = 0;
            HDC_CUDA_RET_INT(cudaMalloc(&m->d_host_model, bytes));
            m->host_model_bytes = bytes;
        }
        return m->host_call_drained(m->model_host_points_last(lst, h_vis, h_uvws, s));
    }
    return m->host_call_drained(m->model_host_pipelined(lst, h_vis, h_uvws, s));
}

namespace hdc {
// Channel chunks: chunk c is uploaded on stream 0, predicted on stream 1
// once uploaded, and downloaded on stream 2 once predicted, so the copies of
// one chunk overlap the predict of its neighbours.  The caller's stream
// orders the whole call (the first upload waits for it; it waits for the
// last download), and the call returns with the host buffer updated.
int Modeller::model_host_pipelined(double lst, JonesF32* h_vis, UVW* h_uvws, cudaStream_t s) {
    if (!pipe_s[0]) {
        for (int i = 0; i < 3; i++) HDC_CUDA_RET_INT(cudaStreamCreateWithFlags(&pipe_s[i], cudaStreamNonBlocking));
        for (auto& ev : pipe_ev) HDC_CUDA_RET_INT(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    }
    int rc0 = take_error(false);
    if (rc0) return rc0;
    cudaEvent_t* up = pipe_ev;                      // chunk uploaded
    cudaEvent_t* done = pipe_ev + PIPE_CHUNKS;      // chunk predicted
    cudaEvent_t start = pipe_ev[2 * PIPE_CHUNKS];   // caller's stream reached the call
    cudaEvent_t fin = pipe_ev[2 * PIPE_CHUNKS + 1]; // last download issued
    HDC_CUDA_RET_INT(cudaEventRecord(start, s));
    for (int i = 0; i < 3; i++) HDC_CUDA_RET_INT(cudaStreamWaitEvent(pipe_s[i], start, 0));
    int rc = geometry(lst, pipe_s[1]);
    if (rc) return rc;
    // chunk boundaries: a short first chunk (its upload is the only one the
    // predict waits for) and a short last chunk (its download is the only one
    // nothing overlaps), 1/16 of the channels each; three equal chunks between
    int bounds[PIPE_CHUNKS + 1];
    int nch = 0;
    const int edge = nf / 16;
    if (edge >= 1 && nf - 2 * edge >= PIPE_CHUNKS - 2) {
        nch = PIPE_CHUNKS;
        bounds[0] = 0;
        bounds[1] = edge;
        for (int k = 1; k < PIPE_CHUNKS - 2; k++)
            bounds[1 + k] = edge + (int)((long long)(nf - 2 * edge) * k / (PIPE_CHUNKS - 2));
        bounds[PIPE_CHUNKS - 1] = nf - edge;
        // the tensor point predict runs one CTA per SM and six per channel:
        // middle chunks of a whole number of waves (all but the last) leave no
        // partly filled wave behind
        int n_sm = 0, dev = 0;
        if (t[0].nc > 0 && form == HDC_PREDICT_TENSOR && cudaGetDevice(&dev) == cudaSuccess &&
            cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess && n_sm >= 6) {
            const int mid = nf - 2 * edge, per = (mid + PIPE_CHUNKS - 3) / (PIPE_CHUNKS - 2);
            const int waves = (6 * per + n_sm - 1) / n_sm, c = waves * n_sm / 6;
            if (c >= 1 && (long long)c * (PIPE_CHUNKS - 3) < mid)
                for (int k = 1; k < PIPE_CHUNKS - 2; k++) bounds[1 + k] = edge + k * c;
        }
        bounds[PIPE_CHUNKS] = nf;
    } else {
        nch = std::min(PIPE_CHUNKS, nf);
        for (int k = 0; k <= nch; k++) bounds[k] = (int)((long long)nf * k / nch);
    }
    for (int c = 0; c < nch; c++) {
        const int f0 = bounds[c], f1 = bounds[c + 1];
        const size_t off = (size_t)f0 * nbl, n = (size_t)(f1 - f0) * nbl * sizeof(JonesF32);
        HDC_CUDA_RET_INT(cudaMemcpyAsync(d_host_vis + off, h_vis + off, n, cudaMemcpyHostToDevice, pipe_s[0]));
        HDC_CUDA_RET_INT(cudaEventRecord(up[c], pipe_s[0]));
        HDC_CUDA_RET_INT(cudaStreamWaitEvent(pipe_s[1], up[c], 0));
        rc = model_channels(lst, d_host_vis, false, f0, f1 - f0, pipe_s[1]);
        if (rc) return rc;
        HDC_CUDA_RET_INT(cudaEventRecord(done[c], pipe_s[1]));
        HDC_CUDA_RET_INT(cudaStreamWaitEvent(pipe_s[2], done[c], 0));
        HDC_CUDA_RET_INT(cudaMemcpyAsync(h_vis + off, d_host_vis + off, n, cudaMemcpyDeviceToHost, pipe_s[2]));
    }
    if (h_uvws)
        HDC_CUDA_RET_INT(cudaMemcpyAsync(h_uvws, d_uvws, sizeof(UVW) * nbl, cudaMemcpyDeviceToHost, pipe_s[2]));
    rc = queue_error_check(pipe_s[1]);
    if (rc) return rc;
    HDC_CUDA_RET_INT(cudaEventRecord(fin, pipe_s[2]));
    HDC_CUDA_RET_INT(cudaStreamWaitEvent(s, fin, 0));
    HDC_CUDA_RET_INT(cudaStreamSynchronize(pipe_s[2]));
    return take_error(true);
}
}  // namespace hdc

namespace hdc {
// An error return of a host-buffer call may leave copies of the caller's
// buffer queued: wait for the pipeline's streams first, so that nothing
// reads or writes that buffer after the call returns.
int Modeller::host_call_drained(int rc) {
    if (rc)
        for (auto st : pipe_s)
            if (st) cudaStreamSynchronize(st);
    return rc;
}

namespace {
struct PointsLastCtx {
    Modeller* m;
    JonesF32* h_vis;
    cudaEvent_t ev;
};
// a chunk's points are in: mask its pols, then download it on stream 2
int points_last_chunk_done(void* vctx, int f0, int nch) {
    PointsLastCtx* c = static_cast<PointsLastCtx*>(vctx);
    Modeller* m = c->m;
    const size_t off = (size_t)f0 * m->nbl, n = (size_t)nch * m->nbl;
    HDC_CUDA_RET_INT(launch_mask_pols(m->d_host_vis + off, n, m->pols, m->pipe_s[1]));
    // one event serves every chunk: a wait takes the record made before it
    HDC_CUDA_RET_INT(cudaEventRecord(c->ev, m->pipe_s[1]));
    HDC_CUDA_RET_INT(cudaStreamWaitEvent(m->pipe_s[2], c->ev, 0));
    HDC_CUDA_RET_INT(cudaMemcpyAsync(c->h_vis + off, m->d_host_vis + off, n * sizeof(JonesF32),
                                     cudaMemcpyDeviceToHost, m->pipe_s[2]));
    return HDC_OK;
}
}  // namespace

// Tensor form, shared beam: stream 0 uploads the whole buffer while stream 1
// predicts the Gaussians and shapelets of every channel into d_host_model
// (full-size grids); then the points run in their table chunks (whole waves
// of the Gram kernel), each chunk's visibilities become buffer + staged
// model + points and go back on stream 2 while the next chunk computes.
int Modeller::model_host_points_last(double lst, JonesF32* h_vis, UVW* h_uvws, cudaStream_t s) {
    if (!pipe_s[0]) {
        for (int i = 0; i < 3; i++) HDC_CUDA_RET_INT(cudaStreamCreateWithFlags(&pipe_s[i], cudaStreamNonBlocking));
        for (auto& ev : pipe_ev) HDC_CUDA_RET_INT(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    }
    int rc = take_error(false);
    if (rc) return rc;
    cudaEvent_t start = pipe_ev[0], up = pipe_ev[1], fin = pipe_ev[2];
    HDC_CUDA_RET_INT(cudaEventRecord(start, s));
    for (int i = 0; i < 3; i++) HDC_CUDA_RET_INT(cudaStreamWaitEvent(pipe_s[i], start, 0));
    const size_t bytes = (size_t)nf * nbl * sizeof(JonesF32);
    HDC_CUDA_RET_INT(cudaMemcpyAsync(d_host_vis, h_vis, bytes, cudaMemcpyHostToDevice, pipe_s[0]));
    HDC_CUDA_RET_INT(cudaEventRecord(up, pipe_s[0]));
    rc = geometry(lst, pipe_s[1]);
    if (rc) return rc;
    HDC_CUDA_RET_INT(cudaMemsetAsync(d_host_model, 0, bytes, pipe_s[1]));
    rc = model_channels(lst, d_host_model, false, 0, nf, pipe_s[1], 2 | 4, false);
    if (rc) return rc;
    HDC_CUDA_RET_INT(cudaStreamWaitEvent(pipe_s[1], up, 0));
    void* ws = tensor_workspace(false);
    if (!ws) return HDC_ERR_ALLOC;
    PointsLastCtx ctx{this, h_vis, pipe_ev[3]};
    const TensorChunkOut out{d_host_model, points_last_chunk_done, &ctx};
    EvPair e{};
    prof_begin(0, pipe_s[1], e);
    rc = launch_tensor_points(nf, nbl, ntiles, t[0].nc, d_freqs, d_xyzs, lst - pc.ra, pc.dec, t[0].d_lmn, weights(0),
                              nullptr, d_host_vis, false, ws, d_err, pipe_s[1], tensor_sync(), &out);
    if (rc) return rc;
    prof_end(pipe_s[1], e);
    if (h_uvws)
        HDC_CUDA_RET_INT(cudaMemcpyAsync(h_uvws, d_uvws, sizeof(UVW) * nbl, cudaMemcpyDeviceToHost, pipe_s[2]));
    rc = queue_error_check(pipe_s[1]);
    if (rc) return rc;
    HDC_CUDA_RET_INT(cudaEventRecord(fin, pipe_s[2]));
    HDC_CUDA_RET_INT(cudaStreamWaitEvent(s, fin, 0));
    HDC_CUDA_RET_INT(cudaStreamSynchronize(pipe_s[2]));
    return take_error(true);
}
}  // namespace hdc

extern "C" int hdc_modeller_update_with_a_source(HdcModeller* hm, const HdcSkyModel* source, RADec phase_centre) {
    Modeller* m = reinterpret_cast<Modeller*>(hm);
    if (!m || !source) return HDC_ERR_ARG;
    cudaDeviceSynchronize();
    m->pc = phase_centre;
    int rc = m->build_tables(source);
    if (rc) return rc;
    if (m->form == HDC_PREDICT_TENSOR) return m->tensor_setup();
    return HDC_OK;
}

extern "C" int hdc_modeller_set_profiling(HdcModeller* hm, int enable) {
    Modeller* m = reinterpret_cast<Modeller*>(hm);
    if (!m) return HDC_ERR_ARG;
    m->profiling = enable != 0;
    return HDC_OK;
}

extern "C" int hdc_modeller_profile(HdcModeller* hm, double* out_ms, int reset) {
    Modeller* m = reinterpret_cast<Modeller*>(hm);
    if (!m || !out_ms) return HDC_ERR_ARG;
    m->prof_collect();
    for (int k = 0; k < 4; k++) out_ms[k] = m->prof_ms[k];
    if (reset)
        for (int k = 0; k < 4; k++) m->prof_ms[k] = 0.0;
    return HDC_OK;
}

extern "C" int hdc_modeller_model_timestep_autos_with(HdcModeller* hm, double lst, JonesF32* d_vis,
                                                      hdcStream_t stream) {
    Modeller* m = reinterpret_cast<Modeller*>(hm);
    if (!m || !d_vis) return HDC_ERR_ARG;
    return m->autos(lst, d_vis, (cudaStream_t)stream);
}
