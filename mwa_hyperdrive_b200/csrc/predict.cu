// Direct FP64 sky-model predictor for sm_100a and the drop-in model_* entry
// points (replacing gpu/model.cu of mwa_hyperdrive).
//
// Kernel shape: one thread per (baseline, channel); a CTA covers 256
// consecutive baselines of one channel, so component data is uniform across
// the CTA.  Component tables (LMN, per-channel flux or B S B^H, envelope
// parameters) are streamed through shared memory in chunks by the TMA engine
// (cp.async.bulk) with a two-stage mbarrier pipeline; every thread reads them
// as broadcasts.  The phase 2 pi (u l + v m + w (n - 1)) is formed in turns
// and range-reduced exactly in FP64 (t - rint(t)) before sincospi; the
// accumulation is FP64 and the visibility is updated once per type, as the
// reference does (model/cpu.rs:341-348, gpu/model.cu:171).

#include <atomic>
#include <cstdio>
#include <vector>

#include "predict.cuh"

namespace hdc {

constexpr int DT = 256;  // threads (baselines) per CTA
constexpr int CH = 64;   // components per staged chunk

template <int TYPE>
__device__ __forceinline__ cplx shapelet_envelope(const DirectParams& p, int c, double4 g, double su, double sv) {
    const double x = su * g.z + sv * g.w;
    const double y = su * g.w - sv * g.z;
    const double x_pos = x * g.x + SBF_C;
    const double y_pos = y * g.y + SBF_C;
    const double fx = floor(x_pos), fy = floor(y_pos);
    // Negative positions clamp to 0 as in the reference (gpu/model.cu:63-64;
    // on the CPU path the saturating usize cast does the same); positions past
    // the table end clamp to the last interval so no read leaves the table.
    int xi = fx > 0.0 ? (int)fmin(fx, (double)(SBF_L - 2)) : 0;
    int yi = fy > 0.0 ? (int)fmin(fy, (double)(SBF_L - 2)) : 0;
    const double xfrac = x_pos - fx, yfrac = y_pos - fy;
    const int start = __ldg(p.coeff_start + c), count = __ldg(p.coeff_count + c);
    cplx env = {0.0, 0.0};
    for (int i = 0; i < count; i++) {
        const ShapeletCoeff co = p.coeffs[start + i];
        const double* bx = p.sbf + (size_t)SBF_L * co.n1 + xi;
        const double* by = p.sbf + (size_t)SBF_L * co.n2 + yi;
        const double x_low = __ldg(bx), x_high = __ldg(bx + 1);
        const double y_low = __ldg(by), y_high = __ldg(by + 1);
        const double u_value = x_low + (x_high - x_low) * xfrac;
        const double v_value = y_low + (y_high - y_low) * yfrac;
        const double rest = co.value * u_value * v_value;
        switch ((co.n1 + co.n2) & 3) {
            case 0: env.re += rest; break;
            case 1: env.im += rest; break;
            case 2: env.re -= rest; break;
            default: env.im -= rest; break;
        }
    }
    return env;
}

// The chosen form's shapelet envelope: table positions in FP64 (an FP32
// position near 5000 would move the interpolation point by ~1e-3 of a table
// step), basis values from the FP32 copy of the table, interpolation and
// products in FP32.
__device__ __forceinline__ void shapelet_envelope_f32(const DirectParams& p, int c, double4 g, double su, double sv,
                                                      float& er, float& ei) {
    const double x = su * g.z + sv * g.w;
    const double y = su * g.w - sv * g.z;
    const double x_pos = x * g.x + SBF_C;
    const double y_pos = y * g.y + SBF_C;
    const double fx = floor(x_pos), fy = floor(y_pos);
    const int xi = fx > 0.0 ? (int)fmin(fx, (double)(SBF_L - 2)) : 0;
    const int yi = fy > 0.0 ? (int)fmin(fy, (double)(SBF_L - 2)) : 0;
    const float xfrac = (float)(x_pos - fx), yfrac = (float)(y_pos - fy);
    const int start = __ldg(p.coeff_start + c), count = __ldg(p.coeff_count + c);
    float re = 0.f, im = 0.f;
    for (int i = 0; i < count; i++) {
        const ShapeletCoeff co = p.coeffs[start + i];
        const float* bx = p.sbf32 + (size_t)SBF_L * co.n1 + xi;
        const float* by = p.sbf32 + (size_t)SBF_L * co.n2 + yi;
        const float2 xv = make_float2(__ldg(bx), __ldg(bx + 1));
        const float2 yv = make_float2(__ldg(by), __ldg(by + 1));
        const float u_value = fmaf(xv.y - xv.x, xfrac, xv.x);
        const float v_value = fmaf(yv.y - yv.x, yfrac, yv.x);
        const float rest = (float)co.value * u_value * v_value;
        switch ((co.n1 + co.n2) & 3) {
            case 0: re += rest; break;
            case 1: im += rest; break;
            case 2: re -= rest; break;
            default: im -= rest; break;
        }
    }
    er = re;
    ei = im;
}

// The chosen form's dense shapelet envelope (every order below SDN): the
// basis is interpolated once per order along each axis (one 8-byte gather of
// a (value, next - value) pair each), then contracted with the component's
// signed dense coefficient matrix C (shared memory):
//     env = sum_{n1,n2} C[n1][n2] X[n1] Y[n2],  even n1 + n2 -> re, odd -> im.
__device__ __forceinline__ void shapelet_dense_at(const DirectParams& p, const float* __restrict__ cm, double x_pos,
                                                  double y_pos, float& er, float& ei) {
    const double fx = floor(x_pos), fy = floor(y_pos);
    const int xi = fx > 0.0 ? (int)fmin(fx, (double)(SBF_L - 2)) : 0;
    const int yi = fy > 0.0 ? (int)fmin(fy, (double)(SBF_L - 2)) : 0;
    const float xfrac = (float)(x_pos - fx), yfrac = (float)(y_pos - fy);
    // one 48-byte record per position holds all orders' pairs
    float X[SDN], Y[SDN];
#pragma unroll
    for (int h = 0; h < SDN / 2; h++) {
        const float4 a = __ldg(p.sbfp + (size_t)xi * (SDN / 2) + h);
        const float4 b = __ldg(p.sbfp + (size_t)yi * (SDN / 2) + h);
        X[2 * h] = fmaf(a.y, xfrac, a.x);
        X[2 * h + 1] = fmaf(a.w, xfrac, a.z);
        Y[2 * h] = fmaf(b.y, yfrac, b.x);
        Y[2 * h + 1] = fmaf(b.w, yfrac, b.z);
    }
    float re = 0.f, im = 0.f;
#pragma unroll
    for (int n1 = 0; n1 < SDN; n1++) {
        float tr = 0.f, ti = 0.f;
#pragma unroll
        for (int n2 = 0; n2 < SDN; n2++) {
            if ((n1 + n2) & 1)
                ti = fmaf(cm[n1 * SDN + n2], Y[n2], ti);
            else
                tr = fmaf(cm[n1 * SDN + n2], Y[n2], tr);
        }
        re = fmaf(X[n1], tr, re);
        im = fmaf(X[n1], ti, im);
    }
    er = re;
    ei = im;
}

__device__ __forceinline__ void shapelet_envelope_dense(const DirectParams& p, const float* __restrict__ cm,
                                                        double4 g, double su, double sv, float& er, float& ei) {
    const double x = su * g.z + sv * g.w;
    const double y = su * g.w - sv * g.z;
    shapelet_dense_at(p, cm, x * g.x + SBF_C, y * g.y + SBF_C, er, ei);
}

// shapelet_dense_at for N channels of one component at once: the basis of
// each channel is interpolated as there, and each row of the coefficient
// matrix is read from shared memory once (three 8-byte loads) for all N
// channels; same arithmetic order per channel
template <int N>
__device__ __forceinline__ void shapelet_dense_multi(const DirectParams& p, const float* __restrict__ cm,
                                                     const double (&x_pos)[N], const double (&y_pos)[N],
                                                     float (&er)[N], float (&ei)[N]) {
    float X[N][SDN], Y[N][SDN];
    int xi[N], yi[N];
    float xfrac[N], yfrac[N];
#pragma unroll
    for (int i = 0; i < N; i++) {
        const double fx = floor(x_pos[i]), fy = floor(y_pos[i]);
        xi[i] = fx > 0.0 ? (int)fmin(fx, (double)(SBF_L - 2)) : 0;
        yi[i] = fy > 0.0 ? (int)fmin(fy, (double)(SBF_L - 2)) : 0;
        xfrac[i] = (float)(x_pos[i] - fx);
        yfrac[i] = (float)(y_pos[i] - fy);
        er[i] = 0.f, ei[i] = 0.f;
    }
    // A thread's channels usually share a table interval (their positions
    // differ by the channels' relative frequency spacing): a channel whose
    // interval equals the previous channel's takes its records instead of
    // gathering them again, so only lanes with a new interval load.
#pragma unroll
    for (int h = 0; h < SDN / 2; h++) {
        float4 a, b;
#pragma unroll
        for (int i = 0; i < N; i++) {
            if (i == 0 || xi[i] != xi[i - 1]) a = __ldg(p.sbfp + (size_t)xi[i] * (SDN / 2) + h);
            if (i == 0 || yi[i] != yi[i - 1]) b = __ldg(p.sbfp + (size_t)yi[i] * (SDN / 2) + h);
            X[i][2 * h] = fmaf(a.y, xfrac[i], a.x);
            X[i][2 * h + 1] = fmaf(a.w, xfrac[i], a.z);
            Y[i][2 * h] = fmaf(b.y, yfrac[i], b.x);
            Y[i][2 * h + 1] = fmaf(b.w, yfrac[i], b.z);
        }
    }
    const float2* row = reinterpret_cast<const float2*>(cm);
#pragma unroll
    for (int n1 = 0; n1 < SDN; n1++) {
        float c[SDN];
#pragma unroll
        for (int h = 0; h < SDN / 2; h++) {
            const float2 v = row[n1 * (SDN / 2) + h];
            c[2 * h] = v.x, c[2 * h + 1] = v.y;
        }
#pragma unroll
        for (int i = 0; i < N; i++) {
            float tr = 0.f, ti = 0.f;
#pragma unroll
            for (int n2 = 0; n2 < SDN; n2++) {
                if ((n1 + n2) & 1)
                    ti = fmaf(c[n2], Y[i][n2], ti);
                else
                    tr = fmaf(c[n2], Y[i][n2], tr);
            }
            er[i] = fmaf(X[i][n1], tr, er[i]);
            ei[i] = fmaf(X[i][n1], ti, ei[i]);
        }
    }
}

// FAST (the chosen form's Gaussians and shapelets, shared beam only): the
// phasor from the FP32 quarter-turn polynomials after exact FP64 range
// reduction, envelopes in FP32 (arguments and table positions in FP64),
// each component's term W ph env in FP32
// (W staged once per chunk as FP32), summed in FP32 within a 64-component
// chunk and in FP64 across chunks.  Error ~1e-7 of the visibility.
template <int TYPE, bool TILE_BEAM, bool OUT64, bool FAST>
__global__ void __launch_bounds__(DT) direct_kernel(const DirectParams p) {
    __shared__ alignas(128) double4 s_lmn[2][CH];
    __shared__ alignas(128) JonesF64 s_flux[2][CH];
    __shared__ alignas(128) double4 s_gp[2][CH];
    __shared__ alignas(16) float s_wf[FAST ? CH * 8 : 1];
    __shared__ alignas(16) float s_dense[(FAST && TYPE == 2) ? CH * SDN * SDN : 1];
    __shared__ alignas(8) uint64_t bar[2];

    const int f = blockIdx.y;
    const int bl = blockIdx.x * DT + threadIdx.x;
    const bool active = bl < p.nbl;
    int t1 = 0, t2 = 1;
    if (active) baseline_to_tiles(bl, p.ntiles, t1, t2);

    const double freq = p.freqs[f];
    const double ool = freq / VEL_C;
    double u = 0.0, v = 0.0, w = 0.0;
    if (active) {
        const UVW q = p.uvws[bl];
        if (TYPE == 2) {
            u = q.u * ool;
            v = q.v * ool;
            w = q.w * ool;
        } else {
            u = q.u * freq / VEL_C;
            v = q.v * freq / VEL_C;
            w = q.w * freq / VEL_C;
        }
    }
    const JonesF64* b1 = nullptr;
    const JonesF64* b2 = nullptr;
    if (TILE_BEAM && active) {
        int u1 = p.unflagged_map ? p.unflagged_map[t1] : t1;
        int u2 = p.unflagged_map ? p.unflagged_map[t2] : t2;
        const int col = p.freq_map[f];
        b1 = p.beam + (size_t)p.nc * ((size_t)p.n_uniq_freq * p.tile_map[u1] + col);
        b2 = p.beam + (size_t)p.nc * ((size_t)p.n_uniq_freq * p.tile_map[u2] + col);
    }

    const int nchunks = (p.nc + CH - 1) / CH;
    if (threadIdx.x == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        fence_barrier_init();
    }
    __syncthreads();

    auto issue = [&](int k) {
        const int st = k & 1;
        const int c0 = k * CH;
        const int n = min(CH, p.nc - c0);
        const uint32_t bytes = n * 32u + n * 64u + (TYPE ? n * 32u : 0u);
        mbar_arrive_expect_tx(&bar[st], bytes);
        bulk_g2s(s_lmn[st], p.lmn + c0, n * 32u, &bar[st]);
        bulk_g2s(s_flux[st], p.flux + (size_t)f * p.nc + c0, n * 64u, &bar[st]);
        if (TYPE) bulk_g2s(s_gp[st], p.gp + c0, n * 32u, &bar[st]);
    };
    int issued = 0;  // chunks whose copies thread 0 has issued
    if (threadIdx.x == 0) {
        fence_proxy_async_smem();
        if (!p.stall) {
            if (nchunks > 0) issue(0), issued = 1;
            if (nchunks > 1) issue(1), issued = 2;
        }
    }
    const uint64_t limit = p.wait_ns ? p.wait_ns : 2000000000ull;

    J2 acc = jzero();
    bool aborted = false;
    for (int k = 0; k < nchunks; k++) {
        const int st = k & 1;
        const bool ok = mbar_wait_bounded(&bar[st], (k >> 1) & 1, p.err, limit);
        if (__syncthreads_or(!ok)) {
            // the sum is incomplete: leave the visibilities untouched
            if (threadIdx.x == 0) drain_two_stage(bar, k, issued);
            aborted = true;
            break;
        }
        const int c0 = k * CH;
        const int n = min(CH, p.nc - c0);
        if (FAST) {
            const double* src = reinterpret_cast<const double*>(s_flux[st]);
            for (int i = threadIdx.x; i < n * 8; i += DT) s_wf[i] = (float)src[i];
            if (TYPE == 2 && p.sdense)
                for (int i = threadIdx.x; i < n * SDN * SDN; i += DT)
                    s_dense[i] = __ldg(p.sdense + (size_t)c0 * SDN * SDN + i);
            __syncthreads();
        }
        if (FAST && active) {
            float a[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
            for (int c = 0; c < n; c++) {
                const double4 lmn = s_lmn[st][c];
                float sn, cs;
                phasor_quarter_f32(4.0 * (u * lmn.x + v * lmn.y + w * lmn.z), sn, cs);
                float er = 1.f, ei = 0.f;
                if (TYPE == 1) {
                    // the exponent in FP64 (an FP32 exponent's absolute error,
                    // ~1e-7 of its size, would become the envelope's relative
                    // error); exp of its FP32 head, first order in the tail
                    const double4 g = s_gp[st][c];
                    const double kx = u * g.z + v * g.w;
                    const double ky = u * g.w - v * g.z;
                    const double ex = g.x * (kx * kx) + g.y * (ky * ky);
                    const float exh = (float)ex;
                    er = expf(exh) * (1.f + (float)(ex - (double)exh));
                } else if (TYPE == 2) {
                    const double4 g = s_gp[st][c];
                    const double2 ta = __ldg(p.suv_tile + (size_t)(c0 + c) * p.ntiles + t1);
                    const double2 tb = __ldg(p.suv_tile + (size_t)(c0 + c) * p.ntiles + t2);
                    if (p.sdense)
                        shapelet_envelope_dense(p, s_dense + c * SDN * SDN, g, (ta.x - tb.x) * ool,
                                                (ta.y - tb.y) * ool, er, ei);
                    else
                        shapelet_envelope_f32(p, c0 + c, g, (ta.x - tb.x) * ool, (ta.y - tb.y) * ool, er, ei);
                }
                // ph * env
                const float zr = cs * er - sn * ei, zi = fmaf(cs, ei, sn * er);
                const float* wv = s_wf + c * 8;
#pragma unroll
                for (int e = 0; e < 4; e++) {
                    a[2 * e] += fmaf(wv[2 * e], zr, -wv[2 * e + 1] * zi);
                    a[2 * e + 1] += fmaf(wv[2 * e], zi, wv[2 * e + 1] * zr);
                }
            }
            acc = acc + J2{{a[0], a[1]}, {a[2], a[3]}, {a[4], a[5]}, {a[6], a[7]}};
        } else if (active) {
            for (int c = 0; c < n; c++) {
                const double4 lmn = s_lmn[st][c];
                J2 wj = load_j(s_flux[st][c]);
                if (TILE_BEAM) {
                    const J2 j1 = ldg_j(b1 + c0 + c);
                    const J2 j2 = ldg_j(b2 + c0 + c);
                    wj = (j1 * wj) * herm(j2);
                }
                const double t = u * lmn.x + v * lmn.y + w * lmn.z;
                const cplx ph = phasor_turns(t);
                if (TYPE == 0) {
                    acc = acc + wj * ph;
                } else if (TYPE == 1) {
                    const double4 g = s_gp[st][c];
                    const double kx = u * g.z + v * g.w;
                    const double ky = u * g.w - v * g.z;
                    const double env = exp(g.x * (kx * kx) + g.y * (ky * ky));
                    acc = acc + (wj * ph) * env;
                } else {
                    const double4 g = s_gp[st][c];
                    double su, sv;
                    if (p.suv_bl) {
                        const ShapeletUV q = p.suv_bl[(size_t)bl * p.nc + c0 + c];
                        su = q.u;
                        sv = q.v;
                    } else {
                        const double2 a = __ldg(p.suv_tile + (size_t)(c0 + c) * p.ntiles + t1);
                        const double2 b = __ldg(p.suv_tile + (size_t)(c0 + c) * p.ntiles + t2);
                        su = a.x - b.x;
                        sv = a.y - b.y;
                    }
                    const cplx env = shapelet_envelope<TYPE>(p, c0 + c, g, su * ool, sv * ool);
                    acc = acc + (wj * ph) * env;
                }
            }
        }
        __syncthreads();
        if (threadIdx.x == 0 && k + 2 < nchunks) {
            fence_proxy_async_smem();
            issue(k + 2);
            issued = k + 3;
        }
    }

    if (!active || aborted) return;
    const size_t o = (size_t)f * p.nbl + bl;
    if (OUT64) {
        double2* q = reinterpret_cast<double2*>(reinterpret_cast<JonesF64*>(p.vis) + o);
        double2 a = q[0], b = q[1], c = q[2], d = q[3];
        q[0] = make_double2(a.x + acc.a.re, a.y + acc.a.im);
        q[1] = make_double2(b.x + acc.b.re, b.y + acc.b.im);
        q[2] = make_double2(c.x + acc.c.re, c.y + acc.c.im);
        q[3] = make_double2(d.x + acc.d.re, d.y + acc.d.im);
    } else {
        float4* q = reinterpret_cast<float4*>(reinterpret_cast<JonesF32*>(p.vis) + o);
        float4 a = q[0], b = q[1];
        a.x += (float)acc.a.re;
        a.y += (float)acc.a.im;
        a.z += (float)acc.b.re;
        a.w += (float)acc.b.im;
        b.x += (float)acc.c.re;
        b.y += (float)acc.c.im;
        b.z += (float)acc.d.re;
        b.w += (float)acc.d.im;
        q[0] = a;
        q[1] = b;
    }
}

// The channel-independent FP64 work of one Gaussian or shapelet term of the
// chosen form at baseline (um, vm, wm) [m] (tiles t1, t2): the phase in
// metres, the Gaussian exponent in metres^2 (base 2) or the shapelet
// coordinates, and the dense shapelet envelopes of the FCH channels (cm:
// the component's dense coefficient matrix in shared memory, or NULL).
template <int TYPE, int FCH>
struct FastTerm {
    double tm, exm, su, sv;
    float der[FCH], dei[FCH];
};

template <int TYPE, int FCH>
__device__ __forceinline__ void fast_term(const DirectParams& p, double4 lmn, double4 g, double um, double vm, double wm,
                                          int cglob, int t1, int t2, const double (&ool)[FCH], const float* cm,
                                          FastTerm<TYPE, FCH>& f) {
    f.tm = um * lmn.x + vm * lmn.y + wm * lmn.z;
    f.exm = f.su = f.sv = 0.0;
    if (TYPE == 1) {
        // the exponent in FP64 (an FP32 exponent's absolute error, ~1e-7 of
        // its size, would become the envelope's relative error), in base 2
        // (exp(x) = 2^(x log2 e)): the per-channel exp2f costs fewer
        // instructions than expf (measured)
        const double kx = um * g.z + vm * g.w;
        const double ky = um * g.w - vm * g.z;
        f.exm = (g.x * (kx * kx) + g.y * (ky * ky)) * 1.4426950408889634074;
    } else {
        const double2 ta = __ldg(p.suv_tile + (size_t)cglob * p.ntiles + t1);
        const double2 tb = __ldg(p.suv_tile + (size_t)cglob * p.ntiles + t2);
        f.su = ta.x - tb.x;
        f.sv = ta.y - tb.y;
        if (cm) {
            const double xm = f.su * g.z + f.sv * g.w;
            const double ym = f.su * g.w - f.sv * g.z;
            double xp[FCH], yp[FCH];
#pragma unroll
            for (int i = 0; i < FCH; i++) {
                xp[i] = xm * (ool[i] * g.x) + SBF_C;
                yp[i] = ym * (ool[i] * g.y) + SBF_C;
            }
            shapelet_dense_multi<FCH>(p, cm, xp, yp, f.der, f.dei);
        }
    }
}

// z = envelope x phasor of channel i of a FastTerm (ool_i = its frequency / c).
template <int TYPE, int FCH>
__device__ __forceinline__ void fast_z(const DirectParams& p, const FastTerm<TYPE, FCH>& f, int i, double ool_i,
                                       int cglob, double4 g, bool dense, float& zr, float& zi) {
    float sn, cs;
    phasor_quarter_f32(4.0 * ool_i * f.tm, sn, cs);
    if (TYPE == 1) {
        // exponent in FP64, exp2 in FP32: rounding the exponent to FP32 moves
        // the envelope by ln2 |x| 6e-8 2^-|x| <= 2.2e-8 of the component's flux;
        // a Gaussian's envelope is real
        const float er = exp2f((float)(f.exm * (ool_i * ool_i)));
        zr = cs * er;
        zi = sn * er;
    } else {
        float er, ei;
        if (dense) {
            er = f.der[i];
            ei = f.dei[i];
        } else {
            shapelet_envelope_f32(p, cglob, g, f.su * ool_i, f.sv * ool_i, er, ei);
        }
        zr = cs * er - sn * ei;
        zi = fmaf(cs, ei, sn * er);
    }
}

// vis[o] += acc (JonesF64 or JonesF32 [channel][baseline] at element o).
template <bool OUT64>
__device__ __forceinline__ void add_vis(void* vis, size_t o, const J2& acc) {
    if (OUT64) {
        double2* q = reinterpret_cast<double2*>(reinterpret_cast<JonesF64*>(vis) + o);
        const double2 a0 = q[0], b0 = q[1], c0 = q[2], d0 = q[3];
        q[0] = make_double2(a0.x + acc.a.re, a0.y + acc.a.im);
        q[1] = make_double2(b0.x + acc.b.re, b0.y + acc.b.im);
        q[2] = make_double2(c0.x + acc.c.re, c0.y + acc.c.im);
        q[3] = make_double2(d0.x + acc.d.re, d0.y + acc.d.im);
    } else {
        float4* q = reinterpret_cast<float4*>(reinterpret_cast<JonesF32*>(vis) + o);
        float4 x = q[0], y = q[1];
        x.x += (float)acc.a.re;
        x.y += (float)acc.a.im;
        x.z += (float)acc.b.re;
        x.w += (float)acc.b.im;
        y.x += (float)acc.c.re;
        y.y += (float)acc.c.im;
        y.z += (float)acc.d.re;
        y.w += (float)acc.d.im;
        q[0] = x;
        q[1] = y;
    }
}

// The chosen form's Gaussians and shapelets with FCH channels per thread: a
// CTA covers 256 baselines of FCH consecutive channels, so each component's
// FP64 work that does not depend on the channel -- the phase in metres, the
// Gaussian exponent in metres^2, the shapelet coordinates, their shared-
// memory and table-position loads -- is done once for all FCH channels and
// only scaled per channel (lambda^-1 for the phase and positions, lambda^-2
// for the exponent).  The arithmetic per channel is that of the FAST
// direct_kernel above, except that the accumulation uses W's Hermitian
// symmetry (a shared beam).  Channels per thread, CTAs per SM and components
// per staged chunk by type, chosen by timing: Gaussians (1) 4 channels, 2 CTAs
// per SM, 64 components; shapelets (2) the same but 32 components, to keep
// the static shared memory under 48 KB with the per-channel basis
// coordinates (4 channels beat 2 once a thread's channels share the gathered
// basis-table records: 10.2 against 11.5 ms per mixed step).
template <int TYPE>
struct FastShape {
    static constexpr int FCH = 4;
    static constexpr int MIN_CTAS = 2;
    static constexpr int CHUNK = 64;
};
template <>
struct FastShape<2> {
    static constexpr int FCH = 4;
    static constexpr int MIN_CTAS = 2;
    static constexpr int CHUNK = 32;
};

template <int TYPE, bool OUT64>
__global__ void __launch_bounds__(DT, FastShape<TYPE>::MIN_CTAS) fast_kernel(const DirectParams p) {
    constexpr int FCH = FastShape<TYPE>::FCH;
    constexpr int CH = FastShape<TYPE>::CHUNK;  // components per staged chunk
    __shared__ alignas(128) double4 s_lmn[2][CH];
    __shared__ alignas(128) JonesF64 s_flux[2][FCH][CH];
    __shared__ alignas(128) double4 s_gp[2][CH];
    // W of each channel as (XX, YY, Re XY, Im XY): this kernel runs with a
    // beam shared by all tiles (or none), where W = B S B^H is Hermitian
    // (XX and YY real, YX = conj XY)
    __shared__ alignas(16) float s_wf[FCH][CH * 4];
    __shared__ alignas(16) float s_dense[TYPE == 2 ? CH * SDN * SDN : 1];
    __shared__ alignas(8) uint64_t bar[2];

    const int f0 = blockIdx.y * FCH;
    const int bl = blockIdx.x * DT + threadIdx.x;
    const bool active = bl < p.nbl;
    int t1 = 0, t2 = 1;
    if (active) baseline_to_tiles(bl, p.ntiles, t1, t2);
    int fr[FCH];
    double ool[FCH];
#pragma unroll
    for (int i = 0; i < FCH; i++) {
        fr[i] = min(f0 + i, p.nf - 1);  // a missing last channel repeats the previous one and is not stored
        ool[i] = p.freqs[fr[i]] / VEL_C;
    }
    double um = 0.0, vm = 0.0, wm = 0.0;
    if (active) {
        const UVW q = p.uvws[bl];
        um = q.u, vm = q.v, wm = q.w;
    }

    const int nchunks = (p.nc + CH - 1) / CH;
    if (threadIdx.x == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        fence_barrier_init();
    }
    __syncthreads();

    auto issue = [&](int k) {
        const int st = k & 1;
        const int c0 = k * CH;
        const int n = min(CH, p.nc - c0);
        const uint32_t bytes = n * 32u + FCH * n * 64u + n * 32u;
        mbar_arrive_expect_tx(&bar[st], bytes);
        bulk_g2s(s_lmn[st], p.lmn + c0, n * 32u, &bar[st]);
#pragma unroll
        for (int i = 0; i < FCH; i++) bulk_g2s(s_flux[st][i], p.flux + (size_t)fr[i] * p.nc + c0, n * 64u, &bar[st]);
        bulk_g2s(s_gp[st], p.gp + c0, n * 32u, &bar[st]);
    };
    int issued = 0;  // chunks whose copies thread 0 has issued
    if (threadIdx.x == 0) {
        fence_proxy_async_smem();
        if (!p.stall) {
            if (nchunks > 0) issue(0), issued = 1;
            if (nchunks > 1) issue(1), issued = 2;
        }
    }
    const uint64_t limit = p.wait_ns ? p.wait_ns : 2000000000ull;

    J2 acc[FCH];
#pragma unroll
    for (int i = 0; i < FCH; i++) acc[i] = jzero();
    bool aborted = false;
    for (int k = 0; k < nchunks; k++) {
        const int st = k & 1;
        const bool ok = mbar_wait_bounded(&bar[st], (k >> 1) & 1, p.err, limit);
        if (__syncthreads_or(!ok)) {
            // the sum is incomplete: leave the visibilities untouched
            if (threadIdx.x == 0) drain_two_stage(bar, k, issued);
            aborted = true;
            break;
        }
        const int c0 = k * CH;
        const int n = min(CH, p.nc - c0);
#pragma unroll
        for (int i = 0; i < FCH; i++) {
            const double* src = reinterpret_cast<const double*>(s_flux[st][i]);
            for (int e = threadIdx.x; e < n * 4; e += DT) {
                const int q = e & 3;  // XX re (0), YY re (6), XY re (2), XY im (3) of the component's 8
                s_wf[i][e] = (float)src[(e >> 2) * 8 + (q == 0 ? 0 : (q == 1 ? 6 : q))];
            }
        }
        if (TYPE == 2 && p.sdense)
            for (int e = threadIdx.x; e < n * SDN * SDN; e += DT) s_dense[e] = __ldg(p.sdense + (size_t)c0 * SDN * SDN + e);
        __syncthreads();
        if (active) {
            float a[FCH][8];
#pragma unroll
            for (int i = 0; i < FCH; i++)
#pragma unroll
                for (int e = 0; e < 8; e++) a[i][e] = 0.f;
            for (int c = 0; c < n; c++) {
                const double4 g = s_gp[st][c];
                FastTerm<TYPE, FCH> term;
                fast_term<TYPE, FCH>(p, s_lmn[st][c], g, um, vm, wm, c0 + c, t1, t2, ool,
                                     TYPE == 2 && p.sdense ? s_dense + c * SDN * SDN : nullptr, term);
#pragma unroll
                for (int i = 0; i < FCH; i++) {
                    float zr, zi;
                    fast_z<TYPE, FCH>(p, term, i, ool[i], c0 + c, g, p.sdense != nullptr, zr, zi);
                    // a += W z with W Hermitian: 12 fused multiply-adds
                    const float4 wv = *reinterpret_cast<const float4*>(s_wf[i] + c * 4);
                    a[i][0] = fmaf(wv.x, zr, a[i][0]);
                    a[i][1] = fmaf(wv.x, zi, a[i][1]);
                    a[i][2] = fmaf(-wv.w, zi, fmaf(wv.z, zr, a[i][2]));
                    a[i][3] = fmaf(wv.w, zr, fmaf(wv.z, zi, a[i][3]));
                    a[i][4] = fmaf(wv.w, zi, fmaf(wv.z, zr, a[i][4]));
                    a[i][5] = fmaf(-wv.w, zr, fmaf(wv.z, zi, a[i][5]));
                    a[i][6] = fmaf(wv.y, zr, a[i][6]);
                    a[i][7] = fmaf(wv.y, zi, a[i][7]);
                }
            }
#pragma unroll
            for (int i = 0; i < FCH; i++)
                acc[i] = acc[i] + J2{{a[i][0], a[i][1]}, {a[i][2], a[i][3]}, {a[i][4], a[i][5]}, {a[i][6], a[i][7]}};
        }
        __syncthreads();
        if (threadIdx.x == 0 && k + 2 < nchunks) {
            fence_proxy_async_smem();
            issue(k + 2);
            issued = k + 3;
        }
    }

    if (!active || aborted) return;
#pragma unroll
    for (int i = 0; i < FCH; i++) {
        if (f0 + i >= p.nf) break;
        add_vis<OUT64>(p.vis, (size_t)(f0 + i) * p.nbl + bl, acc[i]);
    }
}

// The chosen form's Gaussians and shapelets with a beam per tile: each
// thread takes one baseline (p, q) and FastTileShape::FCH consecutive channels, as
// fast_kernel does.  Per staged chunk of components the CTA forms in shared
// memory G = B_u S (FP32) and H = B_u (FP64) for every unique tile u and each
// of its channels (B the tile's beam Jones at the channel's beam frequency,
// S the component's instrumental flux), laid out [channel][component][unique
// tile] so that a warp's threads, which share tile p and mostly share the
// unique beam of tile q, read the same or neighbouring records.  A
// visibility term is then z G_p H_q^H = B_p (z S) B_q^H: the phasor and
// envelope z in FP32 exactly as fast_kernel computes them, z G_p in FP32,
// and its product with H_q^H accumulated in FP64 (32 fused multiply-adds).
// Measured on the tests' skies (p99.9 of the error, Gaussians / shapelets):
// this form 3.4e-7 / 5.3e-7; FP32 two-product sums added into FP64
// accumulators 4.2e-7 / 5.9e-7 (7 % faster Gaussians); everything in FP32,
// chunk sums included, 1.0-1.15e-6, over the 1e-6 bar.
// Channels per thread and components per staged chunk by type, chosen by
// timing on 17 unique tiles (one timestep, 128 tiles, 384 channels):
// Gaussians (1) 2 x 16 (4 x 8: 9.4 -> 10.8 ms, 156 registers); shapelets (2)
// 4 x 8, whose channels then share more gathered basis records (2 x 16: 5.4
// ms, 4 x 8: 4.6 ms, bit-identical).  Both stage 32 (channel, component)
// records per unique tile, so the shared memory does not depend on the type.
template <int TYPE>
struct FastTileShape {
    static constexpr int FCH = 2;
    static constexpr int CH = 16;
};
template <>
struct FastTileShape<2> {
    static constexpr int FCH = 4;
    static constexpr int CH = 8;
};
constexpr int FT_RECS = 32;    // FCH x CH of every type
constexpr int FT_MAX_NU = 32;  // unique tiles (more: the FP64 per-tile kernel)
static_assert(FastTileShape<1>::FCH * FastTileShape<1>::CH == FT_RECS, "per-tile records");
static_assert(FastTileShape<2>::FCH * FastTileShape<2>::CH == FT_RECS, "per-tile records");

inline size_t fast_tile_smem_bytes(int nu) { return (size_t)FT_RECS * nu * 6 * sizeof(float4); }

template <int TYPE, bool OUT64>
__global__ void __launch_bounds__(DT, 1) fast_tile_kernel(const DirectParams p) {
    constexpr int FCH = FastTileShape<TYPE>::FCH;
    constexpr int CH = FastTileShape<TYPE>::CH;
    __shared__ alignas(128) double4 s_lmn[2][CH];
    __shared__ alignas(128) JonesF64 s_flux[2][FCH][CH];
    __shared__ alignas(128) double4 s_gp[2][CH];
    __shared__ alignas(16) float s_dense[TYPE == 2 ? CH * SDN * SDN : 1];
    __shared__ alignas(8) uint64_t bar[2];
    // [FCH][CH][nu] records of 96 bytes: G (2 float4: a, b | c, d), then H
    // (4 double2: a, b, c, d)
    extern __shared__ float4 s_gh[];
    const int nu = p.n_uniq_tile;

    const int f0 = blockIdx.y * FCH;
    const int bl = blockIdx.x * DT + threadIdx.x;
    const bool active = bl < p.nbl;
    int t1 = 0, t2 = 1;
    if (active) baseline_to_tiles(bl, p.ntiles, t1, t2);
    const int u1 = active ? p.tile_map[t1] : 0, u2 = active ? p.tile_map[t2] : 0;
    int fr[FCH], col[FCH];
    double ool[FCH];
#pragma unroll
    for (int i = 0; i < FCH; i++) {
        fr[i] = min(f0 + i, p.nf - 1);  // a missing last channel repeats the previous one and is not stored
        ool[i] = p.freqs[fr[i]] / VEL_C;
        col[i] = p.freq_map[fr[i]];
    }
    double um = 0.0, vm = 0.0, wm = 0.0;
    if (active) {
        const UVW q = p.uvws[bl];
        um = q.u, vm = q.v, wm = q.w;
    }

    const int nchunks = (p.nc + CH - 1) / CH;
    if (threadIdx.x == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        fence_barrier_init();
    }
    __syncthreads();

    auto issue = [&](int k) {
        const int st = k & 1;
        const int c0 = k * CH;
        const int n = min(CH, p.nc - c0);
        const uint32_t bytes = n * 32u + FCH * n * 64u + n * 32u;
        mbar_arrive_expect_tx(&bar[st], bytes);
        bulk_g2s(s_lmn[st], p.lmn + c0, n * 32u, &bar[st]);
#pragma unroll
        for (int i = 0; i < FCH; i++) bulk_g2s(s_flux[st][i], p.flux + (size_t)fr[i] * p.nc + c0, n * 64u, &bar[st]);
        bulk_g2s(s_gp[st], p.gp + c0, n * 32u, &bar[st]);
    };
    int issued = 0;
    if (threadIdx.x == 0) {
        fence_proxy_async_smem();
        if (!p.stall) {
            if (nchunks > 0) issue(0), issued = 1;
            if (nchunks > 1) issue(1), issued = 2;
        }
    }
    const uint64_t limit = p.wait_ns ? p.wait_ns : 2000000000ull;

    J2 acc[FCH];
#pragma unroll
    for (int i = 0; i < FCH; i++) acc[i] = jzero();
    bool aborted = false;
    for (int k = 0; k < nchunks; k++) {
        const int st = k & 1;
        const bool ok = mbar_wait_bounded(&bar[st], (k >> 1) & 1, p.err, limit);
        if (__syncthreads_or(!ok)) {
            if (threadIdx.x == 0) drain_two_stage(bar, k, issued);
            aborted = true;
            break;
        }
        const int c0 = k * CH;
        const int n = min(CH, p.nc - c0);
        // G = B S and H = B of every (channel, component, unique tile)
        for (int e = threadIdx.x; e < FCH * CH * nu; e += DT) {
            const int u = e % nu, c = (e / nu) % CH, i = e / (nu * CH);
            if (c >= n) continue;
            const J2 b = ldg_j(p.beam + ((size_t)u * p.n_uniq_freq + col[i]) * p.nc + c0 + c);
            const J2 g = b * load_j(s_flux[st][i][c]);
            float4* rf = s_gh + (size_t)e * 6;
            rf[0] = make_float4((float)g.a.re, (float)g.a.im, (float)g.b.re, (float)g.b.im);
            rf[1] = make_float4((float)g.c.re, (float)g.c.im, (float)g.d.re, (float)g.d.im);
            double2* r = reinterpret_cast<double2*>(rf + 2);
            r[0] = make_double2(b.a.re, b.a.im);
            r[1] = make_double2(b.b.re, b.b.im);
            r[2] = make_double2(b.c.re, b.c.im);
            r[3] = make_double2(b.d.re, b.d.im);
        }
        if (TYPE == 2 && p.sdense)
            for (int e = threadIdx.x; e < n * SDN * SDN; e += DT) s_dense[e] = __ldg(p.sdense + (size_t)c0 * SDN * SDN + e);
        __syncthreads();
        if (active) {
            for (int c = 0; c < n; c++) {
                const double4 g = s_gp[st][c];
                FastTerm<TYPE, FCH> term;
                fast_term<TYPE, FCH>(p, s_lmn[st][c], g, um, vm, wm, c0 + c, t1, t2, ool,
                                     TYPE == 2 && p.sdense ? s_dense + c * SDN * SDN : nullptr, term);
#pragma unroll
                for (int i = 0; i < FCH; i++) {
                    float zr, zi;
                    fast_z<TYPE, FCH>(p, term, i, ool[i], c0 + c, g, p.sdense != nullptr, zr, zi);
                    const float4* rg = s_gh + ((size_t)(i * CH + c) * nu + u1) * 6;
                    const double2* rh = reinterpret_cast<const double2*>(s_gh + ((size_t)(i * CH + c) * nu + u2) * 6 + 2);
                    const float4 g0 = rg[0], g1 = rg[1];
                    const cplx za = {(double)(zr * g0.x - zi * g0.y), (double)fmaf(zr, g0.y, zi * g0.x)};
                    const cplx zb = {(double)(zr * g0.z - zi * g0.w), (double)fmaf(zr, g0.w, zi * g0.z)};
                    const cplx zc = {(double)(zr * g1.x - zi * g1.y), (double)fmaf(zr, g1.y, zi * g1.x)};
                    const cplx zd = {(double)(zr * g1.z - zi * g1.w), (double)fmaf(zr, g1.w, zi * g1.z)};
                    const double2 ha = rh[0], hb = rh[1], hc = rh[2], hd = rh[3];
                    J2& m = acc[i];
                    m.a.re = fma(za.re, ha.x, fma(za.im, ha.y, fma(zb.re, hb.x, fma(zb.im, hb.y, m.a.re))));
                    m.a.im = fma(za.im, ha.x, fma(-za.re, ha.y, fma(zb.im, hb.x, fma(-zb.re, hb.y, m.a.im))));
                    m.b.re = fma(za.re, hc.x, fma(za.im, hc.y, fma(zb.re, hd.x, fma(zb.im, hd.y, m.b.re))));
                    m.b.im = fma(za.im, hc.x, fma(-za.re, hc.y, fma(zb.im, hd.x, fma(-zb.re, hd.y, m.b.im))));
                    m.c.re = fma(zc.re, ha.x, fma(zc.im, ha.y, fma(zd.re, hb.x, fma(zd.im, hb.y, m.c.re))));
                    m.c.im = fma(zc.im, ha.x, fma(-zc.re, ha.y, fma(zd.im, hb.x, fma(-zd.re, hb.y, m.c.im))));
                    m.d.re = fma(zc.re, hc.x, fma(zc.im, hc.y, fma(zd.re, hd.x, fma(zd.im, hd.y, m.d.re))));
                    m.d.im = fma(zc.im, hc.x, fma(-zc.re, hc.y, fma(zd.im, hd.x, fma(-zd.re, hd.y, m.d.im))));
                }
            }
        }
        __syncthreads();
        if (threadIdx.x == 0 && k + 2 < nchunks) {
            fence_proxy_async_smem();
            issue(k + 2);
            issued = k + 3;
        }
    }

    if (!active || aborted) return;
#pragma unroll
    for (int i = 0; i < FCH; i++) {
        if (f0 + i >= p.nf) break;
        add_vis<OUT64>(p.vis, (size_t)(f0 + i) * p.nbl + bl, acc[i]);
    }
}

template <int TYPE, bool OUT64>
static cudaError_t launch_fast_tile(const DirectParams& p, cudaStream_t s) {
    const size_t smem = fast_tile_smem_bytes(p.n_uniq_tile);
    // the opt-in above 48 KB of dynamic shared memory, once per device
    static std::atomic<bool> attr[64];
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    if (!attr[dev].load(std::memory_order_relaxed)) {
        e = cudaFuncSetAttribute(fast_tile_kernel<TYPE, OUT64>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)fast_tile_smem_bytes(FT_MAX_NU));
        if (e != cudaSuccess) return e;
        attr[dev].store(true, std::memory_order_relaxed);
    }
    const dim3 grid((p.nbl + DT - 1) / DT, (p.nf + FastTileShape<TYPE>::FCH - 1) / FastTileShape<TYPE>::FCH);
    fast_tile_kernel<TYPE, OUT64><<<grid, DT, smem, s>>>(p);
    return cudaSuccess;
}

template <int TYPE>
static cudaError_t launch_t(bool tile_beam, bool out64, bool fast, const DirectParams& p, cudaStream_t s) {
    dim3 grid((p.nbl + DT - 1) / DT, p.nf);
    if (tile_beam && fast && TYPE != 0) {
        const cudaError_t e = out64 ? launch_fast_tile<TYPE == 0 ? 1 : TYPE, true>(p, s)
                                    : launch_fast_tile<TYPE == 0 ? 1 : TYPE, false>(p, s);
        if (e != cudaSuccess) return e;
    } else if (tile_beam) {
        if (out64)
            direct_kernel<TYPE, true, true, false><<<grid, DT, 0, s>>>(p);
        else
            direct_kernel<TYPE, true, false, false><<<grid, DT, 0, s>>>(p);
    } else if (fast && TYPE != 0) {
        constexpr int FCH = FastShape<TYPE == 0 ? 1 : TYPE>::FCH;
        const dim3 fgrid((p.nbl + DT - 1) / DT, (p.nf + FCH - 1) / FCH);
        if (out64)
            fast_kernel<TYPE == 0 ? 1 : TYPE, true><<<fgrid, DT, 0, s>>>(p);
        else
            fast_kernel<TYPE == 0 ? 1 : TYPE, false><<<fgrid, DT, 0, s>>>(p);
    } else if (fast) {
        if (out64)
            direct_kernel<TYPE, false, true, true><<<grid, DT, 0, s>>>(p);
        else
            direct_kernel<TYPE, false, false, true><<<grid, DT, 0, s>>>(p);
    } else {
        if (out64)
            direct_kernel<TYPE, false, true, false><<<grid, DT, 0, s>>>(p);
        else
            direct_kernel<TYPE, false, false, false><<<grid, DT, 0, s>>>(p);
    }
    count_launches(1);
    return cudaGetLastError();
}

// hdc_test_stall_next_predict: wait limit [ns] for the next direct launch,
// which then issues no table copies (0: off).
static std::atomic<unsigned long long> g_stall_next_ns{0};

const char* kernel_error_string(int word) {
    if (word & KERR_TIMEOUT)
        return "a predict kernel gave up waiting for its staged component tables (bounded wait ran out); "
               "the visibilities of the affected CTAs were left unchanged";
    if (word & KERR_INDEX) return "a kernel found an index outside its table (shapelet order or beam map)";
    if (word) return "a kernel reported an unknown error";
    return NULL;
}

int kernel_error_status(int word) {
    if (word & KERR_TIMEOUT) return HDC_ERR_TIMEOUT;
    if (word) return HDC_ERR_ARG;
    return HDC_OK;
}

cudaError_t launch_direct(int ty, bool tile_beam, bool out64, const DirectParams& p_in, cudaStream_t s, bool fast) {
    DirectParams p = p_in;
    if (p.nc <= 0 || p.nbl <= 0 || p.nf <= 0) return cudaSuccess;
    if (g_stall_next_ns.load(std::memory_order_relaxed)) {
        const unsigned long long ns = g_stall_next_ns.exchange(0);
        if (ns) {
            p.stall = 1;
            p.wait_ns = ns;
        }
    }
    // the FP32 form needs per-tile shapelet UVs and the FP32 basis table, and
    // with per-tile beams a unique-tile count it can stage (not the points,
    // whose chosen form is the tensor kernel)
    fast = fast && (ty != 2 || (p.suv_tile && !p.suv_bl && p.sbf32)) &&
           (!tile_beam || (ty != 0 && p.n_uniq_tile > 0 && p.n_uniq_tile <= FT_MAX_NU && !p.unflagged_map));
    if (fast && ty == 2 && p.sdense && !p.sbfp) return cudaErrorInvalidValue;
    if (ty == 0) return launch_t<0>(tile_beam, out64, fast, p, s);
    if (ty == 1) return launch_t<1>(tile_beam, out64, fast, p, s);
    return launch_t<2>(tile_beam, out64, fast, p, s);
}

// Auto-correlations: one thread per (tile, channel) (gpu/model.cu:368-485;
// the envelope is 1 for every component type).
__global__ void autos_kernel(const AutosParams p) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= p.ntiles * p.nf) return;
    const int f = i % p.nf;
    const int tile = i / p.nf;
    J2 acc = jzero();
    const JonesF64* bj = nullptr;
    if (p.beam) {
        const int ut = p.unflagged_map ? p.unflagged_map[tile] : tile;
        bj = p.beam + (size_t)p.nc_total * ((size_t)p.n_uniq_freq * p.tile_map[ut] + p.freq_map[f]);
    }
    for (int c = 0; c < p.nc_total; c++) {
        J2 sj = ldg_j(p.flux + (size_t)f * p.nc_total + c);
        if (bj) {
            const J2 b = ldg_j(bj + c);
            sj = (b * sj) * herm(b);
        }
        acc = acc + sj;
    }
    JonesF32* o = p.vis + (size_t)f * p.ntiles + tile;
    o->j00_re += (float)acc.a.re;
    o->j00_im += (float)acc.a.im;
    o->j01_re += (float)acc.b.re;
    o->j01_im += (float)acc.b.im;
    o->j10_re += (float)acc.c.re;
    o->j10_im += (float)acc.c.im;
    o->j11_re += (float)acc.d.re;
    o->j11_im += (float)acc.d.im;
}

cudaError_t launch_autos(const AutosParams& p, cudaStream_t s) {
    if (p.ntiles * p.nf == 0 || p.nc_total == 0) return cudaSuccess;
    const int n = p.ntiles * p.nf;
    autos_kernel<<<(n + 255) / 256, 256, 0, s>>>(p);
    count_launches(1);
    return cudaGetLastError();
}

__global__ void mask_pols_kernel(JonesF32* vis, size_t n, int pols) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    JonesF32 j = vis[i];
    const bool k0 = pols == 1 || pols == 3 || pols == 4;
    const bool k1 = pols == 4;
    const bool k3 = pols == 2 || pols == 3 || pols == 4;
    if (!k0) j.j00_re = j.j00_im = 0.0f;
    if (!k1) j.j01_re = j.j01_im = 0.0f;
    j.j10_re = j.j10_im = 0.0f;
    if (!k3) j.j11_re = j.j11_im = 0.0f;
    vis[i] = j;
}

cudaError_t launch_mask_pols(JonesF32* vis, size_t n, int pols, cudaStream_t s) {
    if (pols == 0 || n == 0) return cudaSuccess;
    mask_pols_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(vis, n, pols);
    count_launches(1);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Drop-in layer: the reference's component tables -> per-type direct tables.
// ---------------------------------------------------------------------------

// One flux-model group of a component type as the reference passes it.
struct GroupIn {
    int n;
    const LmnRime* lmns;
    const JonesF64* fds;  // PL/CPL: [n] at 150 MHz; list: [nf][n]
    const double* sis;
    const double* qs;
    const GaussianParams* gps;
    const ShapeletUV* suvs;  // [nbl][n]
    const ShapeletCoeff* coeffs;
    const int* num_coeffs;
};

struct PrepIn {
    GroupIn g[3];  // power law, curved power law, list
    int nc, nf, nbl, type;
    const double* freqs;
    double4* lmn;
    JonesF64* flux;   // [nf][flux_ld]
    int flux_ld;
    double4* gp;
    ShapeletUV* suv;  // [nbl][nc]
};

// Per (channel, component): instrumental flux at the channel as the reference
// GPU kernels extrapolate it from 150 MHz (gpu/model.cu:16-28), plus the
// component's LMN in turns and envelope parameters.
__global__ void dropin_prep_kernel(const PrepIn in) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const int f = blockIdx.y;
    if (c >= in.nc) return;
    int grp = 0, k = c;
    if (k >= in.g[0].n) {
        k -= in.g[0].n;
        grp = 1;
        if (k >= in.g[1].n) {
            k -= in.g[1].n;
            grp = 2;
        }
    }
    const GroupIn& g = in.g[grp];
    const double freq = in.freqs[f];
    JonesF64 s;
    if (grp == 2) {
        s = g.fds[(size_t)f * g.n + k];
    } else {
        const double ratio = pow(freq / POWER_LAW_FD_REF_FREQ, g.sis[k]);
        J2 j = load_j(g.fds[k]) * ratio;
        if (grp == 1) {
            const double lt = log(freq / POWER_LAW_FD_REF_FREQ);
            j = j * exp(g.qs[k] * lt * lt);
        }
        s = store_j(j);
    }
    in.flux[(size_t)f * in.flux_ld + c] = s;
    if (f == 0) {
        const LmnRime l = g.lmns[k];
        in.lmn[c] = make_double4(l.l * INV_TAU, l.m * INV_TAU, l.n * INV_TAU, 0.0);
        if (in.type >= 1) {
            const GaussianParams gp = g.gps[k];
            double sp, cp;
            sincos(gp.pa, &sp, &cp);
            if (in.type == 1)
                in.gp[c] = make_double4(GAUSSIAN_EXP_CONST * (gp.maj * gp.maj), GAUSSIAN_EXP_CONST * (gp.min * gp.min), sp, cp);
            else
                in.gp[c] = make_double4(gp.maj * SHAPELET_CONST, -gp.min * SHAPELET_CONST, sp, cp);
        }
    }
}

__global__ void dropin_suv_kernel(const PrepIn in) {
    // gather the three groups' [nbl][n_g] shapelet UVs into [nbl][nc]
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)in.nbl * in.nc) return;
    const int bl = (int)(i / in.nc);
    int k = (int)(i % in.nc);
    int grp = 0;
    if (k >= in.g[0].n) {
        k -= in.g[0].n;
        grp = 1;
        if (k >= in.g[1].n) {
            k -= in.g[1].n;
            grp = 2;
        }
    }
    in.suv[i] = in.g[grp].suvs[(size_t)bl * in.g[grp].n + k];
}

// Exclusive scan of per-component coefficient counts (single thread; the
// component counts here are small) and repacking of the three groups'
// coefficient arrays into one table.
// Coefficients whose orders fall outside the basis table (n >= SBF_N) would
// index past it; they are replaced by a zero coefficient and flagged in *err
// (KERR_INDEX) so that the entry point can return an error.
__global__ void dropin_coeff_kernel(const PrepIn in, int* start, int* count, ShapeletCoeff* out, int* err) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    int off = 0, c = 0;
    for (int grp = 0; grp < 3; grp++) {
        int goff = 0;
        for (int k = 0; k < in.g[grp].n; k++, c++) {
            const int nk = in.g[grp].num_coeffs[k];
            start[c] = off;
            count[c] = nk;
            for (int i = 0; i < nk; i++) {
                ShapeletCoeff co = in.g[grp].coeffs[goff + i];
                if (co.n1 >= SBF_N || co.n2 >= SBF_N) {
                    *err |= KERR_INDEX;
                    co.value = 0.0;
                    co.n1 = 0;
                    co.n2 = 0;
                }
                out[off + i] = co;
            }
            off += nk;
            goff += nk;
        }
    }
}

static size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

// Sum of per-component coefficient counts needs a device read; the drop-in
// entry point copies the counts back (small) to size the repacked table.
static const char* dropin_model(int type, const GroupIn g[3], const Addresses* a, const UVW* d_uvws,
                                const JonesF64* d_beam_jones, void* d_vis_fb, bool out64) {
    const int nc = g[0].n + g[1].n + g[2].n;
    if (nc == 0) return NULL;
    const int nf = a->num_freqs, nbl = a->num_baselines;
    int total_coeffs = 0;
    if (type == 2) {
        for (int grp = 0; grp < 3; grp++) {
            if (g[grp].n == 0) continue;
            int* h = (int*)malloc(sizeof(int) * g[grp].n);
            if (!h) return "host allocation failed";
            cudaError_t e = cudaMemcpy(h, g[grp].num_coeffs, sizeof(int) * g[grp].n, cudaMemcpyDeviceToHost);
            if (e != cudaSuccess) {
                free(h);
                set_error("model_shapelets: %s", cudaGetErrorString(e));
                return cudaGetErrorString(e);
            }
            for (int k = 0; k < g[grp].n; k++) total_coeffs += h[k];
            free(h);
        }
    }
    size_t off_lmn = 0;
    size_t off_flux = align256(off_lmn + sizeof(double4) * nc);
    size_t off_gp = align256(off_flux + sizeof(JonesF64) * (size_t)nf * nc);
    size_t off_suv = align256(off_gp + sizeof(double4) * nc);
    size_t off_cs = align256(off_suv + (type == 2 ? sizeof(ShapeletUV) * (size_t)nbl * nc : 0));
    size_t off_cc = align256(off_cs + sizeof(int) * nc);
    size_t off_co = align256(off_cc + sizeof(int) * nc);
    size_t total = align256(off_co + sizeof(ShapeletCoeff) * (size_t)(total_coeffs + 1));
    char* ws = (char*)device_scratch(total);
    if (!ws) return "out of device memory";
    int* errw = dropin_error_word();
    if (!errw) return "device error word unavailable";

    PrepIn in;
    for (int i = 0; i < 3; i++) in.g[i] = g[i];
    in.nc = nc;
    in.nf = nf;
    in.nbl = nbl;
    in.type = type;
    in.freqs = a->d_freqs;
    in.lmn = (double4*)(ws + off_lmn);
    in.flux = (JonesF64*)(ws + off_flux);
    in.flux_ld = nc;
    in.gp = (double4*)(ws + off_gp);
    in.suv = (ShapeletUV*)(ws + off_suv);
    dim3 pg((nc + 127) / 128, nf);
    dropin_prep_kernel<<<pg, 128>>>(in);
    count_launches(1);
    HDC_CUDA_RET_STR(cudaGetLastError());
    int* cstart = (int*)(ws + off_cs);
    int* ccount = (int*)(ws + off_cc);
    ShapeletCoeff* co = (ShapeletCoeff*)(ws + off_co);
    if (type == 2) {
        size_t n = (size_t)nbl * nc;
        dropin_suv_kernel<<<(unsigned)((n + 255) / 256), 256>>>(in);
        count_launches(1);
        HDC_CUDA_RET_STR(cudaGetLastError());
        dropin_coeff_kernel<<<1, 1>>>(in, cstart, ccount, co, errw);
        count_launches(1);
        HDC_CUDA_RET_STR(cudaGetLastError());
        int h = 0;
        HDC_CUDA_RET_STR(cudaMemcpy(&h, errw, sizeof(int), cudaMemcpyDeviceToHost));
        if (h & KERR_INDEX) {
            cudaMemset(errw, 0, sizeof(int));
            set_error("model_shapelets: a shapelet coefficient order is outside 0..%d", SBF_N - 1);
            return "model_shapelets: shapelet coefficient order outside the basis table";
        }
    }
    DirectParams p = {};
    p.nbl = nbl;
    p.nf = nf;
    p.ntiles = (int)((1.0 + sqrt(1.0 + 8.0 * nbl)) / 2.0 + 0.5);
    p.nc = nc;
    p.freqs = a->d_freqs;
    p.uvws = d_uvws;
    p.lmn = in.lmn;
    p.flux = in.flux;
    p.gp = in.gp;
    p.beam = d_beam_jones;
    p.tile_map = a->d_tile_map;
    p.unflagged_map = a->d_tile_index_to_unflagged_tile_index_map;
    p.freq_map = a->d_freq_map;
    p.n_uniq_freq = a->num_unique_beam_freqs;
    p.sbf = a->d_shapelet_basis_values ? a->d_shapelet_basis_values : device_shapelet_basis();
    p.coeffs = co;
    p.coeff_start = cstart;
    p.coeff_count = ccount;
    p.suv_bl = type == 2 ? in.suv : nullptr;
    p.suv_tile = nullptr;
    p.vis = d_vis_fb;
    p.err = errw;
    const bool tile_beam = d_beam_jones != nullptr;
    HDC_CUDA_RET_STR(launch_direct(type, tile_beam, out64, p, 0));
    // a bounded wait that ran out leaves part of d_vis_fb without this call's
    // sum: report it (and clear the word) instead of returning success
    return take_word_sync(errw, type == 0 ? "model_points" : type == 1 ? "model_gaussians" : "model_shapelets");
}

// Bytes of workspace the point-source drop-in path needs for nc components
// and nf channels (derived LMN and per-channel flux tables).
size_t points_workspace_bytes(int nc, int nf) {
    size_t off_flux = align256(sizeof(double4) * (size_t)nc);
    size_t off_gp = align256(off_flux + sizeof(JonesF64) * (size_t)nf * nc);
    return align256(off_gp + sizeof(double4) * (size_t)nc);
}

// The point-source drop-in path over a workspace and kernel error word the
// caller provides.  Allocates nothing and runs on the legacy default stream.
const char* points_with_workspace(const Points* comps, const Addresses* a, const UVW* d_uvws,
                                  const JonesF64* d_beam_jones, JonesF32* d_vis_fb, void* ws, size_t ws_bytes,
                                  int* err_word) {
    GroupIn g[3] = {};
    g[0] = GroupIn{comps->num_power_laws, comps->power_law_lmns, comps->power_law_fds, comps->power_law_sis};
    g[1] = GroupIn{comps->num_curved_power_laws, comps->curved_power_law_lmns, comps->curved_power_law_fds,
                   comps->curved_power_law_sis, comps->curved_power_law_qs};
    g[2] = GroupIn{comps->num_lists, comps->list_lmns, comps->list_fds};
    const int nc = g[0].n + g[1].n + g[2].n;
    if (nc == 0) return NULL;
    const int nf = a->num_freqs, nbl = a->num_baselines;
    if (points_workspace_bytes(nc, nf) > ws_bytes) return "workspace too small for this many channels x components";
    char* w = (char*)ws;
    PrepIn in = {};
    for (int i = 0; i < 3; i++) in.g[i] = g[i];
    in.nc = nc;
    in.nf = nf;
    in.nbl = nbl;
    in.type = 0;
    in.freqs = a->d_freqs;
    in.lmn = (double4*)w;
    in.flux = (JonesF64*)(w + align256(sizeof(double4) * (size_t)nc));
    in.flux_ld = nc;
    in.gp = (double4*)(w + align256(align256(sizeof(double4) * (size_t)nc) + sizeof(JonesF64) * (size_t)nf * nc));
    dim3 pg((nc + 127) / 128, nf);
    dropin_prep_kernel<<<pg, 128>>>(in);
    count_launches(1);
    HDC_CUDA_RET_STR(cudaGetLastError());
    DirectParams p = {};
    p.nbl = nbl;
    p.nf = nf;
    p.ntiles = (int)((1.0 + sqrt(1.0 + 8.0 * nbl)) / 2.0 + 0.5);
    p.nc = nc;
    p.freqs = a->d_freqs;
    p.uvws = d_uvws;
    p.lmn = in.lmn;
    p.flux = in.flux;
    p.gp = in.gp;
    p.beam = d_beam_jones;
    p.tile_map = a->d_tile_map;
    p.unflagged_map = a->d_tile_index_to_unflagged_tile_index_map;
    p.freq_map = a->d_freq_map;
    p.n_uniq_freq = a->num_unique_beam_freqs;
    p.vis = d_vis_fb;
    p.err = err_word;
    HDC_CUDA_RET_STR(launch_direct(0, d_beam_jones != nullptr, false, p, 0));
    return take_word_sync(err_word, "model_points_noalloc");
}

}  // namespace hdc

using namespace hdc;

static void point_groups(const Points* comps, GroupIn g[3]) {
    g[0] = GroupIn{comps->num_power_laws, comps->power_law_lmns, comps->power_law_fds, comps->power_law_sis};
    g[1] = GroupIn{comps->num_curved_power_laws, comps->curved_power_law_lmns, comps->curved_power_law_fds,
                   comps->curved_power_law_sis, comps->curved_power_law_qs};
    g[2] = GroupIn{comps->num_lists, comps->list_lmns, comps->list_fds};
}

extern "C" const char* model_points(const Points* comps, const Addresses* a, const UVW* d_uvws,
                                    const JonesF64* d_beam_jones, JonesF32* d_vis_fb) {
    GroupIn g[3] = {};
    point_groups(comps, g);
    return dropin_model(0, g, a, d_uvws, d_beam_jones, d_vis_fb, false);
}

extern "C" const char* model_points_f64out(const Points* comps, const Addresses* a, const UVW* d_uvws,
                                           const JonesF64* d_beam_jones, JonesF64* d_vis_fb) {
    GroupIn g[3] = {};
    point_groups(comps, g);
    return dropin_model(0, g, a, d_uvws, d_beam_jones, d_vis_fb, true);
}

// W [nf][nc] = B S B^H with the beam row of one unique tile
__global__ void shared_beam_kernel(const JonesF64* S, const JonesF64* beam, int beam_tile, const int* freq_map,
                                   int n_uniq_freq, int nc, int nf, JonesF64* W) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const int f = blockIdx.y;
    if (c >= nc || f >= nf) return;
    const J2 b = load_j(beam[((size_t)beam_tile * n_uniq_freq + freq_map[f]) * nc + c]);
    W[(size_t)f * nc + c] = store_j((b * load_j(S[(size_t)f * nc + c])) * herm(b));
}

extern "C" const char* model_points_tc(const Points* comps, const Addresses* a, const XYZ* d_tile_xyzs,
                                       double lst_rad, RADec phase_centre, const JonesF64* d_beam_jones,
                                       JonesF32* d_vis_fb) {
    GroupIn g[3] = {};
    point_groups(comps, g);
    const int nc = g[0].n + g[1].n + g[2].n;
    if (nc == 0) return NULL;
    const int nf = a->num_freqs, nbl = a->num_baselines;
    const int ntiles = (int)((1.0 + sqrt(1.0 + 8.0 * nbl)) / 2.0 + 0.5);
    if (ntiles * (ntiles - 1) / 2 != nbl || !d_tile_xyzs) return "model_points_tc: invalid arguments";
    // the beam row of every tile: one row for all tiles (a shared beam, the
    // cheaper form: W = B S B^H per component) or per-tile rows (block form)
    int beam_tile = -1, n_uniq_tile = 0;
    std::vector<int> row(ntiles);
    if (d_beam_jones) {
        std::vector<int> um(ntiles), tm;
        if (!a->d_tile_map || !a->d_freq_map) return "model_points_tc: beam maps missing";
        if (a->d_tile_index_to_unflagged_tile_index_map)
            HDC_CUDA_RET_STR(cudaMemcpy(um.data(), a->d_tile_index_to_unflagged_tile_index_map, sizeof(int) * ntiles,
                                        cudaMemcpyDeviceToHost));
        else
            for (int t = 0; t < ntiles; t++) um[t] = t;
        int mx = 0;
        for (int t = 0; t < ntiles; t++) {
            if (um[t] < 0) return "model_points_tc: tile map out of range";
            mx = std::max(mx, um[t]);
        }
        tm.resize(mx + 1);
        HDC_CUDA_RET_STR(cudaMemcpy(tm.data(), a->d_tile_map, sizeof(int) * (mx + 1), cudaMemcpyDeviceToHost));
        bool shared = true;
        for (int t = 0; t < ntiles; t++) {
            row[t] = tm[um[t]];
            if (row[t] < 0) return "model_points_tc: tile map out of range";
            n_uniq_tile = std::max(n_uniq_tile, row[t] + 1);
            shared = shared && row[t] == row[0];
        }
        if (shared) beam_tile = row[0];
    }
    const bool tile_beam = d_beam_jones && beam_tile < 0;
    size_t off_lmn = 0;
    size_t off_flux = align256(off_lmn + sizeof(double4) * nc);
    size_t off_w = align256(off_flux + sizeof(JonesF64) * (size_t)nf * nc);
    size_t off_gp = align256(off_w + (d_beam_jones && !tile_beam ? sizeof(JonesF64) * (size_t)nf * nc : 0));
    size_t off_map = align256(off_gp + sizeof(double4) * nc);
    size_t off_ws = align256(off_map + sizeof(int) * (size_t)ntiles);
    size_t total = align256(off_ws + tensor_workspace_bytes(nf, nbl, ntiles, nc, tile_beam, false, false));
    char* ws = (char*)device_scratch(total);
    if (!ws) return "out of device memory";
    PrepIn in = {};
    for (int i = 0; i < 3; i++) in.g[i] = g[i];
    in.nc = nc;
    in.nf = nf;
    in.nbl = nbl;
    in.type = 0;
    in.freqs = a->d_freqs;
    in.lmn = (double4*)(ws + off_lmn);
    in.flux = (JonesF64*)(ws + off_flux);
    in.flux_ld = nc;
    in.gp = (double4*)(ws + off_gp);
    dim3 pg((nc + 127) / 128, nf);
    dropin_prep_kernel<<<pg, 128>>>(in);
    count_launches(1);
    HDC_CUDA_RET_STR(cudaGetLastError());
    const JonesF64* W = in.flux;
    TensorBeam tb = {};
    if (d_beam_jones && !tile_beam) {
        JonesF64* Wb = (JonesF64*)(ws + off_w);
        shared_beam_kernel<<<pg, 128>>>(in.flux, d_beam_jones, beam_tile, a->d_freq_map, a->num_unique_beam_freqs, nc,
                                        nf, Wb);
        count_launches(1);
        HDC_CUDA_RET_STR(cudaGetLastError());
        W = Wb;
    } else if (tile_beam) {
        int* d_row = (int*)(ws + off_map);
        HDC_CUDA_RET_STR(cudaMemcpy(d_row, row.data(), sizeof(int) * ntiles, cudaMemcpyHostToDevice));
        tb.beam = d_beam_jones;
        tb.tile_map = d_row;
        tb.freq_map = a->d_freq_map;
        tb.n_uniq_tile = n_uniq_tile;
        tb.n_uniq_freq = a->num_unique_beam_freqs;
    }
    int* errw = dropin_error_word();
    if (!errw) return "device error word unavailable";
    const int rc = launch_tensor_points(nf, nbl, ntiles, nc, a->d_freqs, d_tile_xyzs, lst_rad - phase_centre.ra,
                                        phase_centre.dec, in.lmn, W, tile_beam ? &tb : nullptr, d_vis_fb, false,
                                        ws + off_ws, errw, 0, nullptr);
    if (rc) return hdc_last_error();
    return take_word_sync(errw, "model_points_tc");
}

extern "C" const char* model_gaussians(const Gaussians* comps, const Addresses* a, const UVW* d_uvws,
                                       const JonesF64* d_beam_jones, JonesF32* d_vis_fb) {
    GroupIn g[3] = {};
    g[0] = GroupIn{comps->num_power_laws, comps->power_law_lmns, comps->power_law_fds, comps->power_law_sis, nullptr,
                   comps->power_law_gps};
    g[1] = GroupIn{comps->num_curved_power_laws, comps->curved_power_law_lmns, comps->curved_power_law_fds,
                   comps->curved_power_law_sis, comps->curved_power_law_qs, comps->curved_power_law_gps};
    g[2] = GroupIn{comps->num_lists, comps->list_lmns, comps->list_fds, nullptr, nullptr, comps->list_gps};
    return dropin_model(1, g, a, d_uvws, d_beam_jones, d_vis_fb, false);
}

extern "C" const char* model_gaussians_f64out(const Gaussians* comps, const Addresses* a, const UVW* d_uvws,
                                              const JonesF64* d_beam_jones, JonesF64* d_vis_fb) {
    GroupIn g[3] = {};
    g[0] = GroupIn{comps->num_power_laws, comps->power_law_lmns, comps->power_law_fds, comps->power_law_sis, nullptr,
                   comps->power_law_gps};
    g[1] = GroupIn{comps->num_curved_power_laws, comps->curved_power_law_lmns, comps->curved_power_law_fds,
                   comps->curved_power_law_sis, comps->curved_power_law_qs, comps->curved_power_law_gps};
    g[2] = GroupIn{comps->num_lists, comps->list_lmns, comps->list_fds, nullptr, nullptr, comps->list_gps};
    return dropin_model(1, g, a, d_uvws, d_beam_jones, d_vis_fb, true);
}

extern "C" const char* model_shapelets(const Shapelets* comps, const Addresses* a, const UVW* d_uvws,
                                       const JonesF64* d_beam_jones, JonesF32* d_vis_fb) {
    GroupIn g[3] = {};
    g[0] = GroupIn{comps->num_power_laws,           comps->power_law_lmns,          comps->power_law_fds,
                   comps->power_law_sis,            nullptr,                        comps->power_law_gps,
                   comps->power_law_shapelet_uvs,   comps->power_law_shapelet_coeffs, comps->power_law_num_shapelet_coeffs};
    g[1] = GroupIn{comps->num_curved_power_laws,
                   comps->curved_power_law_lmns,
                   comps->curved_power_law_fds,
                   comps->curved_power_law_sis,
                   comps->curved_power_law_qs,
                   comps->curved_power_law_gps,
                   comps->curved_power_law_shapelet_uvs,
                   comps->curved_power_law_shapelet_coeffs,
                   comps->curved_power_law_num_shapelet_coeffs};
    g[2] = GroupIn{comps->num_lists,          comps->list_lmns,           comps->list_fds,
                   nullptr,                   nullptr,                    comps->list_gps,
                   comps->list_shapelet_uvs,  comps->list_shapelet_coeffs, comps->list_num_shapelet_coeffs};
    return dropin_model(2, g, a, d_uvws, d_beam_jones, d_vis_fb, false);
}

extern "C" const char* model_shapelets_f64out(const Shapelets* comps, const Addresses* a, const UVW* d_uvws,
                                              const JonesF64* d_beam_jones, JonesF64* d_vis_fb) {
    GroupIn g[3] = {};
    g[0] = GroupIn{comps->num_power_laws,           comps->power_law_lmns,          comps->power_law_fds,
                   comps->power_law_sis,            nullptr,                        comps->power_law_gps,
                   comps->power_law_shapelet_uvs,   comps->power_law_shapelet_coeffs, comps->power_law_num_shapelet_coeffs};
    g[1] = GroupIn{comps->num_curved_power_laws,
                   comps->curved_power_law_lmns,
                   comps->curved_power_law_fds,
                   comps->curved_power_law_sis,
                   comps->curved_power_law_qs,
                   comps->curved_power_law_gps,
                   comps->curved_power_law_shapelet_uvs,
                   comps->curved_power_law_shapelet_coeffs,
                   comps->curved_power_law_num_shapelet_coeffs};
    g[2] = GroupIn{comps->num_lists,          comps->list_lmns,           comps->list_fds,
                   nullptr,                   nullptr,                    comps->list_gps,
                   comps->list_shapelet_uvs,  comps->list_shapelet_coeffs, comps->list_num_shapelet_coeffs};
    return dropin_model(2, g, a, d_uvws, d_beam_jones, d_vis_fb, true);
}

extern "C" const char* model_autos(int num_tiles, int num_freqs, const double* freqs, const Points* points,
                                   const Gaussians* gaussians, const Shapelets* shapelets, const JonesF64* beam_jones,
                                   const int* tile_map, const int* freq_map, int num_fee_freqs,
                                   const int* tile_index_to_unflagged_tile_index_map, JonesF32* vis_fb) {
    // Build one concatenated flux table over all nine groups, in the
    // reference's direction order (gpu/model.cu:380-470).
    GroupIn gs[9] = {};
    gs[0] = GroupIn{points->num_power_laws, points->power_law_lmns, points->power_law_fds, points->power_law_sis};
    gs[1] = GroupIn{points->num_curved_power_laws, points->curved_power_law_lmns, points->curved_power_law_fds,
                    points->curved_power_law_sis, points->curved_power_law_qs};
    gs[2] = GroupIn{points->num_lists, points->list_lmns, points->list_fds};
    gs[3] = GroupIn{gaussians->num_power_laws, gaussians->power_law_lmns, gaussians->power_law_fds,
                    gaussians->power_law_sis};
    gs[4] = GroupIn{gaussians->num_curved_power_laws, gaussians->curved_power_law_lmns,
                    gaussians->curved_power_law_fds, gaussians->curved_power_law_sis, gaussians->curved_power_law_qs};
    gs[5] = GroupIn{gaussians->num_lists, gaussians->list_lmns, gaussians->list_fds};
    gs[6] = GroupIn{shapelets->num_power_laws, shapelets->power_law_lmns, shapelets->power_law_fds,
                    shapelets->power_law_sis};
    gs[7] = GroupIn{shapelets->num_curved_power_laws, shapelets->curved_power_law_lmns,
                    shapelets->curved_power_law_fds, shapelets->curved_power_law_sis, shapelets->curved_power_law_qs};
    gs[8] = GroupIn{shapelets->num_lists, shapelets->list_lmns, shapelets->list_fds};
    int nc_total = 0;
    for (int i = 0; i < 9; i++) nc_total += gs[i].n;
    if (nc_total == 0) return NULL;
    size_t flux_bytes = align256(sizeof(JonesF64) * (size_t)num_freqs * nc_total);
    size_t lmn_bytes = align256(sizeof(double4) * (size_t)nc_total);
    char* ws = (char*)device_scratch(flux_bytes + 3 * lmn_bytes + 256);
    if (!ws) return "out of device memory";
    JonesF64* flux = (JonesF64*)ws;
    // Prepare each component type's three groups as one table, then copy its
    // columns into the concatenated table.
    int col = 0;
    for (int ty = 0; ty < 3; ty++) {
        PrepIn in = {};
        int nty = 0;
        for (int i = 0; i < 3; i++) {
            in.g[i] = gs[3 * ty + i];
            nty += in.g[i].n;
        }
        if (nty == 0) continue;
        in.nc = nty;
        in.nf = num_freqs;
        in.type = 0;  // envelope parameters are not needed for autos
        in.freqs = freqs;
        in.lmn = (double4*)(ws + flux_bytes);
        in.gp = (double4*)(ws + flux_bytes + lmn_bytes);
        in.flux = flux + col;
        in.flux_ld = nc_total;
        dim3 pg((nty + 127) / 128, num_freqs);
        dropin_prep_kernel<<<pg, 128>>>(in);
        count_launches(1);
        HDC_CUDA_RET_STR(cudaGetLastError());
        col += nty;
    }
    AutosParams p;
    p.ntiles = num_tiles;
    p.nf = num_freqs;
    p.nc_total = nc_total;
    p.flux = flux;
    p.beam = beam_jones;
    p.tile_map = tile_map;
    p.unflagged_map = tile_index_to_unflagged_tile_index_map;
    p.freq_map = freq_map;
    p.n_uniq_freq = num_fee_freqs;
    p.vis = vis_fb;
    HDC_CUDA_RET_STR(launch_autos(p, 0));
    return NULL;
}

extern "C" int hdc_test_stall_next_predict(unsigned long long wait_ns) {
    g_stall_next_ns.store(wait_ns);
    return HDC_OK;
}

extern "C" const char* hdc_kernel_error_string(int word) { return kernel_error_string(word); }
