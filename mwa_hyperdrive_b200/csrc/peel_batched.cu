// Batched peeling: every source's ionospheric fit of a pass from one pass
// over the data (this project's chosen form of peel_gpu,
// params/peel/gpu.rs:25-757).
//
// Source models: a source that is one point component at its own position
// has, in its own frame, the same model on every baseline (phase 1, a beam
// shared by all tiles), so it is kept as one Jones per (timestep, channel);
// any other source's model is materialised at high resolution.
//
// The reference peels sources one after another (Gauss-Seidel): rotate the
// whole high-resolution residual to the source, add the source back, average
// to low resolution, fit (alpha, beta, gain), subtract the re-fitted source,
// move on -- about ten passes over the high-resolution data per source.
// Here a pass fits all sources against the same residual (Jacobi), in the
// phase-centre frame throughout:
//   1. accumulate sweep: for every low-resolution bin and source s,
//        D_s = <w (R rot_s + M_s iono_s(old))>,  Mr_s = <w M_s iono_s(old)>
//      with rot_s = exp(-2 pi i (w_s - w_pc) / lambda) the rotation to the
//      source and <.> the weighted mean over the timeblock and each channel
//      group (the reference's rotate, add_model and vis_average_tfb);
//   2. all sources' iono_loop fits in one launch per iteration
//      (iono_loop_batched_on, the reference's arithmetic);
//   3. apply sweep: R += sum_s conj(rot_s) M_s (iono_s(old) - iono_s(new))
//      (the reference's subtract_iono, rotated back).
// Every phase on a baseline is a difference of per-tile phases (uvw_pq =
// uvw_p - uvw_q), so the rotation and ionospheric phasors come from per-tile
// tables [source][timestep][channel][tile] -- 128 phasors where a baseline
// loop would evaluate 8128 -- and a baseline takes tab[p] conj(tab[q]).
// With one source this is the reference's sequence exactly (up to rounding:
// FP32 products and sums with FP32 phasors after an exact FP64 range
// reduction, as against its f32 intermediates); with several,
// sources
// fitted in the same pass do not see each other's updates until the next
// pass.  The source models M_s (high resolution, source frame) are predicted
// once per timeblock by the modeller and reused by every pass.
//
// The accumulate sweep's CTA shape (low-resolution bins x sources per CTA;
// sources in a CTA share the residual loads through L1) is chosen by timing
// the candidates on the first call for a problem shape (the sweep only
// writes its low-resolution outputs, so trial runs have no side effects).

#include <chrono>
#include <cmath>
#include <map>
#include <memory>
#include <mutex>
#include <tuple>
#include <vector>

#include "modeller.cuh"

namespace hdc {
cudaError_t k_xyzs_to_uvws(const XYZ* xyzs, const double* lmsts, UVW* uvws, RADec pc, int ntiles, int nbl, int nt,
                           cudaStream_t s);
cudaError_t k_weights_average(const float* w, float* lo, int nt, int nbl, int nf, int favg, cudaStream_t s);
size_t iono_batched_scratch_bytes(int nsrc, int nbl, int nf);
const char* iono_loop_batched_on(const JonesF32* d_resid, const float* d_w, const JonesF32* d_model,
                                 JonesF32* d_model_rot, void* d_scratch, IonoConsts* consts, int nsrc, int nbl, int nf,
                                 int niter, const UVW* d_uvws, const double* d_lambdas, double convergence,
                                 cudaStream_t s);

namespace pb {

struct SweepArgs {
    const JonesF32* resid;  // [nt][nf][nbl], phase-centre frame
    const float* w;         // [nt][nf][nbl]
    const JonesF32* models; // [nsrc][nt][nf][nbl], source frames (general sources)
    const JonesF32* ptab;   // [nsrc][nt][nf]: point-at-centre sources' models, or null
    // per-tile phasors [nsrc][nt][nf][ntiles]; a baseline's factor is
    // tab[p] conj(tab[q]) for its tiles p, q (the phases are differences of
    // per-tile phases, since uvw_pq = uvw_p - uvw_q)
    const float2* rot;      // exp(-2 pi i (w_src,p - w_pc,p) / lambda): to the source frame
    const float2* io_old;   // exp(-2 pi i (alpha u_p + beta v_p) lambda) of the old constants
    const float2* ap_old;   // conj(rot) io_old (apply sweep)
    const float2* ap_new;   // conj(rot) io_new (apply sweep)
    const IonoConsts* old;  // [nsrc]
    const IonoConsts* neu;  // [nsrc] (apply sweep)
    JonesF32* d_lo;         // [nsrc][nlo][nbl]
    JonesF32* m_lo;         // [nsrc][nlo][nbl]
    int nt, nf, nbl, ntiles, nsrc, favg;
};

// exp(i arg) as (cos, sin): the argument (radians) in FP64, reduced exactly
// in quarter turns, then the FP32 quarter-turn polynomials (< 1 ulp of FP32;
// the residual is stored in FP32, so a per-term phasor error of ~1e-7 is at
// its rounding level)
__device__ __forceinline__ float2 phase_f(double arg) {
    float sn, cs;
    phasor_quarter_f32(arg * 0.63661977236758134308, sn, cs);  // 2 / pi
    return make_float2(cs, sn);
}

__device__ __forceinline__ float2 cmulf(float2 a, float2 b) {
    return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
// a conj(b)
__device__ __forceinline__ float2 cmulcf(float2 a, float2 b) {
    return make_float2(fmaf(a.x, b.x, a.y * b.y), fmaf(a.y, b.x, -a.x * b.y));
}

// per-tile UVWs [frame][t][tile] in the frames of the sources (0 .. ns - 1)
// and the phase centre (ns), as xyzs_to_uvws computes them for baselines
__global__ void tile_uvw_kernel(const XYZ* __restrict__ xyz, const double* __restrict__ lmsts,
                                const double2* __restrict__ radec, int nframes, int nt, int ntiles, UVW* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nframes * nt * ntiles) return;
    const int p = i % ntiles, t = (i / ntiles) % nt, fr = i / (ntiles * nt);
    const XYZ a = xyz[(size_t)t * ntiles + p];
    double s_ha, c_ha, s_dec, c_dec;
    sincos(radec[fr].y, &s_dec, &c_dec);
    sincos(lmsts[t] - radec[fr].x, &s_ha, &c_ha);
    out[i] = UVW{s_ha * a.x + c_ha * a.y, -s_dec * c_ha * a.x + s_dec * s_ha * a.y + c_dec * a.z,
                 c_dec * c_ha * a.x - c_dec * s_ha * a.y + s_dec * a.z};
}

// rot[s][t][f][p] = exp(-2 pi i (w_s,p - w_pc,p) / lambda_f)
__global__ void rot_table_kernel(const UVW* __restrict__ tuvw, const double* __restrict__ inv_lam, int ns, int nt,
                                 int nf, int ntiles, float2* __restrict__ rot) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)ns * nt * nf * ntiles) return;
    const int p = (int)(i % ntiles), f = (int)((i / ntiles) % nf), t = (int)((i / ((size_t)ntiles * nf)) % nt);
    const int src = (int)(i / ((size_t)ntiles * nf * nt));
    const double dw = tuvw[((size_t)src * nt + t) * ntiles + p].w - tuvw[((size_t)ns * nt + t) * ntiles + p].w;
    rot[i] = phase_f(-TAU * dw * inv_lam[f]);
}

// out[s][t][f][p] = [conj(rot) x] exp(-2 pi i (alpha u_s,p + beta v_s,p) lambda_f),
// the ionospheric phase exactly 1 when alpha = beta = 0 (as add_model skips it)
__global__ void iono_table_kernel(const UVW* __restrict__ tuvw, const double* __restrict__ lam,
                                  const IonoConsts* __restrict__ k, const float2* __restrict__ rot, int ns, int nt,
                                  int nf, int ntiles, float2* __restrict__ out) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)ns * nt * nf * ntiles) return;
    const int p = (int)(i % ntiles), f = (int)((i / ntiles) % nf), t = (int)((i / ((size_t)ntiles * nf)) % nt);
    const int src = (int)(i / ((size_t)ntiles * nf * nt));
    const IonoConsts c = k[src];
    float2 v = make_float2(1.f, 0.f);
    if (c.alpha != 0.0 || c.beta != 0.0) {
        const UVW q = tuvw[((size_t)src * nt + t) * ntiles + p];
        v = phase_f(-TAU * (q.u * c.alpha + q.v * c.beta) * lam[f]);
    }
    out[i] = rot ? cmulcf(v, rot[i]) : v;
}

// a Jones matrix as four complex FP32 numbers
struct JF {
    float2 v[4];
};
__device__ __forceinline__ JF load_jf(const JonesF32& j) {
    const float4* p = reinterpret_cast<const float4*>(&j);
    const float4 a = p[0], b = p[1];
    return JF{{make_float2(a.x, a.y), make_float2(a.z, a.w), make_float2(b.x, b.y), make_float2(b.z, b.w)}};
}

__device__ __forceinline__ JonesF32 to_f32(const J2& v) {
    return JonesF32{(float)v.a.re, (float)v.a.im, (float)v.b.re, (float)v.b.im,
                    (float)v.c.re, (float)v.c.im, (float)v.d.re, (float)v.d.im};
}

// blockDim (BX, SY): x = low-resolution bins, y = sources of this CTA's chunk
// Grid: one dimension, source groups fastest -- the CTAs of all source
// groups of a bin block run close together, so each residual tile comes
// from DRAM once and from L2 for the other sources.  Products are formed and
// summed in FP32 (the data are FP32; a bin sums nt x favg = 128 samples,
// ~1e-7 relative rounding), at 64 registers so that 4 CTAs share an SM.
template <int BX, int SY>
__global__ void __launch_bounds__(BX* SY, 4) accumulate_kernel(const SweepArgs A) {
    const int nlo = A.nf / A.favg;
    const int ngrp = (A.nsrc + SY - 1) / SY;
    const int bin = (int)(blockIdx.x / ngrp) * BX + threadIdx.x;
    const int src = (int)(blockIdx.x % ngrp) * SY + threadIdx.y;
    if (bin >= nlo * A.nbl || src >= A.nsrc) return;
    const int bl = bin % A.nbl, flo = bin / A.nbl;
    int tp, tq;
    baseline_to_tiles(bl, A.ntiles, tp, tq);
    const float g = (float)A.old[src].gain;
    const size_t nvis = (size_t)A.nt * A.nf * A.nbl;
    const JonesF32* M = A.ptab ? nullptr : A.models + (size_t)src * nvis;
    float2 sd[4] = {}, sm[4] = {};
    float sw = 0.f;
    for (int t = 0; t < A.nt; t++) {
        for (int fc = flo * A.favg; fc < flo * A.favg + A.favg; fc++) {
            const size_t i = ((size_t)t * A.nf + fc) * A.nbl + bl;
            const float wt = A.w[i];
            const size_t tb = (((size_t)src * A.nt + t) * A.nf + fc) * A.ntiles;
            const float2 rot = cmulcf(A.rot[tb + tp], A.rot[tb + tq]);
            const float2 io1 = cmulcf(A.io_old[tb + tp], A.io_old[tb + tq]);
            const float2 io = make_float2(io1.x * g, io1.y * g);
            const JF mj = load_jf(A.ptab ? A.ptab[((size_t)src * A.nt + t) * A.nf + fc] : M[i]);
            const JF r = load_jf(A.resid[i]);
#pragma unroll
            for (int e = 0; e < 4; e++) {
                const float2 m = cmulf(mj.v[e], io);
                const float2 d = cmulf(r.v[e], rot);
                sd[e].x = fmaf(d.x + m.x, wt, sd[e].x);
                sd[e].y = fmaf(d.y + m.y, wt, sd[e].y);
                sm[e].x = fmaf(m.x, wt, sm[e].x);
                sm[e].y = fmaf(m.y, wt, sm[e].y);
            }
            sw += wt;
        }
    }
    const double ws = sw;
    const double acc_d[8] = {sd[0].x, sd[0].y, sd[1].x, sd[1].y, sd[2].x, sd[2].y, sd[3].x, sd[3].y};
    const double acc_m[8] = {sm[0].x, sm[0].y, sm[1].x, sm[1].y, sm[2].x, sm[2].y, sm[3].x, sm[3].y};
    const double inv = 1.0 / (ws > 0.0 ? ws : 1.0);
    const size_t o = ((size_t)src * nlo + flo) * A.nbl + bl;
    A.d_lo[o] = JonesF32{(float)(acc_d[0] * inv), (float)(acc_d[1] * inv), (float)(acc_d[2] * inv),
                         (float)(acc_d[3] * inv), (float)(acc_d[4] * inv), (float)(acc_d[5] * inv),
                         (float)(acc_d[6] * inv), (float)(acc_d[7] * inv)};
    A.m_lo[o] = JonesF32{(float)(acc_m[0] * inv), (float)(acc_m[1] * inv), (float)(acc_m[2] * inv),
                         (float)(acc_m[3] * inv), (float)(acc_m[4] * inv), (float)(acc_m[5] * inv),
                         (float)(acc_m[6] * inv), (float)(acc_m[7] * inv)};
}

// one thread per high-resolution visibility; all sources' updates, summed in
// FP32 and added to the residual once:
//   R += sum_s M_s conj(rot_s) (g_old io_old - g_new io_new)
// with conj(rot) io per baseline = ap[p] conj(ap[q]) from the per-tile tables
__global__ void __launch_bounds__(256) apply_kernel(JonesF32* resid, const SweepArgs A) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const size_t nvis = (size_t)A.nt * A.nf * A.nbl;
    if (i >= nvis) return;
    const int bl = (int)(i % A.nbl);
    const int f = (int)((i / A.nbl) % A.nf);
    const int t = (int)(i / ((size_t)A.nbl * A.nf));
    int tp, tq;
    baseline_to_tiles(bl, A.ntiles, tp, tq);
    float2 dl[4] = {};
#pragma unroll 4  // several sources' table loads in flight
    for (int s = 0; s < A.nsrc; s++) {
        const IonoConsts ko = A.old[s], kn = A.neu[s];
        if (ko.alpha == kn.alpha && ko.beta == kn.beta && ko.gain == kn.gain) continue;
        const size_t tb = (((size_t)s * A.nt + t) * A.nf + f) * A.ntiles;
        const float2 po = cmulcf(A.ap_old[tb + tp], A.ap_old[tb + tq]);
        const float2 pn = cmulcf(A.ap_new[tb + tp], A.ap_new[tb + tq]);
        const float go = (float)ko.gain, gn = (float)kn.gain;
        const float2 bd = make_float2(fmaf(go, po.x, -gn * pn.x), fmaf(go, po.y, -gn * pn.y));
        const JF m = load_jf(A.ptab ? A.ptab[((size_t)s * A.nt + t) * A.nf + f] : A.models[(size_t)s * nvis + i]);
#pragma unroll
        for (int e = 0; e < 4; e++) {
            const float2 c = cmulf(m.v[e], bd);
            dl[e].x += c.x, dl[e].y += c.y;
        }
    }
    float4* p = reinterpret_cast<float4*>(resid + i);
    const float4 a = p[0], b = p[1];
    p[0] = make_float4(a.x + dl[0].x, a.y + dl[0].y, a.z + dl[1].x, a.w + dl[1].y);
    p[1] = make_float4(b.x + dl[2].x, b.y + dl[2].y, b.z + dl[3].x, b.w + dl[3].y);
}

// ptab[(src * nt + t) * nf + f] = W[f][src] as FP32 (W = B S B^H of the
// combined point-source modeller at timestep t)
__global__ void point_table_kernel(const JonesF64* __restrict__ W, int ns, int nf, int nt, int t,
                                   JonesF32* __restrict__ ptab) {
    const int src = blockIdx.x * blockDim.x + threadIdx.x, f = blockIdx.y;
    if (src >= ns) return;
    const JonesF64 w = W[(size_t)f * ns + src];
    ptab[((size_t)src * nt + t) * nf + f] = JonesF32{(float)w.j00_re, (float)w.j00_im, (float)w.j01_re, (float)w.j01_im,
                                                     (float)w.j10_re, (float)w.j10_im, (float)w.j11_re, (float)w.j11_im};
}

// The same sums with the residual staged in shared memory: a CTA takes SB
// consecutive baselines of one low-resolution channel, loads their
// nt x favg samples of residual and weight once (coalesced), and its 256
// threads (SB baselines x 256 / SB source lanes) then run every source of the
// pass over them, so the residual crosses L2 once per pass instead of once per
// source.  Shared memory: samples x SB x 36 bytes.
constexpr int SB = 16;
__global__ void __launch_bounds__(256) accumulate_staged_kernel(const SweepArgs A) {
    extern __shared__ float4 st_smem[];
    const int nlo = A.nf / A.favg, ns_samp = A.nt * A.favg;
    const int nbb = (A.nbl + SB - 1) / SB;
    const int flo = (int)(blockIdx.x / nbb), bl0 = (int)(blockIdx.x % nbb) * SB;
    float4* R = st_smem;                                          // [sample][SB][2]
    float* W = reinterpret_cast<float*>(st_smem + (size_t)ns_samp * SB * 2);  // [sample][SB]
    for (int i = threadIdx.x; i < ns_samp * SB * 2; i += blockDim.x) {
        const int h = i & 1, b = (i >> 1) % SB, k = (i >> 1) / SB;
        const int t = k / A.favg, fc = flo * A.favg + k % A.favg, bl = bl0 + b;
        float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
        if (bl < A.nbl) v = reinterpret_cast<const float4*>(A.resid + ((size_t)t * A.nf + fc) * A.nbl + bl)[h];
        R[i] = v;
    }
    for (int i = threadIdx.x; i < ns_samp * SB; i += blockDim.x) {
        const int b = i % SB, k = i / SB;
        const int t = k / A.favg, fc = flo * A.favg + k % A.favg, bl = bl0 + b;
        W[i] = bl < A.nbl ? A.w[((size_t)t * A.nf + fc) * A.nbl + bl] : 0.f;
    }
    __syncthreads();
    const int b = threadIdx.x % SB, lanes = blockDim.x / SB;
    const int bl = bl0 + b;
    if (bl >= A.nbl) return;
    int tp, tq;
    baseline_to_tiles(bl, A.ntiles, tp, tq);
    const size_t nvis = (size_t)A.nt * A.nf * A.nbl;
    for (int src = threadIdx.x / SB; src < A.nsrc; src += lanes) {
        const float g = (float)A.old[src].gain;
        const JonesF32* M = A.ptab ? nullptr : A.models + (size_t)src * nvis;
        float2 sd[4] = {}, sm[4] = {};
        float sw = 0.f;
        for (int k = 0; k < ns_samp; k++) {
            const int t = k / A.favg, fc = flo * A.favg + k % A.favg;
            const float wt = W[k * SB + b];
            const size_t tb = (((size_t)src * A.nt + t) * A.nf + fc) * A.ntiles;
            const float2 rot = cmulcf(A.rot[tb + tp], A.rot[tb + tq]);
            const float2 io1 = cmulcf(A.io_old[tb + tp], A.io_old[tb + tq]);
            const float2 io = make_float2(io1.x * g, io1.y * g);
            const JF mj = load_jf(A.ptab ? A.ptab[((size_t)src * A.nt + t) * A.nf + fc]
                                         : M[((size_t)t * A.nf + fc) * A.nbl + bl]);
            const float4 r0 = R[(k * SB + b) * 2], r1 = R[(k * SB + b) * 2 + 1];
            const JF r = {{make_float2(r0.x, r0.y), make_float2(r0.z, r0.w), make_float2(r1.x, r1.y),
                           make_float2(r1.z, r1.w)}};
#pragma unroll
            for (int e = 0; e < 4; e++) {
                const float2 m = cmulf(mj.v[e], io);
                const float2 d = cmulf(r.v[e], rot);
                sd[e].x = fmaf(d.x + m.x, wt, sd[e].x);
                sd[e].y = fmaf(d.y + m.y, wt, sd[e].y);
                sm[e].x = fmaf(m.x, wt, sm[e].x);
                sm[e].y = fmaf(m.y, wt, sm[e].y);
            }
            sw += wt;
        }
        const double inv = 1.0 / ((double)sw > 0.0 ? (double)sw : 1.0);
        const size_t o = ((size_t)src * nlo + flo) * A.nbl + bl;
        A.d_lo[o] = JonesF32{(float)(sd[0].x * inv), (float)(sd[0].y * inv), (float)(sd[1].x * inv),
                             (float)(sd[1].y * inv), (float)(sd[2].x * inv), (float)(sd[2].y * inv),
                             (float)(sd[3].x * inv), (float)(sd[3].y * inv)};
        A.m_lo[o] = JonesF32{(float)(sm[0].x * inv), (float)(sm[0].y * inv), (float)(sm[1].x * inv),
                             (float)(sm[1].y * inv), (float)(sm[2].x * inv), (float)(sm[2].y * inv),
                             (float)(sm[3].x * inv), (float)(sm[3].y * inv)};
    }
}

size_t staged_smem_bytes(const SweepArgs& A) { return (size_t)A.nt * A.favg * SB * 36; }

void launch_staged(const SweepArgs& A, cudaStream_t s) {
    const unsigned grid = (unsigned)((A.nf / A.favg) * ((A.nbl + SB - 1) / SB));
    accumulate_staged_kernel<<<grid, 256, staged_smem_bytes(A), s>>>(A);
    count_launches(1);
}

struct Variant {
    int bx, sy;
    void (*launch)(const SweepArgs&, cudaStream_t);
};

template <int BX, int SY>
void launch_acc(const SweepArgs& A, cudaStream_t s) {
    const int nbins = (A.nf / A.favg) * A.nbl;
    const unsigned grid = (unsigned)((nbins + BX - 1) / BX) * (unsigned)((A.nsrc + SY - 1) / SY);
    accumulate_kernel<BX, SY><<<grid, dim3(BX, SY), 0, s>>>(A);
    count_launches(1);
}

// the last variant (bins 0 in the report: one CTA per SB baselines, every
// source) stages the residual; it runs only when its shared memory fits
const Variant kVariants[] = {{256, 1, launch_acc<256, 1>},
                             {128, 2, launch_acc<128, 2>},
                             {64, 4, launch_acc<64, 4>},
                             {32, 8, launch_acc<32, 8>},
                             {SB, 0, launch_staged}};
constexpr int kNumVariants = sizeof(kVariants) / sizeof(kVariants[0]);
constexpr size_t kStagedSmemMax = 200 * 1024;

std::mutex g_tune_mu;
std::map<std::tuple<int, int, int, int, int>, int> g_tuned;  // (nt, nf, nbl, nsrc, favg) -> variant
struct Tuning {
    int bx = 0, sy = 0;
    float ms = 0.f;
} g_last;

// the fastest accumulate variant for this shape (timed once, then cached)
int choose_variant(const SweepArgs& A, cudaStream_t s) {
    const auto key = std::make_tuple(A.nt, A.nf, A.nbl, A.nsrc, A.favg);
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        auto it = g_tuned.find(key);
        if (it != g_tuned.end()) return it->second;
    }
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    int best = 0;
    float best_ms = 1e30f;
    const size_t st_smem = staged_smem_bytes(A);
    const bool staged_ok =
        st_smem <= kStagedSmemMax &&
        cudaFuncSetAttribute(accumulate_staged_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)st_smem) ==
            cudaSuccess;
    cudaGetLastError();
    for (int v = 0; v < kNumVariants; v++) {
        if (kVariants[v].sy == 0 && !staged_ok) continue;
        kVariants[v].launch(A, s);  // warm
        cudaEventRecord(a, s);
        kVariants[v].launch(A, s);
        cudaEventRecord(b, s);
        cudaEventSynchronize(b);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, a, b);
        if (cudaGetLastError() == cudaSuccess && ms < best_ms) {
            best_ms = ms;
            best = v;
        }
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tuned[key] = best;
    g_last = Tuning{kVariants[best].bx, kVariants[best].sy, best_ms};
    return best;
}

// call-scoped device buffers from the library's stream-ordered pool: freed
// blocks stay mapped, so later calls reuse them without new mappings
struct DevBuf {
    void* p = nullptr;
    cudaStream_t s = nullptr;
    bool pooled = false;
    cudaError_t alloc(size_t bytes, cudaStream_t st) {
        s = st;
        pooled = true;
        return pool_malloc_async(&p, bytes, st);
    }
    // large one-off buffers stay outside the pool, which keeps what it holds
    cudaError_t alloc_plain(size_t bytes) { return cudaMalloc(&p, bytes); }
    ~DevBuf() {
        if (p) pooled ? cudaFreeAsync(p, s) : cudaFree(p);
    }
    template <class T>
    T* as() {
        return reinterpret_cast<T*>(p);
    }
};

}  // namespace pb
}  // namespace hdc

using namespace hdc;

#define PB_CK(call)                                                                    \
    do {                                                                               \
        cudaError_t e_ = (call);                                                       \
        if (e_ != cudaSuccess) {                                                       \
            set_error("hdc_peel_timeblock_batched: %s: %s", #call, cudaGetErrorString(e_)); \
            return HDC_ERR_CUDA;                                                       \
        }                                                                              \
    } while (0)

extern "C" int hdc_peel_timeblock_batched(JonesF32* d_resid_tfb, const float* d_weights_tfb, int num_timesteps,
                                          int num_freqs, const double* h_freqs, const XYZ* h_tile_xyzs, int num_tiles,
                                          const double* h_lmsts, double average_lmst, RADec phase_centre,
                                          int num_sources, const HdcSkyModel* h_sources,
                                          const RADec* h_source_positions, IonoConsts* h_iono_consts,
                                          const HdcPeelParams* params, hdcStream_t stream) {
    cudaStream_t s = (cudaStream_t)stream;
    if (!d_resid_tfb || !d_weights_tfb || !h_freqs || !h_tile_xyzs || !h_lmsts || !params || num_tiles < 2 ||
        num_timesteps < 1 || num_freqs < 1 || num_sources < 0 ||
        (num_sources > 0 && (!h_sources || !h_iono_consts || !h_source_positions))) {
        set_error("hdc_peel_timeblock_batched: invalid arguments");
        return HDC_ERR_ARG;
    }
    const int favg = params->freq_average_factor;
    if (favg < 1 || num_freqs % favg != 0) {
        set_error("hdc_peel_timeblock_batched: %d channels are not a multiple of the averaging factor %d", num_freqs,
                  favg);
        return HDC_ERR_ARG;
    }
    if (num_sources == 0) return HDC_OK;
    const int nt = num_timesteps, nf = num_freqs, nbl = num_tiles * (num_tiles - 1) / 2, nlo = nf / favg;
    const int ns = num_sources;
    const size_t nvis = (size_t)nt * nf * nbl;

    std::vector<double> lam(2 * (size_t)nf), lam_lo(nlo);
    for (int f = 0; f < nf; f++) lam[f] = VEL_C / h_freqs[f];
    for (int f = 0; f < nf; f++) lam[nf + f] = 1.0 / lam[f];
    for (int k = 0; k < nlo; k++) {
        double sum = 0.0;
        for (int f = k * favg; f < (k + 1) * favg; f++) sum += h_freqs[f];
        lam_lo[k] = VEL_C / (sum / favg);
    }
    std::vector<XYZ> xyz_t((size_t)nt * num_tiles);
    for (int t = 0; t < nt; t++)
        for (int i = 0; i < num_tiles; i++) xyz_t[(size_t)t * num_tiles + i] = h_tile_xyzs[i];

    // point-at-centre sources keep a (timestep, channel) table; otherwise
    // the models need ns x nvis JonesF32 of device memory
    // (with a beam shared by all tiles, or none: per-tile beams make a
    // point's model depend on the baseline)
    bool points = params->beam_kind == HDC_BEAM_NONE || params->beam_kind == HDC_BEAM_ANALYTIC_DIPOLE;
    for (int i = 0; i < ns && points; i++) {
        const HdcSkyModel& m = h_sources[i];
        points = m.num_components == 1 && m.comp_type[0] == 0 && std::fabs(m.ra[0] - h_source_positions[i].ra) < 1e-12 &&
                 std::fabs(m.dec[0] - h_source_positions[i].dec) < 1e-12;
    }
    size_t free_b = 0, total_b = 0;
    PB_CK(cudaMemGetInfo(&free_b, &total_b));
    const size_t need = points ? sizeof(JonesF32) * (size_t)ns * nt * nf : sizeof(JonesF32) * nvis * (size_t)ns;
    if (need + (size_t)(1u << 30) > free_b) {
        set_error("hdc_peel_timeblock_batched: the %d source models need %zu MB of device memory, %zu MB free", ns,
                  need >> 20, free_b >> 20);
        return HDC_ERR_ALLOC;
    }
    pb::DevBuf b_tuvw, b_radec, b_rot, b_io, b_apo, b_apn;
    pb::DevBuf b_lam, b_lam_lo, b_lmst, b_avg_lmst, b_xyz, b_uv_src, b_uv_lo, b_models, b_dlo, b_mlo, b_mlo_rot,
        b_wlo, b_scr, b_old, b_new;
    PB_CK(b_lam.alloc(sizeof(double) * 2 * nf, s));  // lambda, then 1 / lambda
    PB_CK(b_lam_lo.alloc(sizeof(double) * nlo, s));
    PB_CK(b_lmst.alloc(sizeof(double) * nt, s));
    PB_CK(b_avg_lmst.alloc(sizeof(double), s));
    PB_CK(b_xyz.alloc(sizeof(XYZ) * xyz_t.size(), s));
    if (!points) PB_CK(b_uv_src.alloc(sizeof(UVW) * (size_t)ns * nt * nbl, s));
    const size_t ntab = (size_t)ns * nt * nf * num_tiles;  // per-tile phasor tables
    PB_CK(b_tuvw.alloc(sizeof(UVW) * (size_t)(ns + 1) * nt * num_tiles, s));
    PB_CK(b_radec.alloc(sizeof(double2) * (ns + 1), s));
    PB_CK(b_rot.alloc(sizeof(float2) * ntab, s));
    PB_CK(b_io.alloc(sizeof(float2) * ntab, s));
    PB_CK(b_apo.alloc(sizeof(float2) * ntab, s));
    PB_CK(b_apn.alloc(sizeof(float2) * ntab, s));
    PB_CK(b_uv_lo.alloc(sizeof(UVW) * (size_t)ns * nbl, s));
    PB_CK(points ? b_models.alloc(need, s) : b_models.alloc_plain(need));
    PB_CK(b_dlo.alloc(sizeof(JonesF32) * (size_t)ns * nlo * nbl, s));
    PB_CK(b_mlo.alloc(sizeof(JonesF32) * (size_t)ns * nlo * nbl, s));
    PB_CK(b_mlo_rot.alloc(sizeof(JonesF32) * (size_t)ns * nlo * nbl, s));
    PB_CK(b_wlo.alloc(sizeof(float) * (size_t)nlo * nbl, s));
    PB_CK(b_scr.alloc(iono_batched_scratch_bytes(ns, nbl, nlo), s));
    PB_CK(b_old.alloc(sizeof(IonoConsts) * ns, s));
    PB_CK(b_new.alloc(sizeof(IonoConsts) * ns, s));
    PB_CK(cudaMemcpyAsync(b_lam.p, lam.data(), sizeof(double) * 2 * nf, cudaMemcpyHostToDevice, s));
    PB_CK(cudaMemcpyAsync(b_lam_lo.p, lam_lo.data(), sizeof(double) * nlo, cudaMemcpyHostToDevice, s));
    PB_CK(cudaMemcpyAsync(b_lmst.p, h_lmsts, sizeof(double) * nt, cudaMemcpyHostToDevice, s));
    PB_CK(cudaMemcpyAsync(b_avg_lmst.p, &average_lmst, sizeof(double), cudaMemcpyHostToDevice, s));
    PB_CK(cudaMemcpyAsync(b_xyz.p, xyz_t.data(), sizeof(XYZ) * xyz_t.size(), cudaMemcpyHostToDevice, s));
    PB_CK(k_weights_average(d_weights_tfb, b_wlo.as<float>(), nt, nbl, nf, favg, s));
    // per-tile UVWs in every source's frame and the phase centre's, and the
    // rotation phasors to each source (fixed for the timeblock)
    std::vector<double2> radec(ns + 1);
    for (int i = 0; i < ns; i++) radec[i] = make_double2(h_source_positions[i].ra, h_source_positions[i].dec);
    radec[ns] = make_double2(phase_centre.ra, phase_centre.dec);
    PB_CK(cudaMemcpyAsync(b_radec.p, radec.data(), sizeof(double2) * (ns + 1), cudaMemcpyHostToDevice, s));
    {
        const int n = (ns + 1) * nt * num_tiles;
        pb::tile_uvw_kernel<<<(n + 255) / 256, 256, 0, s>>>(b_xyz.as<XYZ>(), b_lmst.as<double>(),
                                                            b_radec.as<double2>(), ns + 1, nt, num_tiles,
                                                            b_tuvw.as<UVW>());
        pb::rot_table_kernel<<<(unsigned)((ntab + 255) / 256), 256, 0, s>>>(
            b_tuvw.as<UVW>(), b_lam.as<double>() + nf, ns, nt, nf, num_tiles, b_rot.as<float2>());
        count_launches(2);
        PB_CK(cudaGetLastError());
    }
    PB_CK(cudaMemsetAsync(b_models.p, 0, need, s));
    // per source: UVWs in its frame and its high-resolution model (once per
    // timeblock)
    for (int i = 0; i < ns; i++) {
        if (!points)
            PB_CK(k_xyzs_to_uvws(b_xyz.as<XYZ>(), b_lmst.as<double>(), b_uv_src.as<UVW>() + (size_t)i * nt * nbl,
                                 h_source_positions[i], num_tiles, nbl, nt, s));
        PB_CK(k_xyzs_to_uvws(b_xyz.as<XYZ>(), b_avg_lmst.as<double>(), b_uv_lo.as<UVW>() + (size_t)i * nbl,
                             h_source_positions[i], num_tiles, nbl, 1, s));
    }
    if (points) {
        // A single point at its own position has, on every baseline, the model
        // B S B^H (phase 1).  One modeller over all the sources' components
        // (two tiles: the weights do not depend on the baselines or the phase
        // centre) gives B S B^H per (channel, source) after each timestep's
        // geometry; the table kernel stores it as [source][timestep][channel].
        std::vector<int> ctype(ns, HDC_POINT), ftype(ns), fstart(ns), fcount(ns), zero(ns, 0);
        std::vector<double> ra(ns), dec(ns), nil(ns, 0.0), si(ns), q(ns), fds;
        for (int i = 0; i < ns; i++) {
            const HdcSkyModel& m = h_sources[i];
            ra[i] = m.ra[0], dec[i] = m.dec[0], ftype[i] = m.flux_type[0], si[i] = m.si[0], q[i] = m.q[0];
            fstart[i] = (int)(fds.size() / 5);
            fcount[i] = m.fd_count[0];
            fds.insert(fds.end(), m.fds + 5 * (size_t)m.fd_start[0], m.fds + 5 * (size_t)(m.fd_start[0] + m.fd_count[0]));
        }
        const HdcSkyModel all = {ns,          ctype.data(), ra.data(),     dec.data(),   nil.data(), nil.data(),
                                 nil.data(),  ftype.data(), si.data(),     q.data(),     fstart.data(), fcount.data(),
                                 fds.data(),  zero.data(),  zero.data(),   zero.data(),  zero.data(), nil.data()};
        HdcModeller* hm = nullptr;
        int rc = hdc_modeller_new(&all, 0, h_tile_xyzs, 2, h_freqs, num_freqs, phase_centre,
                                  params->array_latitude_rad, params->beam_kind, HDC_PREDICT_DIRECT, &hm);
        if (rc) return rc;
        std::unique_ptr<Modeller> m(reinterpret_cast<Modeller*>(hm));
        for (int t = 0; t < nt; t++) {
            rc = m->geometry(h_lmsts[t], s);
            if (rc) return rc;
            pb::point_table_kernel<<<dim3((ns + 127) / 128, nf), 128, 0, s>>>(m->weights(0), ns, nf, nt, t,
                                                                              b_models.as<JonesF32>());
            count_launches(1);
            PB_CK(cudaGetLastError());
        }
        // the modeller's tables are freed when it goes out of scope: let the
        // table kernels finish reading them first
        PB_CK(cudaStreamSynchronize(s));
    } else {
        for (int i = 0; i < ns; i++) {
            HdcModeller* hm = nullptr;
            int rc = peel_modeller_new(&h_sources[i], h_tile_xyzs, num_tiles, h_freqs, num_freqs,
                                       h_source_positions[i], params, &hm);
            if (rc) return rc;
            std::unique_ptr<Modeller> m(reinterpret_cast<Modeller*>(hm));
            const UVW* uv = b_uv_src.as<UVW>() + (size_t)i * nt * nbl;
            for (int t = 0; t < nt; t++) {
                rc = m->model_uvws(h_lmsts[t], uv + (size_t)t * nbl,
                                   b_models.as<JonesF32>() + (size_t)i * nvis + (size_t)t * nf * nbl, s);
                if (rc) return rc;
            }
        }
    }

    pb::SweepArgs A;
    A.resid = d_resid_tfb;
    A.w = d_weights_tfb;
    A.models = points ? nullptr : b_models.as<JonesF32>();
    A.ptab = points ? b_models.as<JonesF32>() : nullptr;
    A.rot = b_rot.as<float2>();
    A.io_old = b_io.as<float2>();
    A.ap_old = b_apo.as<float2>();
    A.ap_new = b_apn.as<float2>();
    A.old = b_old.as<IonoConsts>();
    A.neu = b_new.as<IonoConsts>();
    A.d_lo = b_dlo.as<JonesF32>();
    A.m_lo = b_mlo.as<JonesF32>();
    A.nt = nt;
    A.nf = nf;
    A.nbl = nbl;
    A.ntiles = num_tiles;
    A.nsrc = ns;
    A.favg = favg;
    std::vector<IonoConsts> fit(ns), next(ns);
    // sources in sub-batches of `batch` in list order: within a sub-batch the
    // fits share the residual (Jacobi); each sub-batch sees the residual the
    // earlier ones left (the reference's Gauss-Seidel order between them)
    const int batch = params->batch_size > 0 ? std::min(params->batch_size, ns) : ns;
    for (int pass = 0; pass < params->num_passes; pass++) {
        for (int b0 = 0; b0 < ns; b0 += batch) {
            const int nb = std::min(batch, ns - b0);
            const size_t tab0 = (size_t)b0 * nt * nf * num_tiles, ntab_b = (size_t)nb * nt * nf * num_tiles;
            pb::SweepArgs B = A;
            B.nsrc = nb;
            B.models = A.models ? A.models + (size_t)b0 * nvis : nullptr;
            B.ptab = A.ptab ? A.ptab + (size_t)b0 * nt * nf : nullptr;
            B.rot = A.rot + tab0;
            B.io_old = A.io_old + tab0;
            B.ap_old = A.ap_old + tab0;
            B.ap_new = A.ap_new + tab0;
            B.old = A.old + b0;
            B.neu = A.neu + b0;
            const UVW* tuvw_b = b_tuvw.as<UVW>() + (size_t)b0 * nt * num_tiles;
            PB_CK(cudaMemcpyAsync(b_old.as<IonoConsts>() + b0, h_iono_consts + b0, sizeof(IonoConsts) * nb,
                                  cudaMemcpyHostToDevice, s));
            const unsigned tgrid = (unsigned)((ntab_b + 255) / 256);
            pb::iono_table_kernel<<<tgrid, 256, 0, s>>>(tuvw_b, b_lam.as<double>(), B.old, nullptr, nb, nt, nf,
                                                        num_tiles, b_io.as<float2>() + tab0);
            count_launches(1);
            PB_CK(cudaGetLastError());
            const int v = pb::choose_variant(B, s);
            pb::kVariants[v].launch(B, s);
            PB_CK(cudaGetLastError());
            for (int i = 0; i < nb; i++) fit[i] = IonoConsts{0.0, 0.0, 1.0};
            const char* err = iono_loop_batched_on(b_dlo.as<JonesF32>(), b_wlo.as<float>(), b_mlo.as<JonesF32>(),
                                                   b_mlo_rot.as<JonesF32>(), b_scr.p, fit.data(), nb, nbl, nlo,
                                                   params->num_loops, b_uv_lo.as<UVW>() + (size_t)b0 * nbl,
                                                   b_lam_lo.as<double>(), params->convergence, s);
            if (err) {
                set_error("hdc_peel_timeblock_batched: %s", err);
                return HDC_ERR_CUDA;
            }
            for (int i = 0; i < nb; i++) {
                const IonoConsts old = h_iono_consts[b0 + i];
                IonoConsts c = {old.alpha + fit[i].alpha, old.beta + fit[i].beta, old.gain * fit[i].gain};
                // the reference's revert rule (gpu.rs:541-627)
                if (std::fabs(c.alpha) > 1e-3 || std::fabs(c.beta) > 1e-3 || c.gain < 0.0 || c.gain > 1.5) c = old;
                next[b0 + i] = c;
            }
            PB_CK(cudaMemcpyAsync(b_new.as<IonoConsts>() + b0, next.data() + b0, sizeof(IonoConsts) * nb,
                                  cudaMemcpyHostToDevice, s));
            pb::iono_table_kernel<<<tgrid, 256, 0, s>>>(tuvw_b, b_lam.as<double>(), B.old, B.rot, nb, nt, nf,
                                                        num_tiles, b_apo.as<float2>() + tab0);
            pb::iono_table_kernel<<<tgrid, 256, 0, s>>>(tuvw_b, b_lam.as<double>(), B.neu, B.rot, nb, nt, nf,
                                                        num_tiles, b_apn.as<float2>() + tab0);
            count_launches(2);
            PB_CK(cudaGetLastError());
            pb::apply_kernel<<<(unsigned)((nvis + 255) / 256), 256, 0, s>>>(d_resid_tfb, B);
            count_launches(1);
            PB_CK(cudaGetLastError());
            PB_CK(cudaStreamSynchronize(s));  // `next` is read by the copy above
            for (int i = 0; i < nb; i++) h_iono_consts[b0 + i] = next[b0 + i];
        }
    }
    PB_CK(cudaStreamSynchronize(s));
    return HDC_OK;
}

extern "C" int hdc_peel_batched_tuning(int* block_bins, int* block_sources, float* ms) {
    std::lock_guard<std::mutex> lk(pb::g_tune_mu);
    if (block_bins) *block_bins = pb::g_last.bx;
    if (block_sources) *block_sources = pb::g_last.sy;
    if (ms) *ms = pb::g_last.ms;
    return HDC_OK;
}
