// Peel kernels for sm_100a: the drop-in set replacing gpu/peel.cu of
// mwa_hyperdrive (xyzs_to_uvws, rotate, average, iono_loop, subtract_iono,
// add_model).
//
// Differences in shape from the reference (results are the same up to
// rounding): every element-wise kernel runs one thread per (time, channel,
// baseline) so that all SMs are busy and accesses are coalesced (the
// reference runs one thread per baseline with time/channel loops, 32 CTAs at
// 8128 baselines); iono_loop runs all its iterations without host round trips
// -- each iteration is one partial-sum kernel plus one single-CTA update
// kernel that keeps the constants in device memory, and the host reads them
// once at the end (the reference copies them back every iteration,
// peel.cu:709).

#include <vector>

#include "common.cuh"

namespace hdc {

constexpr int PT = 256;

__global__ void xyzs_to_uvws_kernel(const XYZ* xyzs, const double* lmsts, UVW* uvws, RADec pc, int ntiles, int nbl,
                                    int nt) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nbl * nt) return;
    const int t = i / nbl, bl = i % nbl;
    int t1, t2;
    baseline_to_tiles(bl, ntiles, t1, t2);
    const XYZ a = xyzs[(size_t)t * ntiles + t1], b = xyzs[(size_t)t * ntiles + t2];
    const double x = a.x - b.x, y = a.y - b.y, z = a.z - b.z;
    double s_ha, c_ha, s_dec, c_dec;
    sincos(pc.dec, &s_dec, &c_dec);
    sincos(lmsts[t] - pc.ra, &s_ha, &c_ha);
    uvws[i] = UVW{s_ha * x + c_ha * y, -s_dec * c_ha * x + s_dec * s_ha * y + c_dec * z,
                  c_dec * c_ha * x - c_dec * s_ha * y + s_dec * z};
}

__device__ __forceinline__ void jf32_mul_f64(JonesF32& j, cplx r) {
    // promote, multiply in f64, demote (peel.cu:78-100)
    const J2 v = load_j32(j) * r;
    j = JonesF32{(float)v.a.re, (float)v.a.im, (float)v.b.re, (float)v.b.im,
                 (float)v.c.re, (float)v.c.im, (float)v.d.re, (float)v.d.im};
}

// JonesF32 * C64 as gpu/common.cuh defines it: the factor is demoted to f32.
__device__ __forceinline__ JonesF32 jf32_mul_c32(const JonesF32& a, cplx r) {
    const float x = (float)r.re, y = (float)r.im;
    return JonesF32{__fsub_rn(__fmul_rn(a.j00_re, x), __fmul_rn(a.j00_im, y)),
                    __fadd_rn(__fmul_rn(a.j00_re, y), __fmul_rn(a.j00_im, x)),
                    __fsub_rn(__fmul_rn(a.j01_re, x), __fmul_rn(a.j01_im, y)),
                    __fadd_rn(__fmul_rn(a.j01_re, y), __fmul_rn(a.j01_im, x)),
                    __fsub_rn(__fmul_rn(a.j10_re, x), __fmul_rn(a.j10_im, y)),
                    __fadd_rn(__fmul_rn(a.j10_re, y), __fmul_rn(a.j10_im, x)),
                    __fsub_rn(__fmul_rn(a.j11_re, x), __fmul_rn(a.j11_im, y)),
                    __fadd_rn(__fmul_rn(a.j11_re, y), __fmul_rn(a.j11_im, x))};
}

__global__ void rotate_kernel(JonesF32* vis, int nt, int nbl, int nf, const UVW* from, const UVW* to,
                              const double* lambdas) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const size_t n = (size_t)nt * nf * nbl;
    if (i >= n) return;
    const int bl = (int)(i % nbl);
    const int f = (int)((i / nbl) % nf);
    const int t = (int)(i / ((size_t)nbl * nf));
    const double arg = -TAU * (to[(size_t)t * nbl + bl].w - from[(size_t)t * nbl + bl].w);
    double s, c;
    sincos(arg / lambdas[f], &s, &c);
    JonesF32 j = vis[i];
    jf32_mul_f64(j, cplx{c, s});
    vis[i] = j;
}

__global__ void average_kernel(const JonesF32* hi, const float* w, JonesF32* lo, int nt, int nbl, int nf, int favg) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int nlo = nf / favg;
    if (i >= nlo * nbl) return;
    const int bl = i % nbl, flo = i / nbl;
    J2 sum = jzero();
    double ws = 0.0;
    for (int t = 0; t < nt; t++)
        for (int fc = flo * favg; fc < flo * favg + favg; fc++) {
            const size_t step = ((size_t)t * nf + fc) * nbl + bl;
            const double wt = w[step];
            sum = sum + load_j32(hi[step]) * wt;
            ws += wt;
        }
    const double d = ws > 0.0 ? ws : 1.0;
    lo[(size_t)flo * nbl + bl] = JonesF32{(float)(sum.a.re / d), (float)(sum.a.im / d), (float)(sum.b.re / d),
                                          (float)(sum.b.im / d),  (float)(sum.c.re / d), (float)(sum.c.im / d),
                                          (float)(sum.d.re / d),  (float)(sum.d.im / d)};
}

// Device state of one iono_loop call, kept at the end of the caller's
// d_iono_fits scratch: the constants, a stop flag and per-(channel, CTA)
// partial sums.
struct IonoDev {
    double alpha, beta, gain;
    int stop;
    int pad;
};

__device__ __forceinline__ double warp_sum(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// One iteration's apply + partial sums (peel.cu:437-486 apply_iono and
// iono_loop_kernel, fused with the baseline reduction of reduce_baselines)
// for one (baseline block, channel) of one source; partials [nblk][7] of
// that channel.
__device__ __forceinline__ void iono_partials_body(const JonesF32* resid, const float* weights,
                                                   const JonesF32* model, JonesF32* model_rot, const IonoDev* st,
                                                   const UVW* uvws, const double* lambdas, int nbl, int f,
                                                   int blk, int nblk, double* partials_f) {
    __shared__ double red[PT / 32][7];
    const int bl = blk * PT + threadIdx.x;
    double v[7] = {0, 0, 0, 0, 0, 0, 0};
    if (bl < nbl) {
        const double u = uvws[bl].u, vv = uvws[bl].v;
        const double arg = -TAU * (u * st->alpha + vv * st->beta);
        double s, c;
        sincos(arg * lambdas[f], &s, &c);
        const size_t step = (size_t)f * nbl + bl;
        const JonesF32 m = jf32_mul_c32(model[step], cplx{c, s} * st->gain);
        model_rot[step] = m;
        const double wt = (double)weights[step];
        const JonesF32 r = resid[step];
        const double ri_re = (double)r.j00_re + (double)r.j11_re;
        const double ri_im = (double)r.j00_im + (double)r.j11_im;
        const double mi_re = (double)m.j00_re + (double)m.j11_re;
        const double mi_im = (double)m.j00_im + (double)m.j11_im;
        const double mr = mi_re * (ri_im - mi_im);
        const double mm = mi_re * mi_re;
        v[0] = wt * mm * u * u;
        v[1] = wt * mm * u * vv;
        v[2] = wt * mm * vv * vv;
        v[3] = wt * mr * u;
        v[4] = wt * mr * vv;
        v[5] = wt * mi_re * ri_re;
        v[6] = wt * mm;
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < 7; k++) {
        const double s = warp_sum(v[k]);
        if (lane == 0) red[warp][k] = s;
    }
    __syncthreads();
    if (threadIdx.x < 7) {
        double s = 0.0;
        for (int w = 0; w < PT / 32; w++) s += red[w][threadIdx.x];
        partials_f[(size_t)blk * 7 + threadIdx.x] = s;
    }
}

// grid (ceil(nbl/PT), nf); partials [nf][gridDim.x][7].
__global__ void __launch_bounds__(PT) iono_partials_kernel(const JonesF32* resid, const float* weights,
                                                           const JonesF32* model, JonesF32* model_rot,
                                                           const IonoDev* st, const UVW* uvws, const double* lambdas,
                                                           int nbl, int nf, double* partials) {
    if (st->stop) return;
    iono_partials_body(resid, weights, model, model_rot, st, uvws, lambdas, nbl, blockIdx.y, blockIdx.x, gridDim.x,
                       partials + (size_t)blockIdx.y * gridDim.x * 7);
}

// The same for a batch of sources: grid (ceil(nbl/PT), nf, nsrc); source s
// reads resid/model/model_rot at s * nf * nbl, weights shared, uvws at
// s * nbl, state st[s], partials [nsrc][nf][nblk][7].
__global__ void __launch_bounds__(PT) iono_partials_batched_kernel(const JonesF32* resid, const float* weights,
                                                                   const JonesF32* model, JonesF32* model_rot,
                                                                   const IonoDev* st, const UVW* uvws,
                                                                   const double* lambdas, int nbl, int nf,
                                                                   double* partials) {
    const int src = blockIdx.z;
    if (st[src].stop) return;
    const size_t off = (size_t)src * nf * nbl;
    iono_partials_body(resid + off, weights, model + off, model_rot + off, st + src, uvws + (size_t)src * nbl,
                       lambdas, nbl, blockIdx.y, blockIdx.x, gridDim.x,
                       partials + ((size_t)src * nf + blockIdx.y) * gridDim.x * 7);
}

// Channel reduction with the lambda scaling and the constants update
// (peel.cu:327-432) for one source; one CTA.
__device__ __forceinline__ void iono_update_body(const double* partials, int nblk, const double* lambdas, int nf,
                                                 IonoDev* st, double convergence) {
    __shared__ double red[PT / 32][7];
    double v[7] = {0, 0, 0, 0, 0, 0, 0};
    for (int f = threadIdx.x; f < nf; f += blockDim.x) {
        double s[7] = {0, 0, 0, 0, 0, 0, 0};
        for (int b = 0; b < nblk; b++)
            for (int k = 0; k < 7; k++) s[k] += partials[((size_t)f * nblk + b) * 7 + k];
        const double lam = lambdas[f], lam2 = lam * lam;
        v[0] += s[0] * lam2;
        v[1] += s[1] * lam2;
        v[2] += s[2] * lam2;
        v[3] += s[3] * -lam;
        v[4] += s[4] * -lam;
        v[5] += s[5];
        v[6] += s[6];
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int k = 0; k < 7; k++) {
        const double s = warp_sum(v[k]);
        if (lane == 0) red[warp][k] = s;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double t[7];
        for (int k = 0; k < 7; k++) {
            t[k] = 0.0;
            for (int w = 0; w < (int)(blockDim.x / 32); w++) t[k] += red[w][k];
        }
        const double a_uu = t[0], a_uv = t[1], a_vv = t[2], A_u = t[3], A_v = t[4], s_vm = t[5], s_mm = t[6];
        const double denom = TAU * (a_uu * a_vv - a_uv * a_uv);
        st->alpha += convergence * (A_u * a_vv - A_v * a_uv) / denom;
        st->beta += convergence * (A_v * a_uu - A_u * a_uv) / denom;
        st->gain *= 1. + convergence * (s_vm / s_mm - 1);
        if (st->gain < 0.0) st->stop = 1;  // peel.cu:711
    }
}

__global__ void iono_update_kernel(const double* partials, int nblk, const double* lambdas, int nf, IonoDev* st,
                                   double convergence) {
    if (st->stop) return;
    iono_update_body(partials, nblk, lambdas, nf, st, convergence);
}

// grid (nsrc): source s updates st[s] from partials [s][nf][nblk][7].
__global__ void iono_update_batched_kernel(const double* partials, int nblk, const double* lambdas, int nf,
                                           IonoDev* st, double convergence) {
    const int src = blockIdx.x;
    if (st[src].stop) return;
    iono_update_body(partials + (size_t)src * nf * nblk * 7, nblk, lambdas, nf, st + src, convergence);
}

__global__ void subtract_iono_kernel(JonesF32* resid, const JonesF32* model, IonoConsts c, IonoConsts old,
                                     const UVW* uvws, const double* lambdas, int nt, int nbl, int nf) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)nt * nf * nbl) return;
    const int bl = (int)(i % nbl);
    const int f = (int)((i / nbl) % nf);
    const int t = (int)(i / ((size_t)nbl * nf));
    const UVW q = uvws[(size_t)t * nbl + bl];
    const double arg = -TAU * (q.u * c.alpha + q.v * c.beta);
    const double old_arg = -TAU * (q.u * old.alpha + q.v * old.beta);
    const double lam = lambdas[f];
    double s, co, so, cold;
    sincos(arg * lam, &s, &co);
    sincos(old_arg * lam, &so, &cold);
    J2 r = load_j32(resid[i]);
    const J2 m = load_j32(model[i]);
    r = r + m * (cplx{cold, so} * old.gain);
    r = r - m * (cplx{co, s} * c.gain);
    resid[i] = JonesF32{(float)r.a.re, (float)r.a.im, (float)r.b.re, (float)r.b.im,
                        (float)r.c.re, (float)r.c.im, (float)r.d.re, (float)r.d.im};
}

__global__ void add_model_kernel(JonesF32* resid, const JonesF32* model, IonoConsts c, const double* lambdas,
                                 const UVW* uvws, int nt, int nf, int nbl) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)nt * nf * nbl) return;
    const int bl = (int)(i % nbl);
    const int f = (int)((i / nbl) % nf);
    const int t = (int)(i / ((size_t)nbl * nf));
    cplx r = {1.0, 0.0};
    if (!(c.alpha == 0.0 && c.beta == 0.0)) {
        const UVW q = uvws[(size_t)t * nbl + bl];
        const double arg = -TAU * (q.u * c.alpha + q.v * c.beta);
        double s, co;
        sincos(arg * lambdas[f], &s, &co);
        r = cplx{co, s};
    }
    const JonesF32 m = jf32_mul_c32(model[i], r * c.gain);
    JonesF32 o = resid[i];
    o.j00_re = __fadd_rn(o.j00_re, m.j00_re);
    o.j00_im = __fadd_rn(o.j00_im, m.j00_im);
    o.j01_re = __fadd_rn(o.j01_re, m.j01_re);
    o.j01_im = __fadd_rn(o.j01_im, m.j01_im);
    o.j10_re = __fadd_rn(o.j10_re, m.j10_re);
    o.j10_im = __fadd_rn(o.j10_im, m.j10_im);
    o.j11_re = __fadd_rn(o.j11_re, m.j11_re);
    o.j11_im = __fadd_rn(o.j11_im, m.j11_im);
    resid[i] = o;
}

static unsigned grid1(size_t n) { return (unsigned)((n + PT - 1) / PT); }

// Host-side body of iono_loop on a stream; also used by the native peel.
const char* iono_loop_on(const JonesF32* d_resid, const float* d_w, const JonesF32* d_model, JonesF32* d_model_rot,
                         JonesF64* d_fits, IonoConsts* consts, int nbl, int nf, int niter, const UVW* d_uvws,
                         const double* d_lambdas, double convergence, cudaStream_t s) {
    if (nbl <= 0 || nf <= 0) return NULL;
    const int nblk = (nbl + PT - 1) / PT;
    // Layout inside d_fits (nf * nbl JonesF64 = 8 doubles each): partials
    // [nf][nblk][7] first, then the IonoDev block.
    const size_t part_doubles = (size_t)nf * nblk * 7;
    const size_t cap_doubles = (size_t)nf * nbl * 8;
    if (part_doubles + 8 > cap_doubles) return "iono_loop: d_iono_fits too small for this shape";
    double* partials = reinterpret_cast<double*>(d_fits);
    IonoDev* st = reinterpret_cast<IonoDev*>(partials + ((part_doubles + 3) & ~(size_t)3));
    IonoDev h = {consts->alpha, consts->beta, consts->gain, 0, 0};
    HDC_CUDA_RET_STR(cudaMemcpyAsync(st, &h, sizeof(h), cudaMemcpyHostToDevice, s));
    dim3 g(nblk, nf);
    for (int it = 0; it < niter; it++) {
        iono_partials_kernel<<<g, PT, 0, s>>>(d_resid, d_w, d_model, d_model_rot, st, d_uvws, d_lambdas, nbl, nf,
                                              partials);
        count_launches(1);
        iono_update_kernel<<<1, PT, 0, s>>>(partials, nblk, d_lambdas, nf, st, convergence);
        count_launches(1);
    }
    HDC_CUDA_RET_STR(cudaGetLastError());
    HDC_CUDA_RET_STR(cudaMemcpyAsync(&h, st, sizeof(h), cudaMemcpyDeviceToHost, s));
    HDC_CUDA_RET_STR(cudaStreamSynchronize(s));
    consts->alpha = h.alpha;
    consts->beta = h.beta;
    consts->gain = h.gain;
    return NULL;
}


// iono_loop for a batch of sources on one stream, every source starting
// from its own constants in `consts` and writing the fitted ones back; one
// host read at the end.  Buffers: resid/model/model_rot [nsrc][nf][nbl],
// uvws [nsrc][nbl]; scratch holds partials [nsrc][nf][nblk][7] then the
// per-source IonoDev states.
size_t iono_batched_scratch_bytes(int nsrc, int nbl, int nf) {
    const int nblk = (nbl + PT - 1) / PT;
    return sizeof(double) * ((size_t)nsrc * nf * nblk * 7 + 4) + sizeof(IonoDev) * (size_t)nsrc;
}

const char* iono_loop_batched_on(const JonesF32* d_resid, const float* d_w, const JonesF32* d_model,
                                 JonesF32* d_model_rot, void* d_scratch, IonoConsts* consts, int nsrc, int nbl, int nf,
                                 int niter, const UVW* d_uvws, const double* d_lambdas, double convergence,
                                 cudaStream_t s) {
    if (nbl <= 0 || nf <= 0 || nsrc <= 0) return NULL;
    const int nblk = (nbl + PT - 1) / PT;
    double* partials = reinterpret_cast<double*>(d_scratch);
    const size_t part_doubles = (size_t)nsrc * nf * nblk * 7;
    IonoDev* st = reinterpret_cast<IonoDev*>(partials + ((part_doubles + 3) & ~(size_t)3));
    std::vector<IonoDev> h(nsrc);
    for (int i = 0; i < nsrc; i++) h[i] = IonoDev{consts[i].alpha, consts[i].beta, consts[i].gain, 0, 0};
    HDC_CUDA_RET_STR(cudaMemcpyAsync(st, h.data(), sizeof(IonoDev) * nsrc, cudaMemcpyHostToDevice, s));
    const dim3 g(nblk, nf, nsrc);
    for (int it = 0; it < niter; it++) {
        iono_partials_batched_kernel<<<g, PT, 0, s>>>(d_resid, d_w, d_model, d_model_rot, st, d_uvws, d_lambdas, nbl,
                                                      nf, partials);
        iono_update_batched_kernel<<<nsrc, PT, 0, s>>>(partials, nblk, d_lambdas, nf, st, convergence);
        count_launches(2);
    }
    HDC_CUDA_RET_STR(cudaGetLastError());
    HDC_CUDA_RET_STR(cudaMemcpyAsync(h.data(), st, sizeof(IonoDev) * nsrc, cudaMemcpyDeviceToHost, s));
    HDC_CUDA_RET_STR(cudaStreamSynchronize(s));
    for (int i = 0; i < nsrc; i++) consts[i] = IonoConsts{h[i].alpha, h[i].beta, h[i].gain};
    return NULL;
}

// Stream-aware launchers (the drop-in entry points below use stream 0).
cudaError_t k_xyzs_to_uvws(const XYZ* xyzs, const double* lmsts, UVW* uvws, RADec pc, int ntiles, int nbl, int nt,
                           cudaStream_t s) {
    const size_t n = (size_t)nbl * nt;
    if (n == 0) return cudaSuccess;
    xyzs_to_uvws_kernel<<<grid1(n), PT, 0, s>>>(xyzs, lmsts, uvws, pc, ntiles, nbl, nt);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t k_rotate(JonesF32* vis, int nt, int nbl, int nf, const UVW* from, const UVW* to, const double* lambdas,
                     cudaStream_t s) {
    const size_t n = (size_t)nt * nf * nbl;
    if (n == 0) return cudaSuccess;
    rotate_kernel<<<grid1(n), PT, 0, s>>>(vis, nt, nbl, nf, from, to, lambdas);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t k_average(const JonesF32* hi, const float* w, JonesF32* lo, int nt, int nbl, int nf, int favg,
                      cudaStream_t s) {
    const size_t n = (size_t)(nf / favg) * nbl;
    if (n == 0) return cudaSuccess;
    average_kernel<<<grid1(n), PT, 0, s>>>(hi, w, lo, nt, nbl, nf, favg);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t k_subtract_iono(JonesF32* resid, const JonesF32* model, IonoConsts c, IonoConsts old, const UVW* uvws,
                            const double* lambdas, int nt, int nbl, int nf, cudaStream_t s) {
    const size_t n = (size_t)nt * nf * nbl;
    if (n == 0) return cudaSuccess;
    subtract_iono_kernel<<<grid1(n), PT, 0, s>>>(resid, model, c, old, uvws, lambdas, nt, nbl, nf);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t k_add_model(JonesF32* resid, const JonesF32* model, IonoConsts c, const double* lambdas, const UVW* uvws,
                        int nt, int nf, int nbl, cudaStream_t s) {
    const size_t n = (size_t)nt * nf * nbl;
    if (n == 0) return cudaSuccess;
    add_model_kernel<<<grid1(n), PT, 0, s>>>(resid, model, c, lambdas, uvws, nt, nf, nbl);
    count_launches(1);
    return cudaGetLastError();
}

// Low-resolution weights: sum over all timesteps and each channel group,
// clamped at 0 (params/peel/mod.rs:709-755 weights_average).
__global__ void weights_average_kernel(const float* w, float* lo, int nt, int nbl, int nf, int favg) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int nlo = nf / favg;
    if (i >= nlo * nbl) return;
    const int bl = i % nbl, flo = i / nbl;
    double sum = 0.0;
    for (int t = 0; t < nt; t++)
        for (int fc = flo * favg; fc < flo * favg + favg; fc++) sum += (double)w[((size_t)t * nf + fc) * nbl + bl];
    lo[i] = fmaxf((float)sum, 0.0f);
}

cudaError_t k_weights_average(const float* w, float* lo, int nt, int nbl, int nf, int favg, cudaStream_t s) {
    const size_t n = (size_t)(nf / favg) * nbl;
    if (n == 0) return cudaSuccess;
    weights_average_kernel<<<grid1(n), PT, 0, s>>>(w, lo, nt, nbl, nf, favg);
    count_launches(1);
    return cudaGetLastError();
}

}  // namespace hdc

using namespace hdc;

extern "C" const char* xyzs_to_uvws(const XYZ* d_xyzs, const double* d_lmsts, UVW* d_uvws, RADec pointing_centre,
                                    int num_tiles, int num_baselines, int num_timesteps) {
    const size_t n = (size_t)num_baselines * num_timesteps;
    if (n == 0) return NULL;
    xyzs_to_uvws_kernel<<<grid1(n), PT>>>(d_xyzs, d_lmsts, d_uvws, pointing_centre, num_tiles, num_baselines,
                                          num_timesteps);
    count_launches(1);
    HDC_CUDA_RET_STR(cudaGetLastError());
    return NULL;
}

extern "C" const char* rotate(JonesF32* vis_fb, const int num_timesteps, const int num_baselines, const int num_freqs,
                              const UVW* uvws_from, const UVW* uvws_to, const double* lambdas) {
    const size_t n = (size_t)num_timesteps * num_freqs * num_baselines;
    if (n == 0) return NULL;
    rotate_kernel<<<grid1(n), PT>>>(vis_fb, num_timesteps, num_baselines, num_freqs, uvws_from, uvws_to, lambdas);
    count_launches(1);
    HDC_CUDA_RET_STR(cudaGetLastError());
    return NULL;
}

extern "C" const char* average(const JonesF32* d_high_res_vis, const float* d_high_res_weights,
                               JonesF32* d_low_res_vis, const int num_timesteps, const int num_baselines,
                               const int num_freqs, const int freq_average_factor) {
    if (freq_average_factor <= 0) return "average: freq_average_factor must be positive";
    const size_t n = (size_t)(num_freqs / freq_average_factor) * num_baselines;
    if (n == 0) return NULL;
    average_kernel<<<grid1(n), PT>>>(d_high_res_vis, d_high_res_weights, d_low_res_vis, num_timesteps, num_baselines,
                                     num_freqs, freq_average_factor);
    count_launches(1);
    HDC_CUDA_RET_STR(cudaGetLastError());
    return NULL;
}

extern "C" const char* iono_loop(const JonesF32* d_vis_residual, const float* d_vis_weights,
                                 const JonesF32* d_vis_model, JonesF32* d_vis_model_rotated, JonesF64* d_iono_fits,
                                 IonoConsts* iono_consts, const int num_baselines, const int num_freqs,
                                 const int num_iterations, const UVW* d_uvws, const double* d_lambdas_m,
                                 const double convergence) {
    return iono_loop_on(d_vis_residual, d_vis_weights, d_vis_model, d_vis_model_rotated, d_iono_fits, iono_consts,
                        num_baselines, num_freqs, num_iterations, d_uvws, d_lambdas_m, convergence, 0);
}

extern "C" const char* subtract_iono(JonesF32* d_vis_residual, const JonesF32* d_vis_model,
                                     const IonoConsts iono_consts, const IonoConsts old_iono_consts, const UVW* d_uvws,
                                     const double* d_lambdas_m, const int num_timesteps, const int num_baselines,
                                     const int num_freqs) {
    const size_t n = (size_t)num_timesteps * num_freqs * num_baselines;
    if (n == 0) return NULL;
    subtract_iono_kernel<<<grid1(n), PT>>>(d_vis_residual, d_vis_model, iono_consts, old_iono_consts, d_uvws,
                                           d_lambdas_m, num_timesteps, num_baselines, num_freqs);
    count_launches(1);
    HDC_CUDA_RET_STR(cudaGetLastError());
    return NULL;
}

extern "C" const char* add_model(JonesF32* d_vis_residual, const JonesF32* d_vis_model, const IonoConsts iono_consts,
                                 const double* d_lambdas_m, const UVW* d_uvws, const int num_timesteps,
                                 const int num_freqs, const int num_baselines) {
    const size_t n = (size_t)num_timesteps * num_freqs * num_baselines;
    if (n == 0) return NULL;
    add_model_kernel<<<grid1(n), PT>>>(d_vis_residual, d_vis_model, iono_consts, d_lambdas_m, d_uvws, num_timesteps,
                                       num_freqs, num_baselines);
    count_launches(1);
    HDC_CUDA_RET_STR(cudaGetLastError());
    return NULL;
}
