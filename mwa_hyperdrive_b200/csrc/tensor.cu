// Tensor-core factored point-source predict (tcgen05, sm_100a).
//
// For one timestep and channel the baseline UVW is a tile difference
// (uvw_pq = uvw_p - uvw_q, as marlu's xyzs_to_cross_uvws builds it), so the
// point-source phasor factors: exp(2 pi i theta_pq,c) = A_pc conj(A_qc) with
// A_pc = exp(2 pi i (u_p l_c + v_p m_c + w_p (n_c - 1)) f / c).  Each
// polarisation ab of the visibility matrix is then a weighted Gram product
//     V^ab = A diag(W^ab) A^H          (tiles x tiles, contracted over components)
// with W = B S B^H the per-component brightness (shared beam).  W is
// Hermitian, so V^YX = (V^XY)^H and V^XX, V^YY are Hermitian: three complex
// products give all four correlations of every baseline.
//
// Kernel: one CTA per (channel, polarisation group); group 0 = XX + YY,
// group 1 = XY.  With X = A diag(W) s (s a power-of-two range scale) and
// Y = A, the real form is
//     Re V = Xr Yr^T + Xi Yi^T,   Im V = Xi Yr^T - Xr Yi^T,
// computed by tcgen05.mma (kind::f16, M = N = 128, K = 16 per instruction,
// FP32 accumulators in TMEM, the minus sign via the A-negate bit).  Producer
// warps compute the FP64 per-tile phases (exact turn-domain range reduction,
// sincospi) for 32 components per stage, form X and Y, split every value into
// an fp16 pair (hi = fp16(x), lo = fp16(x - hi): 22 bits, inputs exact to
// ~2^-24) and write them to shared memory in the K-major core-matrix layout;
// one thread issues the 4 partial products (hi.hi, hi.lo, lo.hi, lo.lo) of
// every term.  Two stages double-buffer producers against the tensor core.
// The epilogue reads TMEM with tcgen05.ld and adds the upper-triangle
// baselines into the visibilities.
//
// Every mbarrier wait is bounded by the global timer; on a timeout the CTA
// records KERR_TIMEOUT, waits (bounded) for its issued MMAs and frees TMEM.

#include <cuda_fp16.h>

#include <cmath>

#include "modeller.cuh"

namespace hdc {
namespace tc {

constexpr int NT = 128;   // tiles = M = N
constexpr int KC = 32;    // components per stage (K elements per operand part)
constexpr int NSTAGE = 2;
constexpr int NPW = 8;    // producer / epilogue warps
constexpr int THREADS = (NPW + 1) * 32;
constexpr int TILE_BYTES = NT * KC * 2;  // one fp16 operand tile, 8 KB
constexpr int LBO = 128;                 // bytes between 8-element K chunks
constexpr int SBO = (KC / 8) * 128;      // bytes between 8-row groups
constexpr int TILES_PER_STAGE = 12;      // Y: 4, X: up to 2 pols x 4
constexpr int STAGE_BYTES = TILES_PER_STAGE * TILE_BYTES;
constexpr int SMEM_BYTES = NSTAGE * STAGE_BYTES + 1024;

struct Params {
    int nf, nbl, ntiles, nc;
    const double* freqs;
    const XYZ* xyzs;
    double s_ha, c_ha, s_dec, c_dec;
    const double4* lmn;    // [nc] turn units
    const JonesF64* W;     // [nf][nc]
    void* vis;             // [nf][nbl]
    int* err;
};

__device__ __forceinline__ uint64_t smem_desc(uint32_t addr) {
    // K-major, no swizzle: start >> 4, LBO >> 4 at bit 16, SBO >> 4 at bit 32,
    // version 1 at bit 46, layout type 0.
    return (uint64_t)((addr >> 4) & 0x3FFF) | ((uint64_t)(LBO >> 4) << 16) | ((uint64_t)(SBO >> 4) << 32) |
           ((uint64_t)1 << 46);
}

// kind::f16 instruction descriptor: f16 A and B, f32 D, K-major, M=N=128.
__host__ __device__ constexpr uint32_t idesc(bool neg_a) {
    return (1u << 4) | (0u << 7) | (0u << 10) | ((neg_a ? 1u : 0u) << 13) | ((uint32_t)(NT >> 3) << 17) |
           ((uint32_t)(NT >> 4) << 24);
}

__device__ __forceinline__ void mma_f16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t id, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
        :
        : "r"(d_tmem), "l"(a), "l"(b), "r"(id), "r"(acc), "r"(0), "r"(0), "r"(0), "r"(0));
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t addr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(addr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

// byte offset of element (row, k) in a K-major core-matrix tile
__device__ __forceinline__ uint32_t tile_off(int row, int k) {
    return (uint32_t)((row >> 3) * SBO + (k >> 3) * LBO + (row & 7) * 16 + (k & 7) * 2);
}

__device__ __forceinline__ void split16(double x, __half& h, __half& l) {
    h = __double2half(x);  // round to nearest even
    l = __double2half(x - (double)__half2float(h));
}

// tile index inside a stage
__device__ __forceinline__ int y_tile(int piece, int part) { return piece * 2 + part; }
__device__ __forceinline__ int x_tile(int pol, int piece, int part) { return 4 + pol * 4 + piece * 2 + part; }

template <bool OUT64>
__global__ void __launch_bounds__(THREADS, 1) gram_kernel(const Params P) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    __shared__ alignas(8) uint64_t full_bar[NSTAGE], empty_bar[NSTAGE], done_bar;
    __shared__ uint32_t tmem_base_s;
    __shared__ float red_s[THREADS / 32];
    __shared__ volatile int abort_s;

    unsigned char* smem = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    const int f = blockIdx.x;
    const int group = blockIdx.y;          // 0: XX+YY, 1: XY
    const int npol = group == 0 ? 2 : 1;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int ncols = group == 0 ? 512 : 256;

    if (tid == 0) {
        for (int s = 0; s < NSTAGE; s++) {
            mbar_init(&full_bar[s], NPW * 32);
            mbar_init(&empty_bar[s], 1);
        }
        mbar_init(&done_bar, 1);
        abort_s = 0;
        fence_barrier_init();
    }
    if (warp == 0) {
        // allocate TMEM (one warp), publish its base address in shared memory
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base_s)),
                     "r"(ncols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }

    // range scale: s = 2^e with max |W component| * s in [8192, 16384)
    const double freq = P.freqs[f];
    float mx = 0.f;
    for (int c = tid; c < P.nc; c += THREADS) {
        const JonesF64 w = P.W[(size_t)f * P.nc + c];
        if (group == 0)
            mx = fmaxf(mx, (float)fmax(fmax(fabs(w.j00_re), fabs(w.j00_im)), fmax(fabs(w.j11_re), fabs(w.j11_im))));
        else
            mx = fmaxf(mx, (float)fmax(fabs(w.j01_re), fabs(w.j01_im)));
    }
    for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if (lane == 0) red_s[warp] = mx;
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    float wmax = 0.f;
    for (int i = 0; i < THREADS / 32; i++) wmax = fmaxf(wmax, red_s[i]);
    const double scale = wmax > 0.f ? exp2(floor(log2(16384.0 / (double)wmax))) : 1.0;
    const double inv_scale = 1.0 / scale;
    const uint32_t tmem = tmem_base_s;
    // A polarisation group whose weights are all exactly zero (e.g. XY/YX of
    // a Stokes-I sky) contributes exactly zero: skip its work.
    const bool skip = !(wmax > 0.f);
    const int nchunks = skip ? 0 : (P.nc + KC - 1) / KC;

    if (warp < NPW) {
        // ------------------------------------------------ producers
        const int r = tid & (NT - 1);  // tile (row of X and of Y)
        const int half = tid >> 7;     // which 16 components of the stage
        double u = 0.0, v = 0.0, w = 0.0;
        const bool real_tile = r < P.ntiles;
        if (real_tile) {
            const XYZ x = P.xyzs[r];
            const double ool = freq / VEL_C;
            u = (P.s_ha * x.x + P.c_ha * x.y) * ool;
            v = (-P.s_dec * P.c_ha * x.x + P.s_dec * P.s_ha * x.y + P.c_dec * x.z) * ool;
            w = (P.c_dec * P.c_ha * x.x - P.c_dec * P.s_ha * x.y + P.s_dec * x.z) * ool;
        }
        for (int k = 0; k < nchunks; k++) {
            const int st = k % NSTAGE;
            if (k >= NSTAGE) {
                const bool ok = mbar_wait_bounded(&empty_bar[st], ((k / NSTAGE) - 1) & 1, P.err);
                if (!ok) abort_s = 1;
            }
            if (abort_s) break;
            unsigned char* sb = smem + st * STAGE_BYTES;
            // two sub-blocks of 8 components -> one 16-byte store per tile each
            for (int sub = 0; sub < 2; sub++) {
                const int kbase = half * 16 + sub * 8;  // k offset inside the stage
                __align__(16) __half yv[4][8];          // [piece*2+part][j]
                __align__(16) __half xv[2][4][8];       // [pol][piece*2+part][j]
#pragma unroll
                for (int j = 0; j < 8; j++) {
                    const int c = k * KC + kbase + j;
                    double ar = 0.0, ai = 0.0;
                    double br[2] = {0.0, 0.0}, bi[2] = {0.0, 0.0};
                    if (c < P.nc && real_tile) {
                        const double2 lm = __ldg(reinterpret_cast<const double2*>(P.lmn + c));
                        const double ln = __ldg(reinterpret_cast<const double*>(P.lmn + c) + 2);
                        const cplx a = phasor_turns(u * lm.x + v * lm.y + w * ln);
                        ar = a.re;
                        ai = a.im;
                        const JonesF64* wp = P.W + (size_t)f * P.nc + c;
                        if (group == 0) {
                            const double2 xx = __ldg(reinterpret_cast<const double2*>(wp));
                            const double2 yy = __ldg(reinterpret_cast<const double2*>(wp) + 3);
                            const cplx bx = a * cplx{xx.x * scale, xx.y * scale};
                            const cplx by = a * cplx{yy.x * scale, yy.y * scale};
                            br[0] = bx.re;
                            bi[0] = bx.im;
                            br[1] = by.re;
                            bi[1] = by.im;
                        } else {
                            const double2 xy = __ldg(reinterpret_cast<const double2*>(wp) + 1);
                            const cplx b = a * cplx{xy.x * scale, xy.y * scale};
                            br[0] = b.re;
                            bi[0] = b.im;
                        }
                    }
                    split16(ar, yv[0][j], yv[2][j]);
                    split16(ai, yv[1][j], yv[3][j]);
                    for (int p = 0; p < npol; p++) {
                        split16(br[p], xv[p][0][j], xv[p][2][j]);
                        split16(bi[p], xv[p][1][j], xv[p][3][j]);
                    }
                }
                const uint32_t off = tile_off(r, kbase);
#pragma unroll
                for (int t = 0; t < 4; t++)
                    *reinterpret_cast<uint4*>(sb + y_tile(t >> 1, t & 1) * TILE_BYTES + off) =
                        *reinterpret_cast<const uint4*>(yv[t]);
                for (int p = 0; p < npol; p++)
#pragma unroll
                    for (int t = 0; t < 4; t++)
                        *reinterpret_cast<uint4*>(sb + x_tile(p, t >> 1, t & 1) * TILE_BYTES + off) =
                            *reinterpret_cast<const uint4*>(xv[p][t]);
            }
            fence_proxy_async_smem();  // make the generic-proxy stores visible to the tensor core
            mbar_arrive(&full_bar[st]);
        }
    } else {
        // ------------------------------------------------ MMA issuer (one thread)
        if (lane == 0) {
            const uint32_t sbase = smem_u32(smem);
            int issued = 0;
            for (int k = 0; k < nchunks; k++) {
                const int st = k % NSTAGE;
                const bool ok = mbar_wait_bounded(&full_bar[st], (k / NSTAGE) & 1, P.err);
                if (!ok) {
                    abort_s = 1;
                    break;
                }
                tc_fence_after();
                const uint32_t sb = sbase + st * STAGE_BYTES;
                for (int p = 0; p < npol; p++) {
                    const uint32_t d_re = tmem + p * 256, d_im = tmem + p * 256 + 128;
                    // (x part, y part, negate A, accumulator)
                    const int terms[4][4] = {{0, 0, 0, 0}, {1, 1, 0, 0}, {1, 0, 0, 1}, {0, 1, 1, 1}};
                    for (int tm = 0; tm < 4; tm++) {
                        const uint32_t d = terms[tm][3] ? d_im : d_re;
                        const uint32_t id = idesc(terms[tm][2] != 0);
                        for (int pa = 0; pa < 2; pa++)
                            for (int pb = 0; pb < 2; pb++)
                                for (int kk = 0; kk < KC / 16; kk++) {
                                    const uint32_t a = sb + x_tile(p, pa, terms[tm][0]) * TILE_BYTES + kk * 2 * LBO;
                                    const uint32_t b = sb + y_tile(pb, terms[tm][1]) * TILE_BYTES + kk * 2 * LBO;
                                    // the first product into each accumulator overwrites it
                                    const bool first = (k == 0) && (tm < 2 ? tm == 0 : tm == 2) && pa == 0 &&
                                                       pb == 0 && kk == 0;
                                    mma_f16(d, smem_desc(a), smem_desc(b), id, first ? 0u : 1u);
                                }
                    }
                }
                mma_commit(&empty_bar[st]);  // stage free once these MMAs have read it
                issued++;
            }
            mma_commit(&done_bar);
            (void)issued;
        }
    }

    // ---------------------------------------------------- epilogue
    __syncthreads();
    const bool aborted = abort_s != 0;
    const bool ok = mbar_wait_bounded(&done_bar, 0, P.err);
    tc_fence_after();
    if (!aborted && ok && !skip && warp < NPW) {
        const int lg = warp & 3;           // TMEM lane group this warp may access
        const int chalf = warp >> 2;       // column half
        const int p = lg * 32 + lane;      // row (tile 1 candidate)
        const uint32_t lane_addr = tmem + ((uint32_t)(lg * 32) << 16);
        const int n = P.ntiles;
        for (int q0 = chalf * 64; q0 < chalf * 64 + 64; q0 += 16) {
            if (group == 0) {
                float xr[16], xi[16], yr[16], yi[16];
                tmem_ld16(lane_addr + q0, xr);
                tmem_ld16(lane_addr + 128 + q0, xi);
                tmem_ld16(lane_addr + 256 + q0, yr);
                tmem_ld16(lane_addr + 384 + q0, yi);
                if (p < n) {
                    for (int j = 0; j < 16; j++) {
                        const int q = q0 + j;
                        if (q <= p || q >= n) continue;
                        const size_t o = (size_t)f * P.nbl + baseline_index(p, q, n);
                        if (OUT64) {
                            JonesF64* vp = reinterpret_cast<JonesF64*>(P.vis) + o;
                            vp->j00_re += xr[j] * inv_scale;
                            vp->j00_im += xi[j] * inv_scale;
                            vp->j11_re += yr[j] * inv_scale;
                            vp->j11_im += yi[j] * inv_scale;
                        } else {
                            JonesF32* vp = reinterpret_cast<JonesF32*>(P.vis) + o;
                            vp->j00_re += (float)(xr[j] * inv_scale);
                            vp->j00_im += (float)(xi[j] * inv_scale);
                            vp->j11_re += (float)(yr[j] * inv_scale);
                            vp->j11_im += (float)(yi[j] * inv_scale);
                        }
                    }
                }
            } else {
                float dr[16], di[16];
                tmem_ld16(lane_addr + q0, dr);
                tmem_ld16(lane_addr + 128 + q0, di);
                if (p < n) {
                    for (int j = 0; j < 16; j++) {
                        const int q = q0 + j;
                        if (q == p || q >= n) continue;
                        // q > p: XY of baseline (p, q); q < p: YX of (q, p) = conj(XY(p, q))
                        const bool upper = q > p;
                        const size_t o = (size_t)f * P.nbl + (upper ? baseline_index(p, q, n) : baseline_index(q, p, n));
                        const double re = dr[j] * inv_scale;
                        const double im = (upper ? 1.0 : -1.0) * di[j] * inv_scale;
                        if (OUT64) {
                            JonesF64* vp = reinterpret_cast<JonesF64*>(P.vis) + o;
                            if (upper) {
                                vp->j01_re += re;
                                vp->j01_im += im;
                            } else {
                                vp->j10_re += re;
                                vp->j10_im += im;
                            }
                        } else {
                            JonesF32* vp = reinterpret_cast<JonesF32*>(P.vis) + o;
                            if (upper) {
                                vp->j01_re += (float)re;
                                vp->j01_im += (float)im;
                            } else {
                                vp->j10_re += (float)re;
                                vp->j10_im += (float)im;
                            }
                        }
                    }
                }
            }
        }
    }
    if (aborted || !ok) {
        if (tid == 0) atomicOr(P.err, KERR_TIMEOUT);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols) : "memory");
    }
}

}  // namespace tc

struct TensorState {
    bool configured = false;
};

int Modeller::tensor_setup() {
    if (ntiles > tc::NT) {
        set_error("the tensor-core predict supports up to %d tiles (have %d)", tc::NT, ntiles);
        return HDC_ERR_UNSUPPORTED;
    }
    if (!tc) tc = new TensorState();
    if (!tc->configured) {
        HDC_CUDA_RET_INT(cudaFuncSetAttribute(tc::gram_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              tc::SMEM_BYTES));
        HDC_CUDA_RET_INT(cudaFuncSetAttribute(tc::gram_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              tc::SMEM_BYTES));
        tc->configured = true;
    }
    return HDC_OK;
}

int Modeller::tensor_points(double lst, void* d_vis, bool out64, cudaStream_t s) {
    if (t[0].nc == 0) return HDC_OK;
    tc::Params P;
    P.nf = nf;
    P.nbl = nbl;
    P.ntiles = ntiles;
    P.nc = t[0].nc;
    P.freqs = d_freqs;
    P.xyzs = d_xyzs;
    const double ha = lst - pc.ra;
    P.s_ha = std::sin(ha);
    P.c_ha = std::cos(ha);
    P.s_dec = std::sin(pc.dec);
    P.c_dec = std::cos(pc.dec);
    P.lmn = t[0].d_lmn;
    P.W = weights(0);
    P.vis = d_vis;
    P.err = d_err;
    dim3 grid(nf, 2);
    if (out64)
        tc::gram_kernel<true><<<grid, tc::THREADS, tc::SMEM_BYTES, s>>>(P);
    else
        tc::gram_kernel<false><<<grid, tc::THREADS, tc::SMEM_BYTES, s>>>(P);
    count_launches(1);
    HDC_CUDA_RET_INT(cudaGetLastError());
    return HDC_OK;
}

void Modeller::tensor_release() {
    delete tc;
    tc = nullptr;
}

}  // namespace hdc
