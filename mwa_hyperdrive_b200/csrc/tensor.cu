// Tensor-core factored point-source predict (tcgen05, sm_100a), exact
// integer accumulation.
//
// For one timestep and channel the baseline UVW is a tile difference
// (uvw_pq = uvw_p - uvw_q, as marlu's xyzs_to_cross_uvws builds it), so the
// point-source phasor factors: exp(2 pi i theta_pq,c) = A_pc conj(A_qc) with
// A_pc = exp(2 pi i (u_p l_c + v_p m_c + w_p (n_c - 1)) f / c).  Each
// polarisation ab of the visibility matrix is then a weighted Gram product
//     V^ab = X Y^H,  X = A diag(W^ab),  Y = A     (tiles x tiles, over components)
// with W = B S B^H the per-component brightness (shared beam).  W is
// Hermitian, so V^YX = (V^XY)^H and V^XX, V^YY are Hermitian: three complex
// products give all four correlations of every baseline.  In real form
//     Re V = Xr Yr^T + Xi Yi^T,   Im V = Xi Yr^T + Xr (-Yi)^T.
//
// Numbers.  A tensor core accumulating in FP32 does not round to nearest, and
// its error grows with every K step.  Here every operand is instead a
// fixed-point integer split into balanced byte digits, and the digit planes
// are multiplied on the integer tensor core (kind::i8, s8 x s8, s32
// accumulators), where every sum is exact:
//   x = rint(X sx), |x| < 2^31 - 2^24 (sx from the channel's largest |W|):
//       x = d0 2^24 + d1 2^16 + d2 2^8 + d3, every d_i in [-128, 127];
//   y = rint(A sy), |y| < 2^22: y = e0 2^16 + e1 2^8 + e2.
// Balanced digits are the bytes of (x + 0x808080) ^ 0x808080: adding 128 to
// each lower digit position and flipping its top bit turns excess-128 bytes
// into two's-complement ones (the flip is applied to four digits of a byte
// plane at once).  They have zero mean, so the products left out
// below do not bias the sum (unsigned lower bytes would: their dropped
// products are all positive and grow with the number of components).
// x y = sum_ij d_i e_j 2^(40 - 8(i + j)); the nine plane products with
// i + j <= 3 are kept (the rest weigh < 2^-30 of full scale), each into the
// accumulator of its class w = i + j, and the epilogue forms
// V = sum_w D_w 2^(40 - 8w) / (sx sy) in FP64.  The only rounding is in the
// inputs: the phase, reduced exactly in FP64 to a quadrant q and a remainder
// r in [-1/2, 1/2] quarter-turns; sin and cos of (pi/2) r from FP32
// polynomials (least-squares fits, mwa_hyperdrive_b200/phasor_poly.py,
// < 0.75 ulp); X = (W sx) A in FP32; the two roundings to integers (2^-23 of A,
// 2^-31 of the channel's largest |X|).  A launch covers at most KPASS
// components, so no s32 sum can overflow.
//
// Kernel: one CTA per (channel, polarisation, half of the tile columns); M =
// 128 tiles (rows of X), 64 tile columns (rows of Y), K = 32 components per
// stage.  Sixteen producer warps compute the per-tile phasors, X and Y, the
// byte planes, and write them to shared memory in the K-major core-matrix
// layout (one warp store = one 128-byte core matrix); the stage's component data
// (l, m, n, W) is staged in shared memory one stage ahead, so the phasor loop
// reads no global memory.  One thread issues the 18 MMAs of a stage (9 plane
// pairs x {Xr, Xi}, N = 128 = [Re | Im] of the 64 columns, which keeps the
// operand bytes read from shared memory per MAC at half of what separate
// N = 64 products would need) into 4 TMEM accumulators (one per class, 128
// columns each = all 512 columns).  Four stages let the producers
// run ahead of the tensor core.  The epilogue reads TMEM with tcgen05.ld,
// combines the classes in FP64 and adds the baselines of its columns into
// the visibilities (XX, YY: q > p; XY: q > p as XY, q < p as YX = conj).
//
// Every mbarrier wait is bounded by the global timer; on a timeout the CTA
// records KERR_TIMEOUT, waits (bounded) for its issued MMAs and frees TMEM.

#include <algorithm>
#include <cmath>

#include <mutex>

#include "modeller.cuh"

namespace hdc {
namespace tc {

constexpr int NT = 128;    // tiles = M
constexpr int NH = 64;     // tile columns per CTA
constexpr int NB = 2 * NH; // MMA N: [Re | Im] of the NH columns
constexpr int KC = 32;     // components per stage = MMA K (bytes)
constexpr int NSTAGE = 4;
constexpr int CRING = NSTAGE + 2;  // component-data ring: producer warps may be NSTAGE stages apart
constexpr int NPW = 16;    // producer / epilogue warps
constexpr int NPT = NPW * 32;   // producer threads
constexpr int THREADS = NPT + 32;
constexpr int XDIG = 4;    // byte planes of x
constexpr int YDIG = 3;    // byte planes of y
constexpr int XT_BYTES = NT * KC;                           // one X plane tile, 4 KB
constexpr int YT_BYTES = NH * KC;                           // one Y plane tile, 2 KB
constexpr int Y_OFF = 2 * XDIG * XT_BYTES;                  // X: [re, im][4 planes]
constexpr int STAGE_BYTES = Y_OFF + 3 * YDIG * YT_BYTES;    // Y: [re, im, -im][3 planes]
constexpr int SMEM_BYTES = NSTAGE * STAGE_BYTES + 1024;
constexpr int LBO = 128;             // bytes between the two 16-byte K core matrices of a row group
constexpr int SBO = (KC / 16) * 128; // bytes between 8-row groups
constexpr int TMEM_COLS = 512;       // 4 classes x NB
constexpr int KPASS = 16384;         // components per launch: 3 pairs x 2 x 2^14 x KPASS < 2^31
constexpr float SY = 4128768.0f;     // 2^22 - 2^16: |A| <= 1 -> |y| < 2^22
// y + 0x8080 as FP32 bits: 1.5 * 2^23 rounds |v| < 2^22 to an integer in
// the mantissa; the extra 0x8080 is the balancing offset of the two lower
// digits.  The mantissa field then holds 2^22 + 0x8080 + y, so byte 2 is the
// top digit + 0x40 and bytes 1, 0 the excess-128 lower digits.
constexpr float YOFF = 12582912.0f + 32896.0f;

// component data of one stage, staged in shared memory (structure of arrays
// so that 16-byte loads of consecutive components are conflict-free)
struct CompStage {
    double l[KC], m[KC], n[KC];  // turn units (n - 1 in n)
    float2 w[KC];                // W of this polarisation times the x scale sx
};

struct Params {
    int nf, nbl, ntiles, nc, c0, cn;
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

// kind::i8 instruction descriptor: s32 D (bits 4-5 = 2), A and B signed
// (bits 7 and 10 = 1), K-major, N at bit 17 (>> 3), M at bit 24 (>> 4).
__host__ __device__ constexpr uint32_t idesc_s8() {
    return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(NB >> 3) << 17) | ((uint32_t)(NT >> 4) << 24);
}

__device__ __forceinline__ void mma_i8(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t id, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
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

// 8 columns of 32 lanes (one per thread) from TMEM; the caller waits with
// tmem_wait_ld before using the registers.
__device__ __forceinline__ void tmem_ld8(uint32_t addr, int* v) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                 : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7])
                 : "r"(addr));
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// byte offset of the 16-byte chunk (row, K half) in a K-major core-matrix tile
__device__ __forceinline__ uint32_t chunk_off(int row, int khalf) {
    return (uint32_t)((row >> 3) * SBO + khalf * LBO + (row & 7) * 16);
}

// Byte planes of 4 integers: word b holds byte b of v[0..3], v[j] at byte j
// (a 4x4 byte transpose).
__device__ __forceinline__ void byte_planes4(const int* v, uint32_t* w) {
    const uint32_t a = (uint32_t)v[0], b = (uint32_t)v[1], c = (uint32_t)v[2], d = (uint32_t)v[3];
    const uint32_t t0 = __byte_perm(a, b, 0x5140), t1 = __byte_perm(c, d, 0x5140);
    const uint32_t t2 = __byte_perm(a, b, 0x7362), t3 = __byte_perm(c, d, 0x7362);
    w[0] = __byte_perm(t0, t1, 0x5410);
    w[1] = __byte_perm(t0, t1, 0x7632);
    w[2] = __byte_perm(t2, t3, 0x5410);
    w[3] = __byte_perm(t2, t3, 0x7632);
}

// per-byte correction of four digits at once: b - 64 for bytes b in [0, 127]
// (b ^ 0x40 when bit 6 is set, b ^ 0xC0 when it is clear; bit 6 moves to
// bit 7 inside its byte).  Excess-128 digits become two's complement with
// a plain XOR 0x80.
__device__ __forceinline__ uint32_t minus64(uint32_t w) {
    return w ^ 0x40404040u ^ ((~w & 0x40404040u) << 1);
}

// all producer threads: barrier 1, true when any of them passed true
__device__ __forceinline__ bool producers_sync_or(bool v) {
    int r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\t"
        "setp.ne.b32 p, %1, 0;\n\t"
        "bar.red.or.pred q, 1, %2, p;\n\t"
        "selp.b32 %0, 1, 0, q;\n\t}"
        : "=r"(r)
        : "r"((int)v), "r"(NPT)
        : "memory");
    return r != 0;
}

// shared-memory tile offsets inside a stage; digit 0 is the signed top byte
__device__ __forceinline__ uint32_t x_tile(int part, int digit) {
    return (uint32_t)((part * XDIG + digit) * XT_BYTES);
}
// Y tiles of one digit lie in the order [Yi | Yr | -Yi] (64 rows each), so
// that [Yr; -Yi] (from the Yr tile) and [Yi; Yr] (from the Yi tile) are
// 128-row B operands: Xr [Yr; -Yi]^T + Xi [Yi; Yr]^T = [Re | Im] of X Y^H.
// part: 0 = Yr, 1 = Yi, 2 = -Yi
__device__ __forceinline__ uint32_t y_tile(int part, int digit) {
    const int slot = part == 0 ? 1 : (part == 1 ? 0 : 2);
    return (uint32_t)(Y_OFF + (digit * 3 + slot) * YT_BYTES);
}
// TMEM column of accumulator class w ([Re | Im], NB columns)
__device__ __forceinline__ uint32_t acc_col(int w) { return (uint32_t)(w * NB); }

template <bool OUT64>
__global__ void __launch_bounds__(THREADS, 1) gram_i8_kernel(const Params P) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    __shared__ alignas(8) uint64_t full_bar[NSTAGE], empty_bar[NSTAGE], done_bar;
    __shared__ uint32_t tmem_base_s;
    __shared__ double red_s[THREADS / 32];
    __shared__ volatile int abort_s;
    __shared__ __align__(16) CompStage comp_s[CRING];
    __shared__ alignas(8) uint64_t comp_bar[CRING];

    unsigned char* smem = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    const int f = blockIdx.x;
    const int pol = blockIdx.y;   // 0: XX, 1: YY, 2: XY
    const int hcol = blockIdx.z;  // tile columns [hcol * NH, hcol * NH + NH)
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    // W component of this polarisation (JonesF64 as 4 double2: xx, xy, yx, yy)
    const int wsel = pol == 0 ? 0 : (pol == 1 ? 3 : 1);

    // largest |W| of the pass sets the x scale
    double mx = 0.0;
    for (int c = tid; c < P.cn; c += THREADS) {
        const double2 w = __ldg(reinterpret_cast<const double2*>(P.W + (size_t)f * P.nc + P.c0 + c) + wsel);
        mx = fmax(mx, hypot(w.x, w.y));
    }
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if (lane == 0) red_s[warp] = mx;
    if (tid == 0) {
        for (int s = 0; s < NSTAGE; s++) {
            mbar_init(&full_bar[s], NPW);  // one arrival per producer warp
            mbar_init(&empty_bar[s], 1);
        }
        for (int s = 0; s < CRING; s++) mbar_init(&comp_bar[s], 1);  // the stashing warp arrives once
        mbar_init(&done_bar, 1);
        abort_s = 0;
        fence_barrier_init();
    }
    __syncthreads();
    double wmax = 0.0;
    for (int i = 0; i < THREADS / 32; i++) wmax = fmax(wmax, red_s[i]);
    // A polarisation whose weights are all exactly zero (e.g. XY of a
    // Stokes-I sky) contributes exactly zero; a column half beyond the
    // last tile has no baselines.
    if (!(wmax > 0.0) || hcol * NH >= P.ntiles) return;
    const float sx = (float)((2147483648.0 - 33554432.0) / wmax);  // (2^31 - 2^25) / max|W|
    const double inv = 1.0 / ((double)sx * (double)SY);

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base_s)),
                     "r"(TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_base_s;
    const int nchunks = (P.cn + KC - 1) / KC;
    const double freq = P.freqs[f];

    if (warp < NPW) {
        // ------------------------------------------------ producers
        // warp = 8 tile rows x 16 components of a stage; lane = (row rl, quad of
        // 4 components), and every thread also takes the row 64 tiles down, so a
        // warp's store of one byte plane is one whole 128-byte core matrix and
        // exactly one of a thread's two rows lies in this CTA's Y half
        const int g = warp & 7;             // rows 8g .. 8g + 7 (and + 64)
        const int kq = warp >> 3;           // components [kq * 16, kq * 16 + 16) of a stage
        const int rl = lane >> 2, quad = lane & 3;
        const int cb = kq * 16 + quad * 4;  // this thread's 4 components
        const int r0 = 8 * g + rl;          // rows r0 and r0 + 64; Y row r0 of tile r0 + 64 hcol
        const int ry = hcol;                // which of the two rows is the Y row
        // Rows of tiles beyond the array get phase 0 (bounded values, so no
        // s32 sum can overflow): their products only reach rows and columns
        // of the accumulators that the epilogue never writes out.
        double u[2], v[2], w[2];            // quarter-turns per unit l, m, n - 1
#pragma unroll
        for (int s2 = 0; s2 < 2; s2++) {
            const int r = r0 + 64 * s2;
            u[s2] = v[s2] = w[s2] = 0.0;
            if (r < P.ntiles) {
                const XYZ x = P.xyzs[r];
                const double oq = 4.0 * freq / VEL_C;
                u[s2] = (P.s_ha * x.x + P.c_ha * x.y) * oq;
                v[s2] = (-P.s_dec * P.c_ha * x.x + P.s_dec * P.s_ha * x.y + P.c_dec * x.z) * oq;
                w[s2] = (P.c_dec * P.c_ha * x.x - P.c_dec * P.s_ha * x.y + P.s_dec * x.z) * oq;
            }
        }
        const double4* lmn = P.lmn + P.c0;
        const JonesF64* Wf = P.W + (size_t)f * P.nc + P.c0;
        // the first KC threads fetch a stage's component data (zeros past the end)
        auto fetch = [&](int k, double2& a, double2& b, double2& wd) {
            const int c = k * KC + tid;
            if (c < P.cn) {
                a = __ldg(reinterpret_cast<const double2*>(lmn + c));
                b = __ldg(reinterpret_cast<const double2*>(lmn + c) + 1);
                wd = __ldg(reinterpret_cast<const double2*>(Wf + c) + wsel);
            } else {
                a = b = wd = make_double2(0.0, 0.0);
            }
        };
        auto stash = [&](int buf, const double2& a, const double2& b, const double2& wd) {
            comp_s[buf].l[tid] = a.x;
            comp_s[buf].m[tid] = a.y;
            comp_s[buf].n[tid] = b.x;
            comp_s[buf].w[tid] = make_float2((float)(wd.x * (double)sx), (float)(wd.y * (double)sx));
        };
        // Software pipeline: iteration k writes the byte planes of stage k
        // from registers and computes the values of stage k + 1 (phasors, X,
        // Y: FP64, conversion and FMA work) in the same straight-line block,
        // so the scheduler interleaves the two kinds of work instead of every
        // producer warp hitting the same pipe at once.  Component data goes
        // through a 3-deep ring: stage j in comp_s[j % 3], stashed two
        // iterations ahead, overwritten only after the barrier that follows
        // its last reader.  Stages past the end read zeros (their values are
        // never written out).
        auto compute = [&](int k, int (&xr)[2][4], int (&xi)[2][4], int (&yr)[4], int (&yi)[4], int (&yn)[4]) {
            const CompStage& cs_ = comp_s[k % CRING];
            double cl[4], cm[4], cn[4];
            float wr[4], wi[4];
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const double2 l2 = *reinterpret_cast<const double2*>(&cs_.l[cb + 2 * h]);
                const double2 m2 = *reinterpret_cast<const double2*>(&cs_.m[cb + 2 * h]);
                const double2 n2 = *reinterpret_cast<const double2*>(&cs_.n[cb + 2 * h]);
                const float4 w2 = *reinterpret_cast<const float4*>(&cs_.w[cb + 2 * h]);
                cl[2 * h] = l2.x, cl[2 * h + 1] = l2.y;
                cm[2 * h] = m2.x, cm[2 * h + 1] = m2.y;
                cn[2 * h] = n2.x, cn[2 * h + 1] = n2.y;
                wr[2 * h] = w2.x, wi[2 * h] = w2.y, wr[2 * h + 1] = w2.z, wi[2 * h + 1] = w2.w;
            }
#pragma unroll
            for (int j = 0; j < 4; j++)
#pragma unroll
                for (int s2 = 0; s2 < 2; s2++) {
                    float sn, cs;
                    phasor_quarter_f32(u[s2] * cl[j] + v[s2] * cm[j] + w[s2] * cn[j], sn, cs);
                    const float Xr = fmaf(wr[j], cs, -wi[j] * sn);
                    const float Xi = fmaf(wr[j], sn, wi[j] * cs);
                    // x + 0x808080 (balancing offset of the three lower digits)
                    xr[s2][j] = __float2int_rn(Xr) + 0x808080;
                    xi[s2][j] = __float2int_rn(Xi) + 0x808080;
                    if (s2 == ry) {
                        // y + 0x8080 + 0x400000 in the FP32 mantissa (one rounding)
                        yr[j] = __float_as_int(__fmaf_rn(cs, SY, YOFF));
                        yi[j] = __float_as_int(__fmaf_rn(sn, SY, YOFF));
                        yn[j] = __float_as_int(__fmaf_rn(-sn, SY, YOFF));
                    }
                }
        };
        auto write_planes = [&](int st, const int (&xr)[2][4], const int (&xi)[2][4], const int (&yr)[4],
                                const int (&yi)[4], const int (&yn)[4]) {
            unsigned char* sb = smem + st * STAGE_BYTES;
            uint32_t pl[4];
            // x planes: bytes 0-2 excess-128 lower digits, byte 3 the signed top digit
#pragma unroll
            for (int s2 = 0; s2 < 2; s2++) {
                const uint32_t xo = chunk_off(r0 + 64 * s2, kq) + quad * 4;
#pragma unroll
                for (int part = 0; part < 2; part++) {
                    byte_planes4(part ? xi[s2] : xr[s2], pl);
#pragma unroll
                    for (int b = 0; b < 4; b++)
                        *reinterpret_cast<uint32_t*>(sb + x_tile(part, 3 - b) + xo) = b < 3 ? pl[b] ^ 0x80808080u : pl[b];
                }
            }
            // y planes: bytes 0-1 excess-128, byte 2 the top digit + 64
            const uint32_t yo = chunk_off(r0, kq) + quad * 4;
#pragma unroll
            for (int part = 0; part < 3; part++) {
                byte_planes4(part == 0 ? yr : (part == 1 ? yi : yn), pl);
                *reinterpret_cast<uint32_t*>(sb + y_tile(part, 2) + yo) = pl[0] ^ 0x80808080u;
                *reinterpret_cast<uint32_t*>(sb + y_tile(part, 1) + yo) = pl[1] ^ 0x80808080u;
                *reinterpret_cast<uint32_t*>(sb + y_tile(part, 0) + yo) = minus64(pl[2]);
            }
        };
        if (tid < KC) {
            double2 a, b, wd;
            fetch(0, a, b, wd);
            stash(0, a, b, wd);
            fetch(1, a, b, wd);
            stash(1, a, b, wd);
        }
        producers_sync_or(false);
        int xr[2][4], xi[2][4], yr[4], yi[4], yn[4];
        compute(0, xr, xi, yr, yi, yn);
        // The producer warps run decoupled: each thread arrives on a stage's
        // full barrier once its planes are written, a warp waits for the
        // tensor core only on the buffer it is about to overwrite, and for
        // the component data only on the ring slot it is about to read (so
        // warps may drift up to NSTAGE stages apart; the ring has room for
        // that).  Any timeout sets abort_s; the others leave at their next
        // stage or their own bounded wait.
        static_assert(KC == 32, "warp 0 stashes the component data");
        for (int k = 0; k < nchunks; k++) {
            const int st = k % NSTAGE;
            double2 na, nb, nw;  // stage k + 2's component data, in flight during this stage
            const bool pre = tid < KC;
            if (pre) fetch(k + 2, na, nb, nw);
            if (k >= NSTAGE && !__all_sync(0xffffffffu, mbar_wait_bounded(&empty_bar[st], ((k / NSTAGE) - 1) & 1, P.err))) {
                abort_s = 1;
                break;
            }
            int nxr[2][4], nxi[2][4], nyr[4], nyi[4], nyn[4];
            write_planes(st, xr, xi, yr, yi, yn);
            // stage k + 1's component data: stages 0 and 1 were published by
            // the barrier above, later ones by warp 0 in its iteration k - 1
            if (k + 1 >= 2 && !__all_sync(0xffffffffu, mbar_wait_bounded(&comp_bar[(k + 1) % CRING],
                                                                           ((k - 1) / CRING) & 1, P.err))) {
                abort_s = 1;
                break;
            }
            compute(k + 1, nxr, nxi, nyr, nyi, nyn);
            fence_proxy_async_smem();  // make the generic-proxy stores visible to the tensor core
            if (pre) stash((k + 2) % CRING, na, nb, nw);
            __syncwarp();  // the lanes' stores and fences before the warp's one arrival
            if (lane == 0) {
                mbar_arrive(&full_bar[st]);
                if (pre) mbar_arrive(&comp_bar[(k + 2) % CRING]);
            }
            if (abort_s != 0) break;
#pragma unroll
            for (int j = 0; j < 4; j++) {
                xr[0][j] = nxr[0][j], xr[1][j] = nxr[1][j], xi[0][j] = nxi[0][j], xi[1][j] = nxi[1][j];
                yr[j] = nyr[j], yi[j] = nyi[j], yn[j] = nyn[j];
            }
        }
    } else {
        // ------------------------------------------------ MMA issuer (one thread)
        if (lane == 0) {
            const uint32_t sbase = smem_u32(smem);
            const uint32_t id = idesc_s8();
            for (int k = 0; k < nchunks; k++) {
                const int st = k % NSTAGE;
                const bool ok = mbar_wait_bounded(&full_bar[st], (k / NSTAGE) & 1, P.err);
                if (!ok) {
                    abort_s = 1;
                    break;
                }
                tc_fence_after();
                // straight-line issue: one base descriptor per stage plus
                // compile-time tile offsets (in 16-byte units, the
                // descriptor's address field); the first product of each
                // class in the launch's first stage overwrites its accumulator
                const uint64_t d0 = smem_desc(sbase + st * STAGE_BYTES);
                const uint32_t acc0 = k > 0 ? 1u : 0u;
#pragma unroll
                for (int i = 0; i < XDIG; i++)
#pragma unroll
                    for (int j = 0; j < YDIG; j++) {
                        const int cls = i + j;
                        if (cls > 3) continue;
                        const bool first = (i == 0) || (i == 1 && j == 2);
                        // [Re | Im] += Xr [Yr; -Yi]^T + Xi [Yi; Yr]^T
                        mma_i8(tmem + acc_col(cls), d0 + (x_tile(0, i) >> 4), d0 + (y_tile(0, j) >> 4), id,
                               first ? acc0 : 1u);
                        mma_i8(tmem + acc_col(cls), d0 + (x_tile(1, i) >> 4), d0 + (y_tile(1, j) >> 4), id, 1u);
                    }
                mma_commit(&empty_bar[st]);  // stage free once these MMAs have read it
            }
            mma_commit(&done_bar);
        }
    }

    // ---------------------------------------------------- epilogue
    __syncthreads();
    const bool aborted = abort_s != 0;
    const bool ok = mbar_wait_bounded(&done_bar, 0, P.err);
    tc_fence_after();
    if (!aborted && ok && warp < NPW && nchunks > 0) {
        const int lg = warp & 3;       // TMEM lane group this warp may access
        const int cq = warp >> 2;      // quarter of the NH columns
        const int p = lg * 32 + lane;  // row: tile p
        const uint32_t lane_addr = tmem + ((uint32_t)(lg * 32) << 16);
        const int n = P.ntiles;
        for (int c0 = cq * (NH / 4); c0 < cq * (NH / 4) + NH / 4; c0 += 8) {
            int a[8][8];  // [class * 2 + re/im][column]
#pragma unroll
            for (int g = 0; g < 8; g++)  // g = class * 2 + (0 Re, 1 Im)
                tmem_ld8(lane_addr + acc_col(g >> 1) + (uint32_t)((g & 1) * NH + c0), a[g]);
            tmem_wait_ld();
            if (p >= n) continue;
#pragma unroll
            for (int j = 0; j < 8; j++) {
                const int q = hcol * NH + c0 + j;
                if (q == p || q >= n) continue;
                if (pol < 2 && q < p) continue;
                double re = 0.0, im = 0.0;
#pragma unroll
                for (int cls = 0; cls < 4; cls++) {
                    const double wgt = ldexp(1.0, 40 - 8 * cls);
                    re += (double)a[cls * 2][j] * wgt;
                    im += (double)a[cls * 2 + 1][j] * wgt;
                }
                re *= inv;
                im *= inv;
                const bool upper = q > p;
                const size_t o = (size_t)f * P.nbl + (upper ? baseline_index(p, q, n) : baseline_index(q, p, n));
                // XY(p, q) for q > p; YX(q, p) = conj(XY(p, q)) for q < p
                const int slot = pol == 0 ? 0 : (pol == 1 ? 3 : (upper ? 1 : 2));
                if (!upper) im = -im;
                if (OUT64) {
                    double2* vp = reinterpret_cast<double2*>(reinterpret_cast<JonesF64*>(P.vis) + o) + slot;
                    double2 cur = *vp;
                    cur.x += re;
                    cur.y += im;
                    *vp = cur;
                } else {
                    float2* vp = reinterpret_cast<float2*>(reinterpret_cast<JonesF32*>(P.vis) + o) + slot;
                    float2 cur = *vp;
                    cur.x += (float)re;
                    cur.y += (float)im;
                    *vp = cur;
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
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
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
        HDC_CUDA_RET_INT(cudaFuncSetAttribute(tc::gram_i8_kernel<false>,
                                              cudaFuncAttributeMaxDynamicSharedMemorySize, tc::SMEM_BYTES));
        HDC_CUDA_RET_INT(cudaFuncSetAttribute(tc::gram_i8_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              tc::SMEM_BYTES));
        tc->configured = true;
    }
    return HDC_OK;
}

// The tensor-core point predict of one timestep over device tables: lmn
// [nc] (turns), W [nf][nc] (B S B^H of a beam shared by all tiles), tile
// XYZs, hour angle and declination of the phase centre; accumulates into
// vis [nf][nbl] (JonesF32, or JonesF64 with out64).
int launch_tensor_points(int nf, int nbl, int ntiles, int nc, const double* d_freqs, const XYZ* d_xyzs, double ha,
                         double dec, const double4* d_lmn, const JonesF64* d_W, void* d_vis, bool out64, int* d_err,
                         cudaStream_t s) {
    if (nc == 0) return HDC_OK;
    if (ntiles > tc::NT) {
        set_error("the tensor-core predict supports up to %d tiles (have %d)", tc::NT, ntiles);
        return HDC_ERR_UNSUPPORTED;
    }
    static std::once_flag once;
    static cudaError_t attr_err = cudaSuccess;
    std::call_once(once, [] {
        attr_err = cudaFuncSetAttribute(tc::gram_i8_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        tc::SMEM_BYTES);
        if (attr_err == cudaSuccess)
            attr_err = cudaFuncSetAttribute(tc::gram_i8_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            tc::SMEM_BYTES);
    });
    HDC_CUDA_RET_INT(attr_err);
    tc::Params P;
    P.nf = nf;
    P.nbl = nbl;
    P.ntiles = ntiles;
    P.nc = nc;
    P.freqs = d_freqs;
    P.xyzs = d_xyzs;
    P.s_ha = std::sin(ha);
    P.c_ha = std::cos(ha);
    P.s_dec = std::sin(dec);
    P.c_dec = std::cos(dec);
    P.lmn = d_lmn;
    P.W = d_W;
    P.vis = d_vis;
    P.err = d_err;
    // passes of at most KPASS components accumulate into the visibilities in turn
    const dim3 grid(nf, 3, (ntiles + tc::NH - 1) / tc::NH);
    for (int c0 = 0; c0 < P.nc; c0 += tc::KPASS) {
        P.c0 = c0;
        P.cn = std::min(tc::KPASS, P.nc - c0);
        if (out64)
            tc::gram_i8_kernel<true><<<grid, tc::THREADS, tc::SMEM_BYTES, s>>>(P);
        else
            tc::gram_i8_kernel<false><<<grid, tc::THREADS, tc::SMEM_BYTES, s>>>(P);
        count_launches(1);
        HDC_CUDA_RET_INT(cudaGetLastError());
    }
    return HDC_OK;
}

int Modeller::tensor_points(double lst, void* d_vis, bool out64, cudaStream_t s) {
    if (t[0].nc == 0) return HDC_OK;
    return launch_tensor_points(nf, nbl, ntiles, t[0].nc, d_freqs, d_xyzs, lst - pc.ra, pc.dec, t[0].d_lmn,
                                weights(0), d_vis, out64, d_err, s);
}

void Modeller::tensor_release() {
    delete tc;
    tc = nullptr;
}

}  // namespace hdc
