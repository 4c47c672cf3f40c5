// Tensor-core factored point-source predict (tcgen05, sm_100a), exact
// integer accumulation.
//
// For one timestep and channel the baseline UVW is a tile difference
// (uvw_pq = uvw_p - uvw_q, as marlu's xyzs_to_cross_uvws builds it), so the
// point-source phasor factors: exp(2 pi i theta_pq,c) = A_pc conj(A_qc) with
// A_pc = exp(2 pi i (u_p l_c + v_p m_c + w_p (n_c - 1)) f / c).
//
// Shared beam (MODE 2, the table form).  Each polarisation ab of the
// visibility matrix is a weighted Gram product
//     V^ab = A (A diag(conj W^ab))^H       (tiles x tiles, over components)
// with W = B S B^H the per-component brightness.  W is Hermitian, so
// V^YX = (V^XY)^H and V^XX, V^YY are Hermitian: three complex products give
// all four correlations of every baseline.  The left operand A is the same
// for every polarisation and column block, so its digit planes (and the
// FP32 phasors the right operand is formed from) are computed once per
// (channel, stage of 32 components) into a table in device memory, which
// the Gram CTAs read with bulk copies (TMA) and L2 loads.
//
// Per-tile beams (MODE 1), the block form: with B_pc the beam of tile p
// towards component c and S_c its instrumental flux,
//     V^ab_pq = sum_{c, y} M^a_{p,(c,y)} conj(N^b_{q,(c,y)}),
//     M^a_{p,(c,y)} = A_pc (B_pc S_c)^{ay},   N^b_{q,(c,y)} = A_qc B_qc^{by},
// a Gram product over K = 2 x components (y the second index of S); again
// XX, YY and XY suffice (S Hermitian: V^YX_pq = conj(V^XY_qp)).  Both
// operands carry the beam, so they are formed in the Gram CTA itself.
//
// With X the left and Y the right operand, in real form
//     Re V = Xr Yr^T + Xi Yi^T,   Im V = Xi Yr^T + Xr (-Yi)^T.
//
// Numbers.  A tensor core accumulating in FP32 does not round to nearest, and
// its error grows with every K step.  Here every operand is instead a
// fixed-point integer split into balanced byte digits, and the digit planes
// are multiplied on the integer tensor core (kind::i8, s8 x s8, s32
// accumulators), where every sum is exact:
//   an operand with dynamic range (A conj(W) in MODE 2, M and N in MODE 1):
//       x = rint(X sx), |x| < 2^31 - 2^24 (sx from the channel's largest |X|),
//       x = d0 2^24 + d1 2^16 + d2 2^8 + d3, every d_i in [-128, 127];
//   the unit phasor A (MODE 2): y = rint(A sy), |y| < 2^22,
//       y = e0 2^16 + e1 2^8 + e2.
// Balanced digits are the bytes of (x + 0x808080) ^ 0x808080: adding 128 to
// each lower digit position and flipping its top bit turns excess-128 bytes
// into two's-complement ones (the flip is applied to four digits of a byte
// plane at once).  They have zero mean, so the products left out below do
// not bias the sum.  x y = sum_ij d_i e_j 2^(XW + YW - 8(i + j)); the plane
// products with i + j <= 3 are kept (9 in MODE 2, 10 in MODE 1; the rest
// weigh < 2^-30 of full scale), each into the accumulator of its class
// w = i + j, and the epilogue forms V = sum_w D_w 2^(XW + YW - 8w) / (sx sy)
// in FP64.  The only rounding is in the inputs: the phase, reduced exactly
// in FP64 to a quadrant q and a remainder r in [-1/2, 1/2] quarter-turns;
// sin and cos of (pi/2) r from FP32 polynomials (least-squares fits,
// mwa_hyperdrive_b200/phasor_poly.py, < 0.75 ulp); the operands formed in
// FP32; the roundings to integers.  A launch covers at most KPASS
// components, so no s32 sum can overflow.
//
// Kernel: one CTA per job = (channel, polarisation, row block of 128 tiles,
// column block of 64 tiles); the jobs of a channel are the blocks that hold a
// baseline of that polarisation (XX, YY: some p < q; XY: all), so any number
// of tiles is covered.  M = 128 tiles (rows of X), 64 tile columns (rows of
// Y), K = 32 bytes per stage (32 components, or 16 components x 2 in MODE
// 1).  MODE 2: a copy warp brings each stage's A planes from the table
// (one bulk copy, prefetched into L2 eight stages ahead) and sixteen
// producer warps form Y = A conj(W) sx from the table's phasors and weights
// and write its byte planes.  MODE 1: the sixteen producer warps compute
// the phasors, beams, X and Y and write all planes.  Planes are in the
// K-major no-swizzle core-matrix layout (one warp store = one 128-byte core
// matrix).  One thread issues the MMAs of a stage (plane pairs x {Xr, Xi},
// N = 128 = [Re | Im] of the 64 columns) into 4 TMEM accumulators (one per
// class, 128 columns each = all 512 columns).  The epilogue reads TMEM with
// tcgen05.ld, combines the classes in FP64 and stores each of its baselines'
// values once into a planar scratch [XX, XY, YX, YY][channel][baseline] (XY
// of p < q as XY, of p > q as YX = conj); a coalesced pass then adds the four
// planes into the visibilities, so every Jones matrix is read and written
// once.
//
// Every mbarrier wait is bounded by the global timer; on a timeout the CTA
// records KERR_TIMEOUT, waits (bounded) for its issued MMAs and copies and
// frees TMEM.

#include <algorithm>
#include <cmath>
#include <mutex>
#include <type_traits>
#include <vector>

#include "modeller.cuh"

namespace hdc {
namespace tc {

constexpr int NT = 128;    // rows of a block = M
constexpr int NH = 64;     // tile columns of a block
constexpr int NB = 2 * NH; // MMA N: [Re | Im] of the NH columns
constexpr int KC = 32;     // K bytes per stage = MMA K
constexpr int NPW = 16;    // producer / epilogue warps
constexpr int NPT = NPW * 32;  // producer threads
constexpr int XT_BYTES = NT * KC;  // one X plane tile, 4 KB
constexpr int YT_BYTES = NH * KC;  // one Y plane tile, 2 KB
constexpr int LBO = 128;             // bytes between the two 16-byte K core matrices of a row group
constexpr int SBO = (KC / 16) * 128; // bytes between 8-row groups
constexpr int TMEM_COLS = 512;       // 4 classes x NB
constexpr int MAXJOBS = 1024;        // jobs per channel in the launch parameters
constexpr float SY0 = 4128768.0f;    // MODE 2: 2^22 - 2^16: |A| <= 1 -> |y| < 2^22
// y + 0x8080 as FP32 bits: 1.5 * 2^23 rounds |v| < 2^22 to an integer in
// the mantissa; the extra 0x8080 is the balancing offset of the two lower
// digits.  The mantissa field then holds 2^22 + 0x8080 + y, so byte 2 is the
// top digit + 0x40 and bytes 1, 0 the excess-128 lower digits.
constexpr float YOFF = 12582912.0f + 32896.0f;
constexpr double FULL31 = 2147483648.0 - 33554432.0;  // 2^31 - 2^25

template <int MODE>
struct Cfg;
template <>
struct Cfg<1> {
    static constexpr int XDIG = 4, YDIG = 4, NSTAGE = 3, CPS = 16;  // components per stage
    static constexpr int KPASS = 8000;  // 4 products x 2 x 2^14 x 2 KPASS < 2^31
    static constexpr int THREADS = NPT + 32;  // producers + the MMA warp
};
// MODE 2 (shared beam, table form): the A operand is the phasor matrix A
// itself (3 digits, as y above), the same for every polarisation, and W
// moves to the B side: V^ab = A (A diag(conj W^ab))^H.  The A planes and
// the FP32 phasors come from a table written once per (channel, stage).
template <>
struct Cfg<2> {
    static constexpr int XDIG = 3, YDIG = 4, NSTAGE = 4, CPS = 32;
    static constexpr int KPASS = 16384;  // 3 products x 2 x 2^14 x KPASS < 2^31
    static constexpr int THREADS = NPT + 64;  // producers + the MMA warp + the copy warp
};
// Table of one (channel, stage): the A planes of each row block ([re, im]
// x 3 digits in the shared-memory layout, 24 KB), then the FP32 phasors
// (cos, sin) of each column block of 64 tiles (rows of 32 components).
constexpr int PL_BYTES = 2 * 3 * XT_BYTES;
constexpr int PH_ROW = KC * 8;
constexpr int PH_BYTES = NH * PH_ROW;
template <int MODE>
struct Lay {
    static constexpr int Y_OFF = 2 * Cfg<MODE>::XDIG * XT_BYTES;                     // X: [re, im][digits]
    static constexpr int STAGE_BYTES = Y_OFF + 3 * Cfg<MODE>::YDIG * YT_BYTES;       // Y: [im, re, -im][digits]
    static constexpr int SMEM_BYTES = Cfg<MODE>::NSTAGE * STAGE_BYTES + 1024;
    static constexpr int CRING = Cfg<MODE>::NSTAGE + 2;  // component ring: warps may be NSTAGE stages apart
};
static_assert(Lay<2>::SMEM_BYTES <= 220 * 1024, "MODE 2 stages exceed shared memory");
static_assert(Lay<2>::STAGE_BYTES % 16 == 0 && PH_ROW % 16 == 0, "bulk copies need 16-byte alignment");
constexpr int PF_STAGES = 8;  // MODE 2: table blocks are prefetched into L2 this many stages ahead

// MODE 1 component data of one stage, staged in shared memory (structure
// of arrays so that 16-byte loads of consecutive components are
// conflict-free)
struct CompStage1 {
    double l[16], m[16], n[16];  // turn units (n - 1 in n)
    float4 s[16][2];             // S (xx, xy | yx, yy as re, im) of this channel
};

struct Params {
    int nf, nbl, ntiles, nc, c0, cn;
    const double* freqs;
    const XYZ* xyzs;
    double s_ha, c_ha, s_dec, c_dec;
    const double4* lmn;    // [nc] turn units
    const JonesF64* W;     // [nf][nc]: MODE 2 B S B^H (or S), MODE 1 S
    // MODE 1: beam [uniq tile][uniq freq][nc], unique row of each tile and
    // column of each channel, and per channel bounds of |B| and |S| entries
    const JonesF64* beam;
    const JonesF32* beam32;  // MODE 1: the beam table in FP32, or NULL (then read from beam)
    const int* tile_map;
    const int* freq_map;
    int n_uniq_freq;
    const double* maxb;
    const double* maxs;
    void* planes;          // [4][nf][nbl] float2 (or double2 with OUT64)
    int* err;
    // MODE 2: channels f0 + blockIdx.y; the table of channel f0 + i at
    // table + i * tab_chan, its stage k at + k * tab_block (row-block planes
    // first, the column-block phasors from tab_ph_off)
    int f0;
    const unsigned char* table;
    size_t tab_chan, tab_block, tab_ph_off;
    // per channel after its stages: W sx of each polarisation (XX, YY, XY)
    // [3][stages x 32] float2, then the three bounds max |W| (double)
    size_t tab_w_off, tab_bound_off;
    int ncb;
    int njobs;
    uint32_t jobs[MAXJOBS];  // pol | rb << 8 | cb << 20
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
template <int MODE>
__device__ __forceinline__ uint32_t x_tile(int part, int digit) {
    return (uint32_t)((part * Cfg<MODE>::XDIG + digit) * XT_BYTES);
}
// Y tiles of one digit lie in the order [Yi | Yr | -Yi] (64 rows each), so
// that [Yr; -Yi] (from the Yr tile) and [Yi; Yr] (from the Yi tile) are
// 128-row B operands: Xr [Yr; -Yi]^T + Xi [Yi; Yr]^T = [Re | Im] of X Y^H.
// part: 0 = Yr, 1 = Yi, 2 = -Yi
template <int MODE>
__device__ __forceinline__ uint32_t y_tile(int part, int digit) {
    const int slot = part == 0 ? 1 : (part == 1 ? 0 : 2);
    return (uint32_t)(Lay<MODE>::Y_OFF + (digit * 3 + slot) * YT_BYTES);
}
// TMEM column of accumulator class w ([Re | Im], NB columns)
__device__ __forceinline__ uint32_t acc_col(int w) { return (uint32_t)(w * NB); }

// The tile's position in quarter-turns per unit l, m, n - 1 at this channel
// (zero for rows beyond the array: bounded values, never written out).
__device__ __forceinline__ void tile_uvw(const Params& P, int tile, double oq, double& u, double& v, double& w) {
    u = v = w = 0.0;
    if (tile < P.ntiles) {
        const XYZ x = P.xyzs[tile];
        u = (P.s_ha * x.x + P.c_ha * x.y) * oq;
        v = (-P.s_dec * P.c_ha * x.x + P.s_dec * P.s_ha * x.y + P.c_dec * x.z) * oq;
        w = (P.c_dec * P.c_ha * x.x - P.c_dec * P.s_ha * x.y + P.s_dec * x.z) * oq;
    }
}

// the beam table row of a tile (its unique tile at unique frequency column
// fm: unique tile x unique frequencies + fm), looked up once per thread; -1
// past the array
__device__ __forceinline__ int beam_base(const Params& P, int tile, int fm) {
    if (tile >= P.ntiles) return -1;
    return __ldg(P.tile_map + tile) * P.n_uniq_freq + fm;
}

// one row of a beam Jones (two complex numbers, FP32): component c of the
// pass in beam table row `base`
__device__ __forceinline__ float4 beam_row(const Params& P, int base, int c, int row) {
    if (base < 0) return make_float4(0.f, 0.f, 0.f, 0.f);
    if (P.beam32) return __ldg(reinterpret_cast<const float4*>(P.beam32 + (size_t)base * P.nc + P.c0 + c) + row);
    const double2* b = reinterpret_cast<const double2*>(P.beam + (size_t)base * P.nc + P.c0 + c) + 2 * row;
    const double2 e0 = __ldg(b), e1 = __ldg(b + 1);
    return make_float4((float)e0.x, (float)e0.y, (float)e1.x, (float)e1.y);
}

template <int MODE, bool OUT64>
__global__ void __launch_bounds__(Cfg<MODE>::THREADS, 1) gram_i8_kernel(const __grid_constant__ Params P) {
    using C = Cfg<MODE>;
    using L = Lay<MODE>;
    constexpr int NSTAGE = C::NSTAGE;
    constexpr int CRING = L::CRING;
    constexpr int NTHR = C::THREADS;
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    __shared__ alignas(8) uint64_t full_bar[NSTAGE], empty_bar[NSTAGE], done_bar;
    __shared__ alignas(8) uint64_t copy_bar[NSTAGE];  // MODE 2: the stage's A planes have landed
    __shared__ uint32_t tmem_base_s;
    __shared__ volatile int abort_s;
    // MODE 1: the ring of component data
    __shared__ __align__(16) CompStage1 comp_s[MODE == 1 ? CRING : 1];
    __shared__ alignas(8) uint64_t comp_bar[MODE == 1 ? CRING : 1];

    unsigned char* smem = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    const int f = P.f0 + blockIdx.y;  // channel (planes, W, frequency)
    const uint32_t job = P.jobs[blockIdx.x];
    const int pol = (int)(job & 0xFF);          // 0: XX, 1: YY, 2: XY
    const int rb = (int)((job >> 8) & 0xFFF);   // rows: tiles [128 rb, 128 rb + 128)
    const int cb = (int)(job >> 20);            // columns: tiles [64 cb, 64 cb + 64)
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int arow = pol == 1 ? 1 : 0, brow = pol == 0 ? 0 : 1;  // MODE 1: beam rows a (of M) and b (of N)

    // operand scales: MODE 2 from the pass's largest |W| of this
    // polarisation (in the table); MODE 1 from the channel's bounds
    // |M| <= 2 max|B| max|S| and |N| <= max|B|
    if (tid == 0) {
        for (int s = 0; s < NSTAGE; s++) {
            mbar_init(&full_bar[s], NPW);  // one arrival per producer warp
            mbar_init(&empty_bar[s], 1);
        }
        if (MODE == 1)
            for (int s = 0; s < CRING; s++) mbar_init(&comp_bar[s], 1);  // the stashing warp arrives once
        if (MODE == 2)
            for (int s = 0; s < NSTAGE; s++) mbar_init(&copy_bar[s], 1);  // the copy thread's expect_tx
        mbar_init(&done_bar, 1);
        abort_s = 0;
        fence_barrier_init();
    }
    __syncthreads();
    double bound, bmax = 1.0;
    if (MODE == 2) {
        bound = reinterpret_cast<const double*>(P.table + (size_t)blockIdx.y * P.tab_chan + P.tab_bound_off)[pol];
    } else {
        bmax = P.maxb[f];
        bound = 2.0 * bmax * P.maxs[f];
    }
    const int n = P.ntiles;
    // A polarisation whose weights are all exactly zero (e.g. XY of a
    // Stokes-I sky) contributes exactly zero: its baselines get zeros.
    const bool zero = !(bound > 0.0);
    const float sx = zero ? 0.f : (float)(FULL31 / bound);
    const float sy = MODE == 2 ? SY0 : (zero ? 0.f : (float)(FULL31 / bmax));
    const double inv = zero ? 0.0 : 1.0 / ((double)sx * (double)sy);
    const int nchunks = zero ? 0 : (P.cn + C::CPS - 1) / C::CPS;

    if (!zero && warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base_s)),
                     "r"(TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_base_s;
    const double freq = P.freqs[f];
    const int fm = MODE == 1 ? __ldg(P.freq_map + f) : 0;

    if (zero) {
        // nothing to multiply
    } else if (warp < NPW) {
        // ------------------------------------------------ producers
        if constexpr (MODE == 2) {
            // Table form: warp (g, kq), lane (rl, quad) forms the B operand
            // of column-block row r = 8 g + rl for the stage's components
            // 16 kq + 4 quad .. + 3, Y = A_qc conj(W_c) sx in 4 digits, from
            // the table's FP32 phasors (read from L2 into registers one stage
            // ahead; the copy warp prefetches them into L2).
            const int g = warp & 7, kq = warp >> 3, rl = lane >> 2, quad = lane & 3;
            const int r = 8 * g + rl;
            const int cl0 = kq * 16 + quad * 4;
            const uint32_t yo = chunk_off(r, kq) + quad * 4;
            const unsigned char* tch = P.table + (size_t)blockIdx.y * P.tab_chan;
            const unsigned char* phq = tch + P.tab_ph_off + (size_t)cb * PH_BYTES + r * PH_ROW + cl0 * 8;
            const float2* wq = reinterpret_cast<const float2*>(tch + P.tab_w_off) + (size_t)pol * nchunks * KC + cl0;
            // stage k's phasors and W sx of this thread's four components
            // (the copy warp prefetches the phasor blocks into L2; past the
            // end: zeros)
            auto load_ph = [&](int k, float4& x, float4& y, float4& u, float4& v) {
                if (k < nchunks) {
                    const float4* q = reinterpret_cast<const float4*>(phq + (size_t)k * P.tab_block);
                    x = __ldg(q);
                    y = __ldg(q + 1);
                    const float4* wv = reinterpret_cast<const float4*>(wq + (size_t)k * KC);
                    u = __ldg(wv);
                    v = __ldg(wv + 1);
                } else {
                    x = y = u = v = make_float4(0.f, 0.f, 0.f, 0.f);
                }
            };
            // one lane polls a barrier for its warp; the others follow it
            // past __syncwarp
            auto warp_wait = [&](uint64_t* bar, uint32_t parity) {
                int ok = 1;
                if (lane == 0) ok = mbar_wait_sleep(bar, parity, P.err);
                ok = __shfl_sync(0xffffffffu, ok, 0);
                __syncwarp();
                return ok != 0;
            };
            float4 a01, a23, w01, w23;
            load_ph(0, a01, a23, w01, w23);
            for (int k = 0; k < nchunks; k++) {
                const int st = k % NSTAGE;
                float4 n01, n23, m01, m23;
                load_ph(k + 1, n01, n23, m01, m23);  // stage k + 1's inputs, in flight during this stage
                const float ac[4] = {a01.x, a01.z, a23.x, a23.z}, as[4] = {a01.y, a01.w, a23.y, a23.w};
                const float wr[4] = {w01.x, w01.z, w23.x, w23.z}, wi[4] = {w01.y, w01.w, w23.y, w23.w};
                int yv[3][4];  // Yr, Yi, -Yi (+ 0x808080, the balancing offset of the three lower digits)
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    const int ir = __float2int_rn(fmaf(wr[j], ac[j], wi[j] * as[j]));
                    const int ii = __float2int_rn(fmaf(wr[j], as[j], -(wi[j] * ac[j])));
                    yv[0][j] = ir + 0x808080;
                    yv[1][j] = ii + 0x808080;
                    yv[2][j] = -ii + 0x808080;
                }
                // the stage buffer's B planes are free once the tensor core
                // is done with stage k - NSTAGE
                if (k >= NSTAGE && !warp_wait(&empty_bar[st], ((k / NSTAGE) - 1) & 1)) {
                    abort_s = 1;
                    break;
                }
                unsigned char* sb = smem + st * L::STAGE_BYTES;
                uint32_t pl[4];
#pragma unroll
                for (int part = 0; part < 3; part++) {
                    byte_planes4(yv[part], pl);
                    // bytes 0-2 excess-128 lower digits, byte 3 the signed top digit
#pragma unroll
                    for (int b = 0; b < 4; b++)
                        *reinterpret_cast<uint32_t*>(sb + y_tile<MODE>(part, 3 - b) + yo) =
                            b < 3 ? pl[b] ^ 0x80808080u : pl[b];
                }
                fence_proxy_async_smem();  // make the generic-proxy stores visible to the tensor core
                __syncwarp();
                if (lane == 0) mbar_arrive(&full_bar[st]);
                if (abort_s != 0) break;
                a01 = n01;
                a23 = n23;
                w01 = m01;
                w23 = m23;
            }
        } else {
        // warp = 8 tile rows x 16 K bytes of a stage; lane = (row rl, quad of
        // 4 K bytes), and every thread also takes the row 64 tiles down, so a
        // warp's store of one byte plane is one whole 128-byte core matrix.
        // Its Y row is column r0 of the column block: one of its two X rows
        // when the column block lies inside the row block, else a third tile.
        const int g = warp & 7;             // rows 8g .. 8g + 7 (and + 64)
        const int kq = warp >> 3;           // K bytes [kq * 16, kq * 16 + 16) of a stage
        const int rl = lane >> 2, quad = lane & 3;
        const int r0 = 8 * g + rl;          // rows r0 and r0 + 64 of the block
        const int ry = cb - 2 * rb;         // the X row that is the Y tile (0 or 1), else separate
        const bool ysep = ry != 0 && ry != 1;
        const int prow[2] = {NT * rb + r0, NT * rb + r0 + 64};
        const int qcol = NH * cb + r0;
        // the three tiles' beam row blocks (MODE 1), looked up once
        const int bbase[3] = {MODE == 1 ? beam_base(P, prow[0], fm) : -1, MODE == 1 ? beam_base(P, prow[1], fm) : -1,
                              MODE == 1 ? beam_base(P, qcol, fm) : -1};
        // The upper 64 rows of the block pair with no column of it when they
        // lie beyond the array, or in an XX / YY block whose columns all lie
        // below them: their X planes stay zero and are not produced.  (Then
        // the Y tile is never one of them: ry != 1.)
        const bool skip_hi = NT * rb + 64 >= n || (pol < 2 && NT * rb + 64 >= NH * cb + NH - 1);
        if (skip_hi) {
            for (int st = 0; st < NSTAGE; st++)
                for (int tile = 0; tile < 2 * C::XDIG; tile++) {
                    uint4* z = reinterpret_cast<uint4*>(smem + st * L::STAGE_BYTES + tile * XT_BYTES + XT_BYTES / 2);
                    for (int i = tid; i < XT_BYTES / 32; i += NPT) z[i] = make_uint4(0u, 0u, 0u, 0u);
                }
        }
        const double oq = 4.0 * freq / VEL_C;
        double u[3], v[3], w[3];  // quarter-turns per unit l, m, n - 1 of the two X rows and the Y tile
        tile_uvw(P, prow[0], oq, u[0], v[0], w[0]);
        tile_uvw(P, prow[1], oq, u[1], v[1], w[1]);
        tile_uvw(P, qcol, oq, u[2], v[2], w[2]);
        const double4* lmn = P.lmn + P.c0;
        const JonesF64* Wf = P.W + (size_t)f * P.nc + P.c0;
        // the first CPS threads fetch a stage's component data (zeros past the end)
        auto fetch = [&](int k, double2& a, double2& b) {
            const int c = k * C::CPS + tid;
            if (c < P.cn) {
                a = __ldg(reinterpret_cast<const double2*>(lmn + c));
                b = __ldg(reinterpret_cast<const double2*>(lmn + c) + 1);
            } else {
                a = b = make_double2(0.0, 0.0);
            }
        };
        // S is read at stash time
        auto stash = [&](int k, int buf, const double2& a, const double2& b) {
            CompStage1& cs = comp_s[buf];
            cs.l[tid] = a.x;
            cs.m[tid] = a.y;
            cs.n[tid] = b.x;
            const int c = k * C::CPS + tid;
            float4 s0 = make_float4(0.f, 0.f, 0.f, 0.f), s1 = s0;
            if (c < P.cn) {
                const double2* sp = reinterpret_cast<const double2*>(Wf + c);
                const double2 xx = __ldg(sp), xy = __ldg(sp + 1), yx = __ldg(sp + 2), yy = __ldg(sp + 3);
                s0 = make_float4((float)xx.x, (float)xx.y, (float)xy.x, (float)xy.y);
                s1 = make_float4((float)yx.x, (float)yx.y, (float)yy.x, (float)yy.y);
            }
            cs.s[tid][0] = s0;
            cs.s[tid][1] = s1;
        };
        // Software pipeline: iteration k writes the byte planes of stage k
        // from registers and computes the values of stage k + 1 in the same
        // straight-line block.  Component data goes through a ring of CRING
        // slots, stashed two stages ahead by the first CPS threads.  Stages
        // past the end read zeros (their values are never written out).
        // compute and write_planes take SKIP (skip_hi) as a compile-time
        // constant, so the two rows' work stays one straight-line block
        auto compute = [&](auto skip_c, int k, int (&xr)[2][4], int (&xi)[2][4], int (&yr)[4], int (&yi)[4],
                           int (&yn)[4]) {
            constexpr bool SKIP = decltype(skip_c)::value;
            const CompStage1& cs_ = comp_s[k % CRING];
            {
                // K bytes 4 quad .. 4 quad + 3 of this warp's 16 = components
                // c0l, c0l + 1 (stage-local) x y in {X, Y}
                const int c0l = kq * 8 + quad * 2;
                const int cg = k * C::CPS + c0l;  // component of the pass
#pragma unroll
                for (int j = 0; j < 2; j++) {
                    const int c = cg + j < P.cn ? cg + j : 0;  // past the end: bounded values, zero S
                    const double cl = cs_.l[c0l + j], cm = cs_.m[c0l + j], cn = cs_.n[c0l + j];
                    const float4 s0 = cs_.s[c0l + j][0], s1 = cs_.s[c0l + j][1];
                    float snq = 0.f, csq = 0.f;
#pragma unroll
                    for (int s2 = 0; s2 < 2; s2++) {
                        if (SKIP && s2 == 1) continue;
                        float sn, cs;
                        phasor_quarter_f32(u[s2] * cl + v[s2] * cm + w[s2] * cn, sn, cs);
                        if (s2 == ry) snq = sn, csq = cs;
                        // (B S)^{a y} = B^{aX} S^{Xy} + B^{aY} S^{Yy}, then times A
                        const float4 b = beam_row(P, bbase[s2], c, arow);  // (B^{aX}, B^{aY}) as re, im
#pragma unroll
                        for (int y = 0; y < 2; y++) {
                            // S^{Xy}: s0 (y = 0: xx, y = 1: xy); S^{Yy}: s1 (yx, yy)
                            const float sxr = y ? s0.z : s0.x, sxi = y ? s0.w : s0.y;
                            const float syr = y ? s1.z : s1.x, syi = y ? s1.w : s1.y;
                            const float tr = b.x * sxr - b.y * sxi + b.z * syr - b.w * syi;
                            const float ti = b.x * sxi + b.y * sxr + b.z * syi + b.w * syr;
                            const float Xr = fmaf(tr, cs, -ti * sn) * sx;
                            const float Xi = fmaf(tr, sn, ti * cs) * sx;
                            xr[s2][2 * j + y] = __float2int_rn(Xr) + 0x808080;
                            xi[s2][2 * j + y] = __float2int_rn(Xi) + 0x808080;
                        }
                    }
                    if (ysep) phasor_quarter_f32(u[2] * cl + v[2] * cm + w[2] * cn, snq, csq);
                    const float4 bq = beam_row(P, bbase[2], c, brow);
#pragma unroll
                    for (int y = 0; y < 2; y++) {
                        const float br = y ? bq.z : bq.x, bi = y ? bq.w : bq.y;
                        const float Yr = fmaf(br, csq, -bi * snq) * sy;
                        const float Yi = fmaf(br, snq, bi * csq) * sy;
                        const int ir = __float2int_rn(Yr), ii = __float2int_rn(Yi);
                        yr[2 * j + y] = ir + 0x808080;
                        yi[2 * j + y] = ii + 0x808080;
                        yn[2 * j + y] = -ii + 0x808080;
                    }
                }
            }
        };
        auto write_planes = [&](auto skip_c, int st, const int (&xr)[2][4], const int (&xi)[2][4], const int (&yr)[4],
                                const int (&yi)[4], const int (&yn)[4]) {
            constexpr bool SKIP = decltype(skip_c)::value;
            unsigned char* sb = smem + st * L::STAGE_BYTES;
            uint32_t pl[4];
            // x planes: bytes 0-2 excess-128 lower digits, byte 3 the signed top digit
#pragma unroll
            for (int s2 = 0; s2 < 2; s2++) {
                if (SKIP && s2 == 1) continue;
                const uint32_t xo = chunk_off(r0 + 64 * s2, kq) + quad * 4;
#pragma unroll
                for (int part = 0; part < 2; part++) {
                    byte_planes4(part ? xi[s2] : xr[s2], pl);
#pragma unroll
                    for (int b = 0; b < 4; b++)
                        *reinterpret_cast<uint32_t*>(sb + x_tile<MODE>(part, 3 - b) + xo) =
                            b < 3 ? pl[b] ^ 0x80808080u : pl[b];
                }
            }
            const uint32_t yo = chunk_off(r0, kq) + quad * 4;
#pragma unroll
            for (int part = 0; part < 3; part++) {
                byte_planes4(part == 0 ? yr : (part == 1 ? yi : yn), pl);
                // as x: bytes 0-2 excess-128, byte 3 signed
#pragma unroll
                for (int b = 0; b < 4; b++)
                    *reinterpret_cast<uint32_t*>(sb + y_tile<MODE>(part, 3 - b) + yo) =
                        b < 3 ? pl[b] ^ 0x80808080u : pl[b];
            }
        };
        if (tid < C::CPS) {
            double2 a, b;
            fetch(0, a, b);
            stash(0, 0, a, b);
            fetch(1, a, b);
            stash(1, 1, a, b);
        }
        producers_sync_or(false);
        auto producer_loop = [&](auto skip_c) {
        int xr[2][4], xi[2][4], yr[4], yi[4], yn[4];
        compute(skip_c, 0, xr, xi, yr, yi, yn);
        // The producer warps run decoupled: each warp arrives on a stage's
        // full barrier once its planes are written, waits for the tensor
        // core only on the buffer it is about to overwrite, and for the
        // component data only on the ring slot it is about to read.  Any
        // timeout sets abort_s; the others leave at their next stage or their
        // own bounded wait.
        for (int k = 0; k < nchunks; k++) {
            const int st = k % NSTAGE;
            double2 na, nb;  // stage k + 2's component data, in flight during this stage
            const bool pre = tid < C::CPS;
            if (pre) fetch(k + 2, na, nb);
            if (k >= NSTAGE &&
                !__all_sync(0xffffffffu, mbar_wait_bounded(&empty_bar[st], ((k / NSTAGE) - 1) & 1, P.err))) {
                abort_s = 1;
                break;
            }
            int nxr[2][4], nxi[2][4], nyr[4], nyi[4], nyn[4];
            write_planes(skip_c, st, xr, xi, yr, yi, yn);
            // stage k + 1's component data: stages 0 and 1 were published by
            // the barrier above, later ones by warp 0 in its iteration k - 1
            if (k + 1 >= 2 && !__all_sync(0xffffffffu, mbar_wait_bounded(&comp_bar[(k + 1) % CRING],
                                                                           ((k - 1) / CRING) & 1, P.err))) {
                abort_s = 1;
                break;
            }
            compute(skip_c, k + 1, nxr, nxi, nyr, nyi, nyn);
            fence_proxy_async_smem();  // make the generic-proxy stores visible to the tensor core
            if (pre) stash(k + 2, (k + 2) % CRING, na, nb);
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
        };
        if (skip_hi)
            producer_loop(std::true_type{});
        else
            producer_loop(std::false_type{});
        }
    } else if (warp == NPW) {
        // ------------------------------------------------ MMA issuer (one thread)
        if (lane == 0) {
            const uint32_t sbase = smem_u32(smem);
            const uint32_t id = idesc_s8();
            for (int k = 0; k < nchunks; k++) {
                const int st = k % NSTAGE;
                bool ok = MODE == 2 ? mbar_wait_sleep(&full_bar[st], (k / NSTAGE) & 1, P.err)
                                    : mbar_wait_bounded(&full_bar[st], (k / NSTAGE) & 1, P.err);
                // MODE 2: the A planes came by bulk copy (complete before
                // the producers arrived; observed here as well)
                if (MODE == 2 && ok) ok = mbar_wait_sleep(&copy_bar[st], (k / NSTAGE) & 1, P.err);
                if (!ok) {
                    abort_s = 1;
                    break;
                }
                tc_fence_after();
                // straight-line issue: one base descriptor per stage plus
                // compile-time tile offsets (in 16-byte units, the
                // descriptor's address field); the first product of each
                // class in the launch's first stage overwrites its accumulator
                const uint64_t d0 = smem_desc(sbase + st * L::STAGE_BYTES);
                const uint32_t acc0 = k > 0 ? 1u : 0u;
#pragma unroll
                for (int i = 0; i < C::XDIG; i++)
#pragma unroll
                    for (int j = 0; j < C::YDIG; j++) {
                        const int cls = i + j;
                        if (cls > 3) continue;
                        const bool first = i == (cls - (C::YDIG - 1) > 0 ? cls - (C::YDIG - 1) : 0);
                        // [Re | Im] += Xr [Yr; -Yi]^T + Xi [Yi; Yr]^T
                        mma_i8(tmem + acc_col(cls), d0 + (x_tile<MODE>(0, i) >> 4), d0 + (y_tile<MODE>(0, j) >> 4),
                               id, first ? acc0 : 1u);
                        mma_i8(tmem + acc_col(cls), d0 + (x_tile<MODE>(1, i) >> 4), d0 + (y_tile<MODE>(1, j) >> 4),
                               id, 1u);
                    }
                mma_commit(&empty_bar[st]);  // stage free once these MMAs have read it
            }
            mma_commit(&done_bar);
        }
    } else if (MODE == 2) {
        // ------------------------------------------------ table copies (one thread)
        // Stage k's A planes (this row block) go into stage buffer k %
        // NSTAGE once the tensor core is done with stage k - NSTAGE.  The
        // A planes and the producers' phasors are prefetched into L2
        // PF_STAGES stages ahead.
        if (lane == 0) {
            const unsigned char* tch = P.table + (size_t)blockIdx.y * P.tab_chan;
            auto a_src = [&](int k) { return tch + (size_t)k * P.tab_block + (size_t)rb * PL_BYTES; };
            auto p_src = [&](int k) { return tch + (size_t)k * P.tab_block + P.tab_ph_off + (size_t)cb * PH_BYTES; };
            auto copy_a = [&](int k) {
                mbar_arrive_expect_tx(&copy_bar[k % NSTAGE], PL_BYTES);
                bulk_g2s(smem + (k % NSTAGE) * L::STAGE_BYTES, a_src(k), PL_BYTES, &copy_bar[k % NSTAGE]);
            };
            for (int k = 0; k < nchunks && k < PF_STAGES; k++) {
                prefetch_l2(a_src(k), PL_BYTES);
                prefetch_l2(p_src(k), PH_BYTES);
            }
            int na = 0;  // copies issued
            for (; na < nchunks && na < NSTAGE; na++) copy_a(na);
            for (int k = 0; na < nchunks; k++) {
                if (k + PF_STAGES < nchunks) {
                    prefetch_l2(a_src(k + PF_STAGES), PL_BYTES);
                    prefetch_l2(p_src(k + PF_STAGES), PH_BYTES);
                }
                if (!mbar_wait_sleep(&empty_bar[k % NSTAGE], (k / NSTAGE) & 1, P.err) || abort_s != 0) {
                    abort_s = 1;
                    break;
                }
                copy_a(na++);
            }
            // no copy may still be in flight when the CTA leaves: wait
            // (bounded) for the last one into each buffer
            for (int j = na > NSTAGE ? na - NSTAGE : 0; j < na; j++)
                mbar_wait_bounded(&copy_bar[j % NSTAGE], (j / NSTAGE) & 1, nullptr);
        }
    }

    // ---------------------------------------------------- epilogue
    __syncthreads();
    const bool aborted = abort_s != 0;
    const bool ok = zero || mbar_wait_sleep(&done_bar, 0, P.err);
    tc_fence_after();
    if (!aborted && ok && warp < NPW) {
        constexpr int XW = 8 * (C::XDIG - 1), YW = 8 * (C::YDIG - 1);
        const int lg = warp & 3;       // TMEM lane group this warp may access
        const int cq = warp >> 2;      // quarter of the NH columns
        const int p = NT * rb + lg * 32 + lane;  // row: tile p
        const uint32_t lane_addr = tmem + ((uint32_t)(lg * 32) << 16);
        const size_t plane = (size_t)P.nf * P.nbl;
        for (int c0 = cq * (NH / 4); c0 < cq * (NH / 4) + NH / 4; c0 += 8) {
            int a[8][8];  // [class * 2 + re/im][column]
            if (!zero) {
#pragma unroll
                for (int g = 0; g < 8; g++)  // g = class * 2 + (0 Re, 1 Im)
                    tmem_ld8(lane_addr + acc_col(g >> 1) + (uint32_t)((g & 1) * NH + c0), a[g]);
                tmem_wait_ld();
            }
            if (p >= n) continue;
#pragma unroll
            for (int j = 0; j < 8; j++) {
                const int q = NH * cb + c0 + j;
                if (q == p || q >= n) continue;
                if (pol < 2 && q < p) continue;
                double re = 0.0, im = 0.0;
                if (!zero) {
#pragma unroll
                    for (int cls = 0; cls < 4; cls++) {
                        const double wgt = ldexp(1.0, XW + YW - 8 * cls);
                        re += (double)a[cls * 2][j] * wgt;
                        im += (double)a[cls * 2 + 1][j] * wgt;
                    }
                    re *= inv;
                    im *= inv;
                }
                const bool upper = q > p;
                const size_t o = (size_t)f * P.nbl + (upper ? baseline_index(p, q, n) : baseline_index(q, p, n));
                // XY(p, q) for q > p; YX(q, p) = conj(XY(p, q)) for q < p
                const int slot = pol == 0 ? 0 : (pol == 1 ? 3 : (upper ? 1 : 2));
                if (!upper) im = -im;
                if (OUT64)
                    reinterpret_cast<double2*>(P.planes)[slot * plane + o] = make_double2(re, im);
                else
                    reinterpret_cast<float2*>(P.planes)[slot * plane + o] = make_float2((float)re, (float)im);
            }
        }
    }
    if (aborted || !ok) {
        if (tid == 0) atomicOr(P.err, KERR_TIMEOUT);
    }
    tc_fence_before();
    __syncthreads();
    if (!zero && warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
    }
}

// MODE 2 operand bounds of one pass: grid (channels of the chunk), 1024
// threads.  For each polarisation (XX, YY, XY) the pass's largest |W| (the
// operand scale sx = (2^31 - 2^25) / max |W|, as in the other forms).
constexpr int BOUND_THREADS = 1024;
__global__ void __launch_bounds__(BOUND_THREADS) weight_bound_kernel(const __grid_constant__ Params P) {
    const int fl = blockIdx.x, f = P.f0 + fl;
    const JonesF64* Wf = P.W + (size_t)f * P.nc + P.c0;
    __shared__ double red[3][BOUND_THREADS / 32];
    double mx[3] = {0.0, 0.0, 0.0};
    for (int c = threadIdx.x; c < P.cn; c += BOUND_THREADS) {
        const double2* w = reinterpret_cast<const double2*>(Wf + c);
        const double2 xx = __ldg(w), xy = __ldg(w + 1), yy = __ldg(w + 3);
        mx[0] = fmax(mx[0], hypot(xx.x, xx.y));
        mx[1] = fmax(mx[1], hypot(yy.x, yy.y));
        mx[2] = fmax(mx[2], hypot(xy.x, xy.y));
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
    for (int p = 0; p < 3; p++) {
        for (int o = 16; o > 0; o >>= 1) mx[p] = fmax(mx[p], __shfl_xor_sync(0xffffffffu, mx[p], o));
        if (lane == 0) red[p][warp] = mx[p];
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        double bound = 0.0;
        for (int i = 0; i < BOUND_THREADS / 32; i++) bound = fmax(bound, red[threadIdx.x][i]);
        reinterpret_cast<double*>(const_cast<unsigned char*>(P.table) + (size_t)fl * P.tab_chan +
                                  P.tab_bound_off)[threadIdx.x] = bound;
    }
}

// MODE 2 table of one pass: grid (stages, 2 x row blocks, channels of the
// chunk), TT = 128 threads; CTA (k, 2 rb + half, f) takes the 64 tiles
// 128 rb + 64 half .. of stage k, i.e. one column block.  Thread (row, kh)
// takes tile 128 rb + 64 half + row and the stage's components 16 kh ..
// 16 kh + 15: their phasors A (the same FP64 phase and FP32 polynomials as
// the in-kernel forms), the 16-byte chunk of each of the six A planes (3
// digits of re and im, the encoding of y above), and the FP32 (cos, sin) row
// of the tile, staged in shared memory (rows padded to 272 bytes:
// conflict-free) so that every warp store to the table is 512 contiguous
// bytes.  The first CTAs of a stage also write its W sx of each
// polarisation.  A CTA this small (17 KB of shared memory) fits on an SM
// beside a Gram CTA, so the next chunk's table can be written while the
// Gram kernel of this one runs.
constexpr int TT = 128;
constexpr int TROW = PH_ROW + 16;
__global__ void __launch_bounds__(TT) phasor_table_kernel(const __grid_constant__ Params P) {
    __shared__ __align__(16) unsigned char phs[NH * TROW];
    __shared__ double2 lm_s[KC];
    __shared__ double n_s[KC];
    const int k = blockIdx.x, rb = blockIdx.y >> 1, half = blockIdx.y & 1, fl = blockIdx.z;
    const int f = P.f0 + fl;
    const int t = threadIdx.x;
    const int row = t >> 1, kh = t & 1;            // row of the 64
    const int brow = NH * half + row;              // row of the 128-row block
    const int tile = NT * rb + brow;
    const double oq = 4.0 * P.freqs[f] / VEL_C;
    double u, v, w;
    tile_uvw(P, tile, oq, u, v, w);
    unsigned char* tch = const_cast<unsigned char*>(P.table) + (size_t)fl * P.tab_chan;
    unsigned char* blk = tch + (size_t)k * P.tab_block;
    const JonesF64* Wf = P.W + (size_t)f * P.nc + P.c0;
    // the stage's component positions, once per CTA (past the end: A = 1,
    // whose W is zero)
    if (t < KC) {
        const int c = k * KC + t;
        double2 a = make_double2(0.0, 0.0);
        double nn = 0.0;
        if (c < P.cn) {
            const double4* lmn = P.lmn + P.c0;
            a = __ldg(reinterpret_cast<const double2*>(lmn + c));
            nn = __ldg(reinterpret_cast<const double*>(lmn + c) + 2);
        }
        lm_s[t] = a;
        n_s[t] = nn;
    } else if (blockIdx.y == 0 && t < KC + 3 * KC) {
        // W sx of polarisation p (XX, YY, XY) for component cl of the stage
        const int p = (t - KC) / KC, cl = (t - KC) % KC, c = k * KC + cl;
        const double bound = reinterpret_cast<const double*>(tch + P.tab_bound_off)[p];
        const float sx = bound > 0.0 ? (float)(FULL31 / bound) : 0.f;
        float2 o = make_float2(0.f, 0.f);
        if (c < P.cn) {
            const double2 wv = __ldg(reinterpret_cast<const double2*>(Wf + c) + (p == 0 ? 0 : (p == 1 ? 3 : 1)));
            o = make_float2((float)(wv.x * (double)sx), (float)(wv.y * (double)sx));
        }
        const int nstg = (P.cn + KC - 1) / KC;
        reinterpret_cast<float2*>(tch + P.tab_w_off)[((size_t)p * nstg + k) * KC + cl] = o;
    }
    __syncthreads();
    int yr[16], yi[16];
#pragma unroll
    for (int j = 0; j < 16; j += 2) {
        float2 ph[2];
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const double2 a = lm_s[kh * 16 + j + h];
            const double cn = n_s[kh * 16 + j + h];
            float sn, cs;
            phasor_quarter_f32(u * a.x + v * a.y + w * cn, sn, cs);
            // y + 0x8080 + 0x400000 in the FP32 mantissa (one rounding)
            yr[j + h] = __float_as_int(__fmaf_rn(cs, SY0, YOFF));
            yi[j + h] = __float_as_int(__fmaf_rn(sn, SY0, YOFF));
            ph[h] = make_float2(cs, sn);
        }
        *reinterpret_cast<float4*>(phs + row * TROW + kh * 128 + j * 8) = make_float4(ph[0].x, ph[0].y, ph[1].x, ph[1].y);
    }
    unsigned char* pb = blk + (size_t)rb * PL_BYTES + chunk_off(brow, kh);
#pragma unroll
    for (int part = 0; part < 2; part++) {
        uint32_t d[3][4];  // [digit][word of 4 components]
#pragma unroll
        for (int q = 0; q < 4; q++) {
            uint32_t pl[4];
            byte_planes4((part ? yi : yr) + 4 * q, pl);
            // bytes 0-1 excess-128, byte 2 the top digit + 64
            d[2][q] = pl[0] ^ 0x80808080u;
            d[1][q] = pl[1] ^ 0x80808080u;
            d[0][q] = minus64(pl[2]);
        }
#pragma unroll
        for (int dg = 0; dg < 3; dg++)
            *reinterpret_cast<uint4*>(pb + (part * 3 + dg) * XT_BYTES) = make_uint4(d[dg][0], d[dg][1], d[dg][2], d[dg][3]);
    }
    __syncthreads();
    // the phasor rows of column block 2 rb + half (if it exists): 16-byte
    // unit i of its 64 rows x 256 bytes
    const int cbt = 2 * rb + half;
    if (cbt < P.ncb) {
        unsigned char* pdst = blk + P.tab_ph_off + (size_t)cbt * PH_BYTES;
#pragma unroll
        for (int i = t; i < NH * (PH_ROW / 16); i += TT) {
            const int rr = i / (PH_ROW / 16), uu = i % (PH_ROW / 16);
            *reinterpret_cast<float4*>(pdst + (size_t)rr * PH_ROW + uu * 16) =
                *reinterpret_cast<const float4*>(phs + rr * TROW + uu * 16);
        }
    }
}

// vis [nf][nbl] += the four planes (one thread per visibility, coalesced)
template <bool OUT64>
__global__ void combine_kernel(const void* planes, void* vis, size_t n) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (OUT64) {
        const double2* pl = reinterpret_cast<const double2*>(planes);
        double2* v = reinterpret_cast<double2*>(reinterpret_cast<JonesF64*>(vis) + i);
#pragma unroll
        for (int s = 0; s < 4; s++) {
            const double2 a = pl[s * n + i];
            double2 b = v[s];
            b.x += a.x;
            b.y += a.y;
            v[s] = b;
        }
    } else {
        const float2* pl = reinterpret_cast<const float2*>(planes);
        float4* v = reinterpret_cast<float4*>(reinterpret_cast<JonesF32*>(vis) + i);
        const float2 xx = pl[i], xy = pl[n + i], yx = pl[2 * n + i], yy = pl[3 * n + i];
        float4 a = v[0], b = v[1];
        a.x += xx.x, a.y += xx.y, a.z += xy.x, a.w += xy.y;
        b.x += yx.x, b.y += yx.y, b.z += yy.x, b.w += yy.y;
        v[0] = a;
        v[1] = b;
    }
}

// vis[i] = (vis[i] + model[i]) + the four planes, for i in [i0, i0 + cnt)
// of n (the host-buffer call's chunks: the other classes' sum, staged in
// model, goes in before the points, as the device call adds them first)
__global__ void combine_model_kernel(const void* planes, JonesF32* vis, const JonesF32* model, size_t n, size_t i0,
                                     size_t cnt) {
    const size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= cnt) return;
    const size_t i = i0 + k;
    const float2* pl = reinterpret_cast<const float2*>(planes);
    float4* v = reinterpret_cast<float4*>(vis + i);
    const float4* m = reinterpret_cast<const float4*>(model + i);
    const float2 xx = pl[i], xy = pl[n + i], yx = pl[2 * n + i], yy = pl[3 * n + i];
    float4 a = v[0], b = v[1];
    const float4 ma = m[0], mb = m[1];
    a.x += ma.x, a.y += ma.y, a.z += ma.z, a.w += ma.w;
    b.x += mb.x, b.y += mb.y, b.z += mb.z, b.w += mb.w;
    a.x += xx.x, a.y += xx.y, a.z += xy.x, a.w += xy.y;
    b.x += yx.x, b.y += yx.y, b.z += yy.x, b.w += yy.y;
    v[0] = a;
    v[1] = b;
}

// Per channel: the largest |entry| of the beam Jones over unique tiles and
// components (at the channel's unique frequency) and of S (MODE 1 scales).
__global__ void beam_bounds_kernel(const JonesF64* beam, int n_uniq_tile, const int* freq_map, int n_uniq_freq,
                                   const JonesF64* S, int nc, int c0, int cn, double* maxb, double* maxs) {
    const int f = blockIdx.x;
    const int fm = freq_map[f];
    double mb = 0.0, ms = 0.0;
    for (int i = threadIdx.x; i < n_uniq_tile * cn; i += blockDim.x) {
        const int u = i / cn, c = i % cn;
        const double2* b = reinterpret_cast<const double2*>(beam + ((size_t)u * n_uniq_freq + fm) * nc + c0 + c);
#pragma unroll
        for (int e = 0; e < 4; e++) mb = fmax(mb, hypot(b[e].x, b[e].y));
    }
    for (int c = threadIdx.x; c < cn; c += blockDim.x) {
        const double2* s = reinterpret_cast<const double2*>(S + (size_t)f * nc + c0 + c);
#pragma unroll
        for (int e = 0; e < 4; e++) ms = fmax(ms, hypot(s[e].x, s[e].y));
    }
    __shared__ double rb[2][32];
    for (int o = 16; o > 0; o >>= 1) {
        mb = fmax(mb, __shfl_xor_sync(0xffffffffu, mb, o));
        ms = fmax(ms, __shfl_xor_sync(0xffffffffu, ms, o));
    }
    if ((threadIdx.x & 31) == 0) rb[0][threadIdx.x >> 5] = mb, rb[1][threadIdx.x >> 5] = ms;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x >> 5); w++) mb = fmax(mb, rb[0][w]), ms = fmax(ms, rb[1][w]);
        mb = fmax(mb, rb[0][0]);
        ms = fmax(ms, rb[1][0]);
        maxb[f] = mb;
        maxs[f] = ms;
    }
}

// The jobs of one channel: (pol, row block, column block) with a baseline of
// that polarisation.  Returns their number (0 if more than MAXJOBS).
int build_jobs(int ntiles, uint32_t* jobs) {
    const int nrb = (ntiles + NT - 1) / NT, ncb = (ntiles + NH - 1) / NH;
    int nj = 0;
    for (int pol = 0; pol < 3; pol++)
        for (int rb = 0; rb < nrb; rb++)
            for (int cb = 0; cb < ncb; cb++) {
                const int rlo = NT * rb, rhi = std::min(NT * rb + NT, ntiles) - 1;
                const int clo = NH * cb, chi = std::min(NH * cb + NH, ntiles) - 1;
                const bool any = pol < 2 ? chi > rlo : (rhi > rlo || chi > clo || rlo != clo);
                if (!any) continue;
                if (nj >= MAXJOBS) return 0;
                jobs[nj++] = (uint32_t)pol | ((uint32_t)rb << 8) | ((uint32_t)cb << 20);
            }
    return nj;
}

// The MODE 2 table of a pass: bytes per (channel, stage) and per channel,
// and the channels of one chunk: as many as fit in TABLE_CAP, rounded down
// to a multiple that fills whole waves of the SMs with jobs.
constexpr size_t TABLE_CAP = (size_t)1 << 30;

struct TableShape {
    int nrb, ncb, nstg, chunk;
    size_t block, chan;
};

static int gcd_int(int a, int b) { return b == 0 ? a : gcd_int(b, a % b); }

static TableShape table_shape(int nf, int ntiles, int cn, int njobs) {
    TableShape t;
    t.nrb = (ntiles + NT - 1) / NT;
    t.ncb = (ntiles + NH - 1) / NH;
    t.nstg = (cn + KC - 1) / KC;
    t.block = (size_t)t.nrb * PL_BYTES + (size_t)t.ncb * PH_BYTES;
    t.chan = (size_t)t.nstg * t.block + (size_t)3 * t.nstg * KC * sizeof(float2) + 32;
    int sms = 148, dev = 0;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaGetLastError();
    const int fit = (int)std::max<size_t>(1, TABLE_CAP / std::max<size_t>(t.chan, 1));
    const int q = sms / gcd_int(sms, std::max(njobs, 1));  // channels per whole number of waves
    t.chunk = std::min(nf, fit >= q ? fit / q * q : fit);
    return t;
}

}  // namespace tc

// Bytes of device workspace the tensor predict needs for nf channels of
// nc components: the four planes, the MODE 1 per-channel bounds and, with
// a shared beam, the MODE 2 table of one chunk of channels.
size_t tensor_workspace_bytes(int nf, int nbl, int ntiles, int nc, bool tile_beam, bool out64, bool two_tables) {
    const size_t planes = (size_t)4 * nf * nbl * (out64 ? 16 : 8);
    size_t bytes = ((planes + 255) & ~(size_t)255) + ((2 * sizeof(double) * (size_t)nf + 255) & ~(size_t)255);
    if (!tile_beam && nc > 0 && nf > 0) {
        std::vector<uint32_t> jobs(tc::MAXJOBS);
        const int nj = tc::build_jobs(ntiles, jobs.data());
        const tc::TableShape t = tc::table_shape(nf, ntiles, std::min(nc, tc::Cfg<2>::KPASS), nj);
        bytes += (two_tables && t.chunk < nf ? 2 : 1) * (size_t)t.chunk * t.chan;
    }
    return bytes + 256;
}

struct TensorState {
    bool configured = false;
    void* ws = nullptr;
    size_t ws_bytes = 0;
    TensorSync sync;
    bool sync_ok = false, sync_failed = false;
};

int tensor_sync_init(TensorSync& t) {
    HDC_CUDA_RET_INT(cudaStreamCreateWithFlags(&t.ts, cudaStreamNonBlocking));
    HDC_CUDA_RET_INT(cudaEventCreateWithFlags(&t.start, cudaEventDisableTiming));
    for (int b = 0; b < 2; b++) {
        HDC_CUDA_RET_INT(cudaEventCreateWithFlags(&t.table_done[b], cudaEventDisableTiming));
        HDC_CUDA_RET_INT(cudaEventCreateWithFlags(&t.gram_done[b], cudaEventDisableTiming));
    }
    return HDC_OK;
}

void tensor_sync_free(TensorSync& t) {
    for (int b = 0; b < 2; b++) {
        if (t.table_done[b]) cudaEventDestroy(t.table_done[b]);
        if (t.gram_done[b]) cudaEventDestroy(t.gram_done[b]);
    }
    if (t.start) cudaEventDestroy(t.start);
    if (t.ts) cudaStreamDestroy(t.ts);
    t = TensorSync();
}

int tensor_configure() {
    static std::once_flag once;
    static cudaError_t attr_err = cudaSuccess;
    std::call_once(once, [] {
        const cudaError_t e[4] = {
            cudaFuncSetAttribute(tc::gram_i8_kernel<1, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 tc::Lay<1>::SMEM_BYTES),
            cudaFuncSetAttribute(tc::gram_i8_kernel<1, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 tc::Lay<1>::SMEM_BYTES),
            cudaFuncSetAttribute(tc::gram_i8_kernel<2, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 tc::Lay<2>::SMEM_BYTES),
            cudaFuncSetAttribute(tc::gram_i8_kernel<2, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 tc::Lay<2>::SMEM_BYTES)};
        for (cudaError_t x : e)
            if (x != cudaSuccess && attr_err == cudaSuccess) attr_err = x;
    });
    HDC_CUDA_RET_INT(attr_err);
    return HDC_OK;
}

int Modeller::tensor_setup() {
    if (!tc) tc = new TensorState();
    int rc = tensor_configure();
    if (rc) return rc;
    if (tc::build_jobs(ntiles, std::vector<uint32_t>(tc::MAXJOBS).data()) == 0) {
        set_error("the tensor-core predict supports up to %d jobs per channel (%d tiles is too many)", tc::MAXJOBS,
                  ntiles);
        return HDC_ERR_UNSUPPORTED;
    }
    tc->configured = true;
    return HDC_OK;
}

// The tensor-core point predict of one timestep over device tables: lmn
// [nc] (turns), W [nf][nc] (B S B^H of a beam shared by all tiles, or S with
// per-tile beams in `beam`), tile XYZs, hour angle and declination of the
// phase centre; accumulates into vis [nf][nbl] (JonesF32, or JonesF64 with
// out64).  ws: tensor_workspace_bytes(nf, nbl, ntiles, nc, per-tile beams,
// out64, sync != NULL) bytes of device memory.  With sync, the tables of a
// shared beam alternate between two buffers and are written on sync->ts,
// each chunk's Gram kernel (on s) waiting for its table and each table for
// the Gram kernel that last read its buffer, so that writing the next
// chunk's table overlaps the current Gram kernel.
int tensor_single_pass() { return tc::Cfg<2>::KPASS; }

int launch_tensor_points(int nf, int nbl, int ntiles, int nc, const double* d_freqs, const XYZ* d_xyzs, double ha,
                         double dec, const double4* d_lmn, const JonesF64* d_W, const TensorBeam* beam, void* d_vis,
                         bool out64, void* ws, int* d_err, cudaStream_t s, TensorSync* sync,
                         const TensorChunkOut* chunk_out) {
    if (nc == 0 || nf == 0) return HDC_OK;
    if (chunk_out && (out64 || (beam && beam->beam) || nc > tc::Cfg<2>::KPASS)) {
        set_error("launch_tensor_points: per-chunk output needs the shared-beam table form, one pass, JonesF32");
        return HDC_ERR_ARG;
    }
    int rc = tensor_configure();
    if (rc) return rc;
    tc::Params P;
    P.njobs = tc::build_jobs(ntiles, P.jobs);
    if (P.njobs == 0) {
        set_error("the tensor-core predict supports up to %d jobs per channel (%d tiles is too many)", tc::MAXJOBS,
                  ntiles);
        return HDC_ERR_UNSUPPORTED;
    }
    const bool tile_beam = beam && beam->beam;
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
    P.beam = tile_beam ? beam->beam : nullptr;
    P.beam32 = tile_beam ? beam->beam32 : nullptr;
    P.tile_map = tile_beam ? beam->tile_map : nullptr;
    P.freq_map = tile_beam ? beam->freq_map : nullptr;
    P.n_uniq_freq = tile_beam ? beam->n_uniq_freq : 0;
    const size_t planes_bytes = (((size_t)4 * nf * nbl * (out64 ? 16 : 8)) + 255) & ~(size_t)255;
    P.planes = ws;
    double* bounds = reinterpret_cast<double*>(static_cast<char*>(ws) + planes_bytes);
    P.maxb = bounds;
    P.maxs = bounds + nf;
    P.err = d_err;
    P.f0 = 0;
    const unsigned char* table0 = static_cast<const unsigned char*>(ws) + planes_bytes +
                                  ((2 * sizeof(double) * (size_t)nf + 255) & ~(size_t)255);
    P.table = table0;
    P.tab_chan = P.tab_block = P.tab_ph_off = P.tab_w_off = P.tab_bound_off = 0;
    P.ncb = 0;
    const int kpass = tile_beam ? tc::Cfg<1>::KPASS : tc::Cfg<2>::KPASS;
    const size_t nvis = (size_t)nf * nbl;
    // passes of at most KPASS components accumulate into the visibilities in turn
    for (int c0 = 0; c0 < P.nc; c0 += kpass) {
        P.c0 = c0;
        P.cn = std::min(kpass, P.nc - c0);
        if (tile_beam) {
            tc::beam_bounds_kernel<<<nf, 256, 0, s>>>(beam->beam, beam->n_uniq_tile, beam->freq_map,
                                                      beam->n_uniq_freq, d_W, nc, c0, P.cn, bounds, bounds + nf);
            count_launches(1);
            HDC_CUDA_RET_INT(cudaGetLastError());
            const dim3 grid(P.njobs, nf);
            if (out64)
                tc::gram_i8_kernel<1, true><<<grid, tc::Cfg<1>::THREADS, tc::Lay<1>::SMEM_BYTES, s>>>(P);
            else
                tc::gram_i8_kernel<1, false><<<grid, tc::Cfg<1>::THREADS, tc::Lay<1>::SMEM_BYTES, s>>>(P);
            count_launches(1);
            HDC_CUDA_RET_INT(cudaGetLastError());
        } else {
            // the table of a chunk of channels, then their Gram products;
            // with sync the tables alternate between two buffers on the
            // second stream
            const tc::TableShape t = tc::table_shape(nf, ntiles, std::min(nc, kpass), P.njobs);
            const int nstg = (P.cn + tc::KC - 1) / tc::KC;
            P.tab_block = t.block;
            P.tab_w_off = (size_t)nstg * t.block;
            P.tab_bound_off = P.tab_w_off + (size_t)3 * nstg * tc::KC * sizeof(float2);
            P.tab_chan = P.tab_bound_off + 32;
            P.tab_ph_off = (size_t)t.nrb * tc::PL_BYTES;
            P.ncb = t.ncb;
            const bool two = sync != nullptr && t.chunk < nf;
            const unsigned char* buf[2] = {table0, table0 + (size_t)t.chunk * t.chan};
            if (two) {
                HDC_CUDA_RET_INT(cudaEventRecord(sync->start, s));
                HDC_CUDA_RET_INT(cudaStreamWaitEvent(sync->ts, sync->start, 0));
            }
            for (int f0 = 0, i = 0; f0 < nf; f0 += t.chunk, i++) {
                const int nch = std::min(t.chunk, nf - f0);
                const int b = two ? (i & 1) : 0;
                cudaStream_t tsx = two ? sync->ts : s;
                P.f0 = f0;
                P.table = buf[b];
                // the buffer's previous reader is done
                if (two && i >= 2) HDC_CUDA_RET_INT(cudaStreamWaitEvent(sync->ts, sync->gram_done[b], 0));
                tc::weight_bound_kernel<<<nch, tc::BOUND_THREADS, 0, tsx>>>(P);
                count_launches(1);
                HDC_CUDA_RET_INT(cudaGetLastError());
                tc::phasor_table_kernel<<<dim3(nstg, 2 * t.nrb, nch), tc::TT, 0, tsx>>>(P);
                count_launches(1);
                HDC_CUDA_RET_INT(cudaGetLastError());
                if (two) {
                    HDC_CUDA_RET_INT(cudaEventRecord(sync->table_done[b], sync->ts));
                    HDC_CUDA_RET_INT(cudaStreamWaitEvent(s, sync->table_done[b], 0));
                }
                const dim3 grid(P.njobs, nch);
                if (out64)
                    tc::gram_i8_kernel<2, true><<<grid, tc::Cfg<2>::THREADS, tc::Lay<2>::SMEM_BYTES, s>>>(P);
                else
                    tc::gram_i8_kernel<2, false><<<grid, tc::Cfg<2>::THREADS, tc::Lay<2>::SMEM_BYTES, s>>>(P);
                count_launches(1);
                HDC_CUDA_RET_INT(cudaGetLastError());
                if (two) HDC_CUDA_RET_INT(cudaEventRecord(sync->gram_done[b], s));
                if (chunk_out) {
                    const size_t i0 = (size_t)f0 * nbl, cnt = (size_t)nch * nbl;
                    tc::combine_model_kernel<<<(unsigned)((cnt + 255) / 256), 256, 0, s>>>(
                        ws, static_cast<JonesF32*>(d_vis), chunk_out->model, nvis, i0, cnt);
                    count_launches(1);
                    HDC_CUDA_RET_INT(cudaGetLastError());
                    rc = chunk_out->done(chunk_out->ctx, f0, nch);
                    if (rc) return rc;
                }
            }
            P.f0 = 0;
            if (chunk_out) return HDC_OK;
        }
        const unsigned blocks = (unsigned)((nvis + 255) / 256);
        if (out64)
            tc::combine_kernel<true><<<blocks, 256, 0, s>>>(ws, d_vis, nvis);
        else
            tc::combine_kernel<false><<<blocks, 256, 0, s>>>(ws, d_vis, nvis);
        count_launches(1);
        HDC_CUDA_RET_INT(cudaGetLastError());
    }
    return HDC_OK;
}

// The modeller's workspace for the tensor predict of up to nf channels.
void* Modeller::tensor_workspace(bool out64) {
    const size_t need = tensor_workspace_bytes(nf, nbl, ntiles, t[0].nc, tile_beams(), out64, tensor_sync() != nullptr);
    if (tc->ws_bytes < need) {
        if (tc->ws) cudaFree(tc->ws);
        tc->ws = nullptr;
        tc->ws_bytes = 0;
        if (cudaMalloc(&tc->ws, need) != cudaSuccess) {
            cudaGetLastError();
            set_error("tensor predict workspace of %zu bytes: allocation failed", need);
            return nullptr;
        }
        tc->ws_bytes = need;
    }
    return tc->ws;
}

// The modeller's second stream for the tensor predict (created on first
// use; NULL if that failed: the predict then runs on one stream).
TensorSync* Modeller::tensor_sync() {
    if (!tc) return nullptr;
    if (!tc->sync_ok) {
        if (tc->sync_failed) return nullptr;
        if (tensor_sync_init(tc->sync) != HDC_OK) {
            cudaGetLastError();
            tensor_sync_free(tc->sync);
            tc->sync_failed = true;
            return nullptr;
        }
        tc->sync_ok = true;
    }
    return &tc->sync;
}

void Modeller::tensor_release() {
    if (tc && tc->sync_ok) tensor_sync_free(tc->sync);
    if (tc && tc->ws) cudaFree(tc->ws);
    delete tc;
    tc = nullptr;
}

}  // namespace hdc
