// Direction-independent calibration (MitchCal / StefCal) for sm_100a:
// calibrate_timeblock of mwa_hyperdrive (di_calibrate/mod.rs:387-968).
//
// Plain form: one CTA per chanblock runs that chanblock's whole iteration
// loop on the device -- every chanblock converges (or fails) independently,
// so the grid needs no inter-CTA synchronisation and each CTA keeps its own
// iteration count, exactly as the reference's rayon loop over chanblocks.
// Per iteration a CTA streams the chanblock's timeblock of data and model
// (f32, promoted to f64) once: each thread owns one baseline for all
// timesteps and forms both tiles' contributions (MitchCal eq. 11,
// calibration_loop, mod.rs:900-968):
//     tile1: top += D (G2 M^H),     bot += (G2 M^H)^H (G2 M^H)
//     tile2: top += D^H (G1 M),     bot += (G1 M)^H (G1 M)
// in registers; tile1 sums are combined across the warp with a segmented
// shuffle reduction (consecutive baselines mostly share tile1) and added to
// shared-memory accumulators, tile2 sums are added with shared-memory
// atomics.  bot is Hermitian with a real diagonal and is kept as 4 reals.
// The per-tile update (top bot^-1), the NaN/failed-tile rules, the
// even-iteration averaging and convergence test and the final failure rules
// follow calibrate() (mod.rs:640-893) with block-wide votes.
//
// Collapsed form: the gains are constant over a timeblock, so the sums over
// its timesteps can be taken once, before the iterations.  With vec(J) =
// (J00, J01, J10, J11) and, per baseline,
//     X = sum_t vec(D_t) vec(M_t)^H    (4x4 complex),
//     C = sum_t vec(M_t) vec(M_t)^H    (4x4 Hermitian),
// the four accumulations above become, for G1 = G_p, G2 = G_q, H = G^H G:
//     tile1 top_ij = sum_kl X[ik][jl] G2_kl      bot_ij = sum_kl C[ik][jl] H2_kl
//     tile2 top_ij = sum_kl conj(X[ki][lj]) G1_kl  bot_ij = sum_kl C[lj][ki] H1_kl
// (each term regrouped, not approximated).  A collapse kernel forms X and C
// from the timeblock's data and model once (one read of both); each
// iteration then reads 48 numbers per baseline instead of 16 per timestep
// and does ~380 instead of 368 x timesteps FLOPs.  The covariances are
// stored in FP64 (HDC_CAL_COLLAPSED) or FP32 (HDC_CAL_COLLAPSED_F32: half
// the bytes per iteration; the rounding moves the solutions by ~1e-7
// relative); all arithmetic is FP64.

#include <mutex>
#include <vector>

#include "common.cuh"

namespace hdc {

constexpr int CT = 256;  // threads per CTA; supports up to CT tiles

struct CalParams {
    const JonesF32* data;  // [nt_total][nchan][nbl]
    const JonesF32* model;
    int t0, t1, nchan, nbl, ntiles;
    JonesF64* di_jones;  // [ntiles][nchan]
    const int* chan_list;  // chanblocks to calibrate (blockIdx.x -> chanblock)
    int max_iter;
    double stop, min_thr;
    int pols;
    HdcCalResult* results;  // [nchan]
    const void* cov;        // collapsed form: [nchan][nblk][48][256] block-major, FP64 or FP32
    int nblk;               // 16 x 16 tile-pair blocks per chanblock
    int nring;              // FP32 collapsed form: shared-memory ring depth (0: direct loads)
    int* err;               // device error word (bounded waits)
};

// Collapsed covariances are stored block-major: the pairs (p, q) of tile
// blocks pb <= qb (16 tiles each), enumerated column-major (qb outer, pb
// inner), each block [48 components][256 lanes] with lane = 16 (p % 16) +
// q % 16 and zeros where p >= q or q >= n -- so one block is one contiguous
// run of 48 x 256 values that a single bulk copy brings into shared memory.
constexpr int BLK = 256;
__host__ __device__ __forceinline__ int cov_blocks(int n) {
    const int nb = (n + 15) / 16;
    return nb * (nb + 1) / 2;
}
__device__ __forceinline__ void cov_block_coords(int b, int& pb, int& qb) {
    qb = 0;
    while ((qb + 1) * (qb + 2) / 2 <= b) qb++;
    pb = b - qb * (qb + 1) / 2;
}

// Covariance components per baseline: X[u][v] re at u*4+v, im at 16+u*4+v;
// C Hermitian: diagonal reals at 32+u, off-diagonal (u<v) re/im at
// 36 + 2*pair, 37 + 2*pair with pair = 0..5 for (01,02,03,12,13,23).
constexpr int NCOV = 48;
__host__ __device__ constexpr int cpair(int u, int v) {
    return u == 0 ? v - 1 : (u == 1 ? v + 1 : 5);
}

struct Herm {  // [a b; conj(b) d], a and d real
    double a, d;
    cplx b;
};
// the iteration kernel adds row and column sums to a Herm as doubles 0..3
static_assert(offsetof(Herm, d) == 8 && offsetof(Herm, b) == 16 && sizeof(Herm) == 32, "Herm layout");

__device__ __forceinline__ J2 load_vis(const JonesF32* p) {
    const float4* q = reinterpret_cast<const float4*>(p);
    const float4 x = __ldg(q), y = __ldg(q + 1);
    return J2{{x.x, x.y}, {x.z, x.w}, {y.x, y.y}, {y.z, y.w}};
}

// Z^H Z for Z = [z0 z1; z2 z3]
__device__ __forceinline__ void add_zhz(Herm& h, const J2& z) {
    h.a += z.a.re * z.a.re + z.a.im * z.a.im + z.c.re * z.c.re + z.c.im * z.c.im;
    h.d += z.b.re * z.b.re + z.b.im * z.b.im + z.d.re * z.d.re + z.d.im * z.d.im;
    h.b = h.b + conj(z.a) * z.b + conj(z.c) * z.d;
}

__device__ __forceinline__ double warp_seg_sum(double v, int key, int lane) {
    // inclusive suffix sum over lanes with the same key; keys are
    // non-decreasing with lane, so each key is a contiguous run
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const double other = __shfl_down_sync(0xffffffffu, v, o);
        const int ok = __shfl_down_sync(0xffffffffu, key, o);
        if (lane + o < 32 && ok == key) v += other;
    }
    return v;
}

__device__ __forceinline__ cplx cdiv(cplx a, cplx b) {
    const double n = b.re * b.re + b.im * b.im;
    return {(a.re * b.re + a.im * b.im) / n, (a.im * b.re - a.re * b.im) / n};
}

// marlu Jones::inv and Jones division (top * bot^-1)
__device__ __forceinline__ J2 jdiv(const J2& top, const J2& bot, int pols) {
    if (pols == 1) return J2{cdiv(top.a, bot.a), {0, 0}, {0, 0}, {0, 0}};
    if (pols == 2) return J2{{0, 0}, {0, 0}, {0, 0}, cdiv(top.d, bot.d)};
    const cplx det = bot.a * bot.d - bot.b * bot.c;
    const cplx inv_det = cdiv(cplx{1.0, 0.0}, det);
    const cplx m = cplx{-inv_det.re, -inv_det.im};
    const J2 inv = J2{inv_det * bot.d, m * bot.b, m * bot.c, inv_det * bot.a};
    return top * inv;
}

__device__ __forceinline__ bool any_nan(const J2& j) {
    return isnan(j.a.re) || isnan(j.a.im) || isnan(j.b.re) || isnan(j.b.im) || isnan(j.c.re) || isnan(j.c.im) ||
           isnan(j.d.re) || isnan(j.d.im);
}

__device__ __forceinline__ double cnorm(cplx a) { return a.re * a.re + a.im * a.im; }

// X and C of one (chanblock, baseline) over the timeblock (thread per
// baseline, chanblock on blockIdx.y); stored structure-of-arrays so that a
// warp's loads of one component are contiguous.
template <typename T>
__global__ void __launch_bounds__(BLK / 2) collapse_kernel(const CalParams P, T* cov) {
    const int b = blockIdx.x >> 1, ch = blockIdx.y, lane = (blockIdx.x & 1) * (BLK / 2) + threadIdx.x;
    int pb, qb;
    cov_block_coords(b, pb, qb);
    const int p = pb * 16 + (lane >> 4), q = qb * 16 + (lane & 15);
    T* out = cov + ((size_t)ch * P.nblk + b) * NCOV * BLK + lane;
    if (!(p < q && q < P.ntiles)) {
#pragma unroll
        for (int k = 0; k < NCOV; k++) out[(size_t)k * BLK] = (T)0;
        return;
    }
    const int bl = baseline_index(p, q, P.ntiles);
    const size_t tstride = (size_t)P.nchan * P.nbl;
    const JonesF32* D0 = P.data + ((size_t)P.t0 * P.nchan + ch) * P.nbl + bl;
    const JonesF32* M0 = P.model + ((size_t)P.t0 * P.nchan + ch) * P.nbl + bl;
    double xr[16], xi[16], cd[4], cr[6], ci[6];
#pragma unroll
    for (int k = 0; k < 16; k++) xr[k] = xi[k] = 0.0;
#pragma unroll
    for (int k = 0; k < 6; k++) cr[k] = ci[k] = 0.0;
#pragma unroll
    for (int k = 0; k < 4; k++) cd[k] = 0.0;
    for (int t = 0; t < P.t1 - P.t0; t++) {
        const J2 dj = load_vis(D0 + t * tstride), mj = load_vis(M0 + t * tstride);
        const cplx d[4] = {dj.a, dj.b, dj.c, dj.d}, m[4] = {mj.a, mj.b, mj.c, mj.d};
#pragma unroll
        for (int u = 0; u < 4; u++)
#pragma unroll
            for (int v = 0; v < 4; v++) {
                // d[u] conj(m[v])
                xr[u * 4 + v] += d[u].re * m[v].re + d[u].im * m[v].im;
                xi[u * 4 + v] += d[u].im * m[v].re - d[u].re * m[v].im;
            }
#pragma unroll
        for (int u = 0; u < 4; u++) {
            cd[u] += m[u].re * m[u].re + m[u].im * m[u].im;
#pragma unroll
            for (int v = u + 1; v < 4; v++) {
                cr[cpair(u, v)] += m[u].re * m[v].re + m[u].im * m[v].im;
                ci[cpair(u, v)] += m[u].im * m[v].re - m[u].re * m[v].im;
            }
        }
    }
#pragma unroll
    for (int k = 0; k < 16; k++) {
        out[(size_t)k * BLK] = (T)xr[k];
        out[(size_t)(16 + k) * BLK] = (T)xi[k];
    }
#pragma unroll
    for (int u = 0; u < 4; u++) out[(size_t)(32 + u) * BLK] = (T)cd[u];
#pragma unroll
    for (int k = 0; k < 6; k++) {
        out[(size_t)(36 + 2 * k) * BLK] = (T)cr[k];
        out[(size_t)(37 + 2 * k) * BLK] = (T)ci[k];
    }
}

// Covariance component k of one lane: from global memory (read-only path),
// or from a ring slot in shared memory through its 32-bit shared address
// (explicit ld.shared: the slot's address is computed at run time, where a
// generic load would be issued otherwise).
template <typename T>
struct CovGlobal {
    const T* cv;
    __device__ __forceinline__ double operator()(int k) const { return (double)__ldg(cv + (size_t)k * BLK); }
};
struct CovShared {
    uint32_t base;  // shared address of component 0 of this lane
    __device__ __forceinline__ double operator()(int k) const {
        float v;
        asm volatile("ld.shared.f32 %0, [%1];" : "=f"(v) : "r"(base + (uint32_t)(k * BLK * sizeof(float))));
        return (double)v;
    }
};

// acc += x g (first: acc = x g), as two fused multiply-adds per part
__device__ __forceinline__ void cmac(cplx& acc, cplx x, cplx g, bool first) {
    acc.re = first ? x.re * g.re : fma(x.re, g.re, acc.re);
    acc.im = first ? x.re * g.im : fma(x.re, g.im, acc.im);
    acc.re = fma(-x.im, g.im, acc.re);
    acc.im = fma(x.im, g.re, acc.im);
}
// acc += conj(x) g (first: acc = conj(x) g)
__device__ __forceinline__ void cmac_conj(cplx& acc, cplx x, cplx g, bool first) {
    acc.re = first ? x.re * g.re : fma(x.re, g.re, acc.re);
    acc.im = first ? x.re * g.im : fma(x.re, g.im, acc.im);
    acc.re = fma(x.im, g.im, acc.re);
    acc.im = fma(-x.im, g.re, acc.im);
}

// One baseline's tile1 and tile2 contributions from its covariances
// (component k from ld(k)), each entry read once:
//   t1_ij = sum_kl X[ik][jl] G2_kl        t2_ij = sum_kl conj(X[ki][lj]) G1_kl
//   h1_ij = sum_kl C[ik][jl] H2_kl        h2_ij = sum_kl C[lj][ki] H1_kl
// With u = 2a + b, v = 2c + d an entry X[u][v] adds X G2[2b+d] to t1[2a+c]
// and conj(X) G1[2a+c] to t2[2b+d]; C[u][v] (and its conjugate C[v][u])
// adds C H2[2b+d] to h1[2a+c] and C H1[2c+a] to h2[2d+b]; only the bot
// entries 00, 11 (real) and 01 are kept.  Every product is added with a
// fused multiply-add.  t1 and h1 are this baseline's (each accumulator
// starts from its first product); t2 and h2 are added straight into the
// caller's running column sums c2 and ch2.
template <class LD>
__device__ __forceinline__ void collapsed_terms(const LD& ld, const J2& g1, const J2& g2, const Herm& H1,
                                                const Herm& H2, J2& t1, Herm& h1, J2& c2, Herm& ch2) {
    const cplx G1[4] = {g1.a, g1.b, g1.c, g1.d}, G2[4] = {g2.a, g2.b, g2.c, g2.d};
    cplx T1[4], T2[4] = {c2.a, c2.b, c2.c, c2.d};
#pragma unroll
    for (int u = 0; u < 4; u++)
#pragma unroll
        for (int v = 0; v < 4; v++) {
            const cplx x{ld(u * 4 + v), ld(16 + u * 4 + v)};
            // T1[2a+c] is first reached at b = d = 0
            cmac(T1[(u >> 1) * 2 + (v >> 1)], x, G2[(u & 1) * 2 + (v & 1)], (u & 1) == 0 && (v & 1) == 0);
            cmac_conj(T2[(u & 1) * 2 + (v & 1)], x, G1[(u >> 1) * 2 + (v >> 1)], false);
        }
    t1 = J2{T1[0], T1[1], T1[2], T1[3]};
    c2 = J2{T2[0], T2[1], T2[2], T2[3]};
    // bot accumulators: entry (u, v) = C[2a+b][2c+d] feeds b1[2a+c] with
    // H2[2b+d] and, read as C[2l+j][2k+i], b2[2i+j] with H1[2k+l].  The
    // results are Hermitian, so only entries 00 and 11 (real parts) and 01
    // are formed; every index below is a compile-time constant once the
    // loops are unrolled, so the unused terms are never computed.
    double b1_00 = 0.0, b1_11 = 0.0, b2_00 = ch2.a, b2_11 = ch2.d;
    cplx b1_01{0.0, 0.0}, b2_01 = ch2.b;
    // r += c h for target entry i (0, 1, 3; 2 is not kept) and entry k of the
    // Hermitian H (0, 3 real; 1 = b; 2 = conj(b)); c real when creal
    auto acc = [](double& r00, double& r11, cplx& r01, int i, cplx c, bool creal, int k, const Herm& H) {
        if (i == 2) return;
        if (k == 0 || k == 3) {
            const double hr = k == 0 ? H.a : H.d;
            if (i == 1) {
                r01.re = fma(c.re, hr, r01.re);
                if (!creal) r01.im = fma(c.im, hr, r01.im);
            } else {
                double& r = i == 0 ? r00 : r11;
                r = fma(c.re, hr, r);
            }
        } else {
            const cplx h = k == 1 ? H.b : conj(H.b);
            if (i == 1) {
                r01.re = fma(c.re, h.re, r01.re);
                r01.im = fma(c.re, h.im, r01.im);
                if (!creal) {
                    r01.re = fma(-c.im, h.im, r01.re);
                    r01.im = fma(c.im, h.re, r01.im);
                }
            } else {
                double& r = i == 0 ? r00 : r11;
                r = fma(c.re, h.re, r);
                if (!creal) r = fma(-c.im, h.im, r);
            }
        }
    };
    auto add = [&](int u, int v, cplx c, bool creal) {
        acc(b1_00, b1_11, b1_01, (u >> 1) * 2 + (v >> 1), c, creal, (u & 1) * 2 + (v & 1), H2);
        acc(b2_00, b2_11, b2_01, (v & 1) * 2 + (u & 1), c, creal, (v >> 1) * 2 + (u >> 1), H1);
    };
#pragma unroll
    for (int u = 0; u < 4; u++) add(u, u, cplx{ld(32 + u), 0.0}, true);
#pragma unroll
    for (int u = 0; u < 4; u++)
#pragma unroll
        for (int v = u + 1; v < 4; v++) {
            const cplx c{ld(36 + 2 * cpair(u, v)), ld(37 + 2 * cpair(u, v))};
            add(u, v, c, false);
            add(v, u, conj(c), false);
        }
    h1 = Herm{b1_00, b1_11, b1_01};
    ch2 = Herm{b2_00, b2_11, b2_01};
}

// Sum of 12 values (t's 8 reals, then h's a, d, b.re, b.im) over the 16
// lanes of a half-warp, reduced and scattered: each round halves the values
// a lane keeps (it sends the half its partner keeps), so after four rounds
// lane j of the half-warp holds the total of value j (zero for j >= 12).
// Every value is summed in the same pairing order on every lane.
__device__ __forceinline__ double row_reduce_scatter16(const J2& t, const Herm& h, int j) {
    double v[16] = {t.a.re, t.a.im, t.b.re, t.b.im, t.c.re, t.c.im, t.d.re, t.d.im,
                    h.a,    h.d,    h.b.re, h.b.im, 0.0,    0.0,    0.0,    0.0};
#pragma unroll
    for (int half = 8; half > 0; half >>= 1) {
        const bool hi = (j & half) != 0;
#pragma unroll
        for (int k = 0; k < half; k++) {
            const double send = hi ? v[k] : v[k + half];
            const double keep = hi ? v[k + half] : v[k];
            v[k] = keep + __shfl_xor_sync(0xffffffffu, send, half);
        }
    }
    return v[0];
}

// The same sums (lane j of each half-warp gets the total of value j, j <
// 12) through shared memory: the warp's own 128-byte segments of components
// 0..23 of the ring slot it has just read (wbase: shared address of the
// segment of component 0) hold the 12 values of its 32 lanes as rows of 16
// doubles (row k + 12 r for value k of half-warp r); lane j of half-warp r
// sums row j + 12 r, starting at column j so that the 12 lanes of a
// half-warp hit different banks.  12 stores and 16 loads per lane in place
// of the shuffles' 15 exchanges and 60 selects.
__device__ __forceinline__ double row_sum_via_slot(uint32_t wbase, const J2& t, const Herm& h, int lane) {
    const int r = lane >> 4, c = lane & 15;
    const double v[12] = {t.a.re, t.a.im, t.b.re, t.b.im, t.c.re, t.c.im, t.d.re, t.d.im, h.a, h.d, h.b.re, h.b.im};
    constexpr uint32_t ROW = BLK * sizeof(float);  // one component of the slot
    __syncwarp();  // every lane's covariance reads before the stores over them
#pragma unroll
    for (int k = 0; k < 12; k++)
        asm volatile("st.shared.f64 [%0], %1;" ::"r"(wbase + (uint32_t)(k + 12 * r) * ROW + (uint32_t)c * 8u),
                     "d"(v[k])
                     : "memory");
    __syncwarp();
    double s = 0.0;
    if (c < 12) {
        const uint32_t row = wbase + (uint32_t)(c + 12 * r) * ROW;
#pragma unroll
        for (int i = 0; i < 16; i++) {
            double x;
            asm volatile("ld.shared.f64 %0, [%1];" : "=d"(x) : "r"(row + (uint32_t)((c + i) & 15) * 8u) : "memory");
            s = i == 0 ? x : s + x;
        }
    }
    return s;
}

// Barrier over one group of the iteration kernel (the whole CTA when it has
// one group; else named barrier 1 + grp over its 256 threads); the _or form
// returns true when any thread of the group passed true.
template <int NG>
__device__ __forceinline__ bool group_sync_or(bool v, int grp) {
    if (NG == 1) return __syncthreads_or(v);
    int r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\t"
        "setp.ne.b32 p, %1, 0;\n\t"
        "bar.red.or.pred q, %2, 256, p;\n\t"
        "selp.b32 %0, 1, 0, q;\n\t}"
        : "=r"(r)
        : "r"((int)v), "r"(1 + grp)
        : "memory");
    return r != 0;
}
template <int NG>
__device__ __forceinline__ void group_sync(int grp) {
    if (NG == 1)
        __syncthreads();
    else
        asm volatile("bar.sync %0, 256;" ::"r"(1 + grp) : "memory");
}

// Threads per CTA of the iteration kernel: the FP32 collapsed form runs two
// groups of 256 (one per parity of the block's storage index) on one
// shared ring.
__host__ __device__ constexpr int cal_threads(int form) { return form == HDC_CAL_COLLAPSED_F32 ? 2 * CT : CT; }

template <int FORM>
__global__ void __launch_bounds__(cal_threads(FORM)) mitchcal_kernel(const CalParams P) {
    constexpr int NTH = cal_threads(FORM);
    extern __shared__ double smem[];
    const int n = P.ntiles;
    J2* G = reinterpret_cast<J2*>(smem);          // current gains
    J2* Gold = G + n;                              // previous gains
    J2* top = Gold + n;                            // accumulators
    Herm* bot = reinterpret_cast<Herm*>(top + n);
    Herm* Hs = bot + n;                                  // G^H G per tile (collapsed form)
    double* prec = reinterpret_cast<double*>(Hs + n);   // [n][4]
    int* failed = reinterpret_cast<int*>(prec + 4 * n);
    // collapsed form: 16 x 16 x 12 block-column partial sums (8-byte aligned)
    double* colbuf = reinterpret_cast<double*>(failed + ((n + 1) & ~1));
    // FP32 collapsed form: the second group's own accumulators, added into
    // top/bot once both groups have swept the blocks
    J2* top1 = reinterpret_cast<J2*>(colbuf + 16 * 16 * 12);
    Herm* bot1 = reinterpret_cast<Herm*>(top1 + (FORM == 2 ? n : 0));

    const int ch = P.chan_list ? P.chan_list[blockIdx.x] : blockIdx.x;
    const int tid = threadIdx.x, lane = tid & 31;
    const int nt = P.t1 - P.t0;
    const size_t tstride = (size_t)P.nchan * P.nbl;
    const JonesF32* D0 = P.data + ((size_t)P.t0 * P.nchan + ch) * P.nbl;
    const JonesF32* M0 = P.model + ((size_t)P.t0 * P.nchan + ch) * P.nbl;

    // FP32 collapsed form: ring of nring covariance blocks after colbuf
    // (16-byte aligned for the bulk copies), one mbarrier per slot
    // slot s holds sequence number ring_tag[s] (blocks are numbered in
    // consumption order over all iterations): a waiter checks the tag before
    // the phase parity, because the warps of one group can reach the next
    // use of a slot while the other group's use in between is still pending,
    // and a parity alone cannot tell two phases apart.  ring_rel counts the
    // warps that have finished reading the slot's current block: the last of
    // the group's warps refills it.
    __shared__ alignas(8) uint64_t ring_bar[4];
    __shared__ uint32_t ring_cnt[4];  // copies issued per slot
    __shared__ uint32_t ring_tag[4], ring_rel[4];
    const bool use_ring = FORM == 2 && P.nring > 0;
    float* ring = reinterpret_cast<float*>((reinterpret_cast<uintptr_t>(bot1 + (FORM == 2 ? n : 0)) + 15) & ~(uintptr_t)15);
    uint32_t jseq = 0;  // covariance blocks consumed so far (all threads alike)
    bool abort_loop = false;

    for (int i = tid; i < n; i += NTH) {
        G[i] = load_j(P.di_jones[(size_t)i * P.nchan + ch]);
        Gold[i] = jzero();
        for (int k = 0; k < 4; k++) prec[4 * i + k] = 0.0;
        failed[i] = 0;
    }
    if (use_ring && tid == 0) {
        for (int s = 0; s < P.nring; s++) {
            mbar_init(&ring_bar[s], 1);
            ring_cnt[s] = 1;  // the first copy, issued below
            ring_tag[s] = (uint32_t)s;
            ring_rel[s] = 0;
        }
        fence_barrier_init();
    }
    __syncthreads();
    if (use_ring && tid == 0) {
        for (int s = 0; s < P.nring; s++) {
            mbar_arrive_expect_tx(&ring_bar[s], NCOV * BLK * sizeof(float));
            bulk_g2s(ring + (size_t)s * NCOV * BLK,
                     static_cast<const float*>(P.cov) + ((size_t)ch * P.nblk + s % P.nblk) * NCOV * BLK,
                     NCOV * BLK * sizeof(float), &ring_bar[s]);
        }
    }

    int iteration = 0;
    while (iteration < P.max_iter) {
        iteration++;
        for (int i = tid; i < n; i += NTH) {
            top[i] = jzero();
            bot[i] = Herm{0.0, 0.0, {0.0, 0.0}};
            if (FORM == 2) {
                top1[i] = jzero();
                bot1[i] = Herm{0.0, 0.0, {0.0, 0.0}};
            }
            if (FORM != 0) {
                Herm h{0.0, 0.0, {0.0, 0.0}};
                add_zhz(h, G[i]);
                Hs[i] = h;
            }
        }
        __syncthreads();

        // ---- accumulate top / bot (calibration_loop) ----
        if (FORM == 0) {
        const int nwarp_bl = (P.nbl + 31) & ~31;
        for (int base = tid & ~31; base < nwarp_bl; base += NTH) {
            const int bl = base + lane;
            const bool active = bl < P.nbl;
            int p = -1 - lane, q = 0;  // unique keys for inactive lanes
            J2 t1 = jzero(), t2 = jzero();
            Herm h1{0, 0, {0, 0}}, h2{0, 0, {0, 0}};
            if (active) {
                baseline_to_tiles(bl, n, p, q);
                const J2 gp = G[p], gq = G[q];
                for (int t = 0; t < nt; t++) {
                    const J2 d = load_vis(D0 + t * tstride + bl);
                    const J2 m = load_vis(M0 + t * tstride + bl);
                    const J2 z1 = gq * herm(m);
                    t1 = t1 + d * z1;
                    add_zhz(h1, z1);
                    const J2 z2 = gp * m;
                    t2 = t2 + herm(d) * z2;
                    add_zhz(h2, z2);
                }
            }
            // tile1 (row) sums: segmented reduction, head lane adds
            double v[12] = {t1.a.re, t1.a.im, t1.b.re, t1.b.im, t1.c.re, t1.c.im,
                            t1.d.re, t1.d.im, h1.a,    h1.d,    h1.b.re, h1.b.im};
#pragma unroll
            for (int k = 0; k < 12; k++) v[k] = warp_seg_sum(v[k], p, lane);
            const int prev = __shfl_up_sync(0xffffffffu, p, 1);
            const bool head = active && (lane == 0 || prev != p);
            if (head) {
                double* tp = reinterpret_cast<double*>(&top[p]);
                for (int k = 0; k < 8; k++) atomicAdd(tp + k, v[k]);
                atomicAdd(&bot[p].a, v[8]);
                atomicAdd(&bot[p].d, v[9]);
                atomicAdd(&bot[p].b.re, v[10]);
                atomicAdd(&bot[p].b.im, v[11]);
            }
            if (active) {
                double* tq = reinterpret_cast<double*>(&top[q]);
                atomicAdd(tq + 0, t2.a.re);
                atomicAdd(tq + 1, t2.a.im);
                atomicAdd(tq + 2, t2.b.re);
                atomicAdd(tq + 3, t2.b.im);
                atomicAdd(tq + 4, t2.c.re);
                atomicAdd(tq + 5, t2.c.im);
                atomicAdd(tq + 6, t2.d.re);
                atomicAdd(tq + 7, t2.d.im);
                atomicAdd(&bot[q].a, h2.a);
                atomicAdd(&bot[q].d, h2.d);
                atomicAdd(&bot[q].b.re, h2.b.re);
                atomicAdd(&bot[q].b.im, h2.b.im);
            }
        }
        } else {
            // collapsed: 16 x 16 blocks of tile pairs (p, q), p < q, in
            // storage order (column block qb outer, row block pb inner);
            // thread (bi, bj) takes pair (16 pb + bi, 16 qb + bj).  Tile-1
            // (row) sums run along a block row (16 consecutive lanes,
            // shuffles) and go to top/bot[p] from one lane; tile-2 (column)
            // sums stay in registers over the whole block column and are
            // reduced across rows once per column block through shared
            // memory -- every accumulator entry has one writer at a time and
            // no atomics.  FP32 covariances arrive through the shared-memory
            // ring (bulk copies issued nring blocks ahead); FP64 ones are
            // loaded directly.
            // FORM 2 runs two groups of 256 threads: group g takes the
            // blocks of odd or even storage index (18 each for 128 tiles),
            // so the two groups consume alternate ring slots, and sums into
            // its own accumulators (group 1: top1/bot1, added to top/bot
            // after the sweep).  A group's warps meet once per column block
            // to reduce its column sums (named barrier 1 + g); the groups
            // meet only at the end of the sweep.  Within a column block the
            // warps do not meet: a row of the block belongs to one warp in
            // every block, so each accumulator entry has one writer.
            constexpr int NG = NTH / BLK;
            const int grp = tid / BLK, gt = tid % BLK;
            const int bi = gt >> 4, bj = gt & 15;
            const int nb = (n + 15) / 16;
            J2* tacc = FORM == 2 && grp == 1 ? top1 : top;
            Herm* bacc = FORM == 2 && grp == 1 ? bot1 : bot;
            bool gabort = false;
            for (int qb = 0; qb < nb; qb++) {
                const int q = qb * 16 + bj;
                // tile q's gain and G^H G are the same for the whole block column
                const J2 gq = q < n ? G[q] : jzero();
                const Herm hq = q < n ? Hs[q] : Herm{0, 0, {0, 0}};
                J2 c2 = jzero();
                Herm ch2{0, 0, {0, 0}};
                // this group's blocks of the column: storage index = grp mod NG
                for (int pb = NG == 1 ? 0 : (grp - qb * (qb + 1) / 2) & 1; pb <= qb && !gabort; pb += NG) {
                    const int p = pb * 16 + bi;
                    const int blk = qb * (qb + 1) / 2 + pb;
                    J2 t1 = jzero();
                    Herm h1{0, 0, {0, 0}};
                    const uint32_t j = jseq + (uint32_t)blk;
                    // the ring is 3 or 2 slots deep: constant divisors
                    const int st = !use_ring ? 0 : P.nring == 3 ? (int)(j % 3u) : (int)(j & 1u);
                    if (use_ring) {
                        const uint32_t ph = (P.nring == 3 ? j / 3u : j >> 1) & 1u;
                        const bool ok = tag_wait_bounded(&ring_tag[st], j, P.err) &&
                                        mbar_wait_bounded(&ring_bar[st], ph, P.err);
                        if (__any_sync(0xffffffffu, !ok)) {
                            gabort = true;
                            break;
                        }
                        if (p < q && q < n)
                            collapsed_terms(CovShared{smem_u32(ring + (size_t)st * NCOV * BLK + gt)}, G[p], gq, Hs[p],
                                            hq, t1, h1, c2, ch2);
                    } else if (p < q && q < n) {
                        const size_t off = ((size_t)ch * P.nblk + blk) * NCOV * BLK + gt;
                        if (FORM == 1)
                            collapsed_terms(CovGlobal<double>{static_cast<const double*>(P.cov) + off}, G[p], gq,
                                            Hs[p], hq, t1, h1, c2, ch2);
                        else
                            collapsed_terms(CovGlobal<float>{static_cast<const float*>(P.cov) + off}, G[p], gq, Hs[p],
                                            hq, t1, h1, c2, ch2);
                    }
                    // row sums over the 16 lanes of the block row: lane bj
                    // gets the total of value bj (top's 8 reals, then bot's
                    // a, d, b.re, b.im, which is Herm's field order)
                    const double rs =
                        use_ring ? row_sum_via_slot(smem_u32(ring + (size_t)st * NCOV * BLK + (gt & ~31)), t1, h1, lane)
                                 : row_reduce_scatter16(t1, h1, bj);
                    if (bj < 12 && p < n)
                        *(bj < 8 ? reinterpret_cast<double*>(&tacc[p]) + bj : reinterpret_cast<double*>(&bacc[p]) + (bj - 8)) +=
                            rs;
                    if (use_ring) {
                        // this warp has read the slot; the group's last warp
                        // to finish it refills it nring blocks ahead (no
                        // barrier: the other warps go on to their next block)
                        __syncwarp();
                        if (lane == 0) {
                            __threadfence_block();  // this warp's reads before its count
                            if (atomicAdd(&ring_rel[st], 1u) == (uint32_t)(BLK / 32 - 1)) {
                                __threadfence_block();  // every warp's reads before the refill
                                ring_rel[st] = 0;
                                const int nxt = (int)((j + (uint32_t)P.nring) % (uint32_t)P.nblk);
                                fence_proxy_async_smem();  // generic reads of the slot before the async write
                                ring_cnt[st] += 1u;
                                mbar_arrive_expect_tx(&ring_bar[st], NCOV * BLK * sizeof(float));
                                bulk_g2s(ring + (size_t)st * NCOV * BLK,
                                         static_cast<const float*>(P.cov) + ((size_t)ch * P.nblk + nxt) * NCOV * BLK,
                                         NCOV * BLK * sizeof(float), &ring_bar[st]);
                                st_release_smem(&ring_tag[st], j + (uint32_t)P.nring);
                            }
                        }
                    }
                }
                // column sums: rows bi and bi ^ 1 share a warp; one partial per warp
                double cv2[12] = {c2.a.re, c2.a.im, c2.b.re, c2.b.im, c2.c.re, c2.c.im,
                                  c2.d.re, c2.d.im, ch2.a,   ch2.d,   ch2.b.re, ch2.b.im};
#pragma unroll
                for (int k = 0; k < 12; k++) cv2[k] += __shfl_xor_sync(0xffffffffu, cv2[k], 16);
                if ((tid & 31) < 16) {
                    double* cb = colbuf + ((size_t)(tid >> 5) * 16 + bj) * 12;
#pragma unroll
                    for (int k = 0; k < 12; k++) cb[k] = cv2[k];
                }
                if (group_sync_or<NG>(gabort, grp)) {
                    gabort = true;
                    break;
                }
                if (gt < 16 * 12) {
                    const int jq = gt / 12, k = gt - jq * 12;
                    const int qq = qb * 16 + jq;
                    double sum = 0.0;
#pragma unroll
                    for (int w = 0; w < BLK / 32; w++) sum += colbuf[((grp * (BLK / 32) + w) * 16 + jq) * 12 + k];
                    if (qq < n)
                        *(k < 8 ? reinterpret_cast<double*>(&tacc[qq]) + k : reinterpret_cast<double*>(&bacc[qq]) + (k - 8)) +=
                            sum;
                }
                group_sync<NG>(grp);
            }
            // both groups' sweeps done: fold group 1's sums into top/bot
            if (__syncthreads_or(gabort)) {
                abort_loop = true;
            } else if (FORM == 2) {
                for (int i = tid; i < n; i += NTH) {
                    top[i] = top[i] + top1[i];
                    bot[i].a += bot1[i].a;
                    bot[i].d += bot1[i].d;
                    bot[i].b = bot[i].b + bot1[i].b;
                }
            }
            if (use_ring) jseq += (uint32_t)P.nblk;
            if (abort_loop) break;
        }
        __syncthreads();

        // ---- iteration-1 check: top == bot (and zeros) (mod.rs:701-750) ----
        if (iteration == 1) {
            int eq = 1, small = 1;
            for (int i = tid; i < n; i += NTH) {
                const J2 tp = top[i];
                const Herm b = bot[i];
                const J2 bj = J2{{b.a, 0.0}, b.b, conj(b.b), {b.d, 0.0}};
                const J2 df = tp - bj;
                const double e[8] = {df.a.re, df.a.im, df.b.re, df.b.im, df.c.re, df.c.im, df.d.re, df.d.im};
                for (int k = 0; k < 8; k++)
                    if (fabs(e[k]) > P.stop) eq = 0;
                const double tv[8] = {tp.a.re, tp.a.im, tp.b.re, tp.b.im, tp.c.re, tp.c.im, tp.d.re, tp.d.im};
                const double bv[8] = {bj.a.re, bj.a.im, bj.b.re, bj.b.im, bj.c.re, bj.c.im, bj.d.re, bj.d.im};
                for (int k = 0; k < 8; k++)
                    if (fabs(tv[k]) > 2.220446049250313e-16 || fabs(bv[k]) > 2.220446049250313e-16) small = 0;
            }
            const int all_eq = __syncthreads_and(eq);
            const int all_small = __syncthreads_and(small);
            if (all_eq) {
                if (all_small)
                    for (int i = tid; i < n; i += NTH) failed[i] = 1;
                __syncthreads();
                break;
            }
        }

        // ---- new gains (mod.rs:753-778) ----
        for (int i = tid; i < n; i += NTH) {
            if (failed[i]) continue;
            const Herm b = bot[i];
            const J2 bj = J2{{b.a, 0.0}, b.b, conj(b.b), {b.d, 0.0}};
            const J2 div = jdiv(top[i], bj, P.pols);
            if (any_nan(div)) {
                failed[i] = 1;
                G[i] = jzero();
                Gold[i] = jzero();
            } else {
                G[i] = div;
            }
        }
        int my_failed = 0;
        for (int i = tid; i < n; i += NTH) my_failed += failed[i];
        __shared__ int s_count;
        if (tid == 0) s_count = 0;
        __syncthreads();
        if (my_failed) atomicAdd(&s_count, my_failed);
        __syncthreads();
        const int nfail = s_count;
        if (n - nfail <= 4) break;

        // ---- even iterations: precision, average, convergence (mod.rs:787-840) ----
        if (iteration % 2 == 0) {
            int below = 1;
            for (int i = tid; i < n; i += NTH) {
                if (!failed[i]) {
                    const J2 g = G[i], o = Gold[i];
                    const J2 df = g - o;
                    prec[4 * i + 0] = cnorm(df.a);
                    prec[4 * i + 1] = cnorm(df.b);
                    prec[4 * i + 2] = cnorm(df.c);
                    prec[4 * i + 3] = cnorm(df.d);
                    G[i] = (g + o) * 0.5;
                }
                for (int k = 0; k < 4; k++)
                    if (!(prec[4 * i + k] < P.stop)) below = 0;
            }
            if (__syncthreads_and(below)) break;
        }
        for (int i = tid; i < n; i += NTH) Gold[i] = G[i];
        __syncthreads();
    }
    __syncthreads();
    // the ring's copies still in flight land before the CTA leaves: the
    // last copy issued to each slot (copies to one slot complete in order)
    if (use_ring && tid == 0) {
        for (int st = 0; st < P.nring; st++)
            if (ring_cnt[st] > 0) mbar_wait_bounded(&ring_bar[st], (ring_cnt[st] - 1) & 1u, P.err);
    }
    __syncthreads();

    // ---- finalise (mod.rs:843-893) ----
    __shared__ double s_max[NTH / 32];
    __shared__ int s_nfail;
    if (tid == 0) s_nfail = 0;
    __syncthreads();
    double mx = -1.7976931348623157e308;  // f64::MIN
    int nf_local = 0;
    for (int i = tid; i < n; i += NTH) {
        if (failed[i]) {
            nf_local++;
            continue;
        }
        for (int k = 3; k >= 0; k--) mx = fmax(mx, prec[4 * i + k]);  // fmax ignores NaN like f64::max
    }
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if (lane == 0) s_max[tid >> 5] = mx;
    if (nf_local) atomicAdd(&s_nfail, nf_local);
    __syncthreads();
    double max_precision = s_max[0];
    for (int w = 1; w < NTH / 32; w++) max_precision = fmax(max_precision, s_max[w]);
    const int num_failed = s_nfail;
    const bool converged = !abort_loop && !(n - num_failed <= 4 || max_precision > P.min_thr);
    const double qnan = __longlong_as_double(0x7ff8000000000000ll);
    for (int i = tid; i < n; i += NTH) {
        JonesF64 out;
        if (!converged || failed[i])
            out = JonesF64{qnan, qnan, qnan, qnan, qnan, qnan, qnan, qnan};
        else
            out = store_j(G[i]);
        P.di_jones[(size_t)i * P.nchan + ch] = out;
    }
    if (tid == 0) P.results[ch] = HdcCalResult{iteration, converged ? 1 : 0, max_precision, num_failed};
}

// Seed failed chanblocks from converged neighbours (mod.rs:473-520):
// pairs (l, r) with l = -1 for a leading run of failures.
__global__ void retry_seed_kernel(JonesF64* dj, int nchan, int ntiles, const int2* pairs, int npairs) {
    const int tile = blockIdx.x * blockDim.x + threadIdx.x;
    if (tile >= ntiles) return;
    for (int k = 0; k < npairs; k++) {
        const int l = pairs[k].x, r = pairs[k].y;
        const J2 rs = load_j(dj[(size_t)tile * nchan + r]);
        if (l >= 0) {
            const J2 ls = load_j(dj[(size_t)tile * nchan + l]);
            for (int i = l + 1; i < r; i++) {
                const double lw = (double)(r - i), rw = (double)(i - l), d = (double)(r - l);
                const J2 s = ls * lw + rs * rw;
                dj[(size_t)tile * nchan + i] =
                    JonesF64{s.a.re / d, s.a.im / d, s.b.re / d, s.b.im / d, s.c.re / d, s.c.im / d, s.d.re / d, s.d.im / d};
            }
        } else {
            for (int i = 0; i < r; i++) dj[(size_t)tile * nchan + i] = store_j(rs);
        }
    }
}

// Per-chanblock calibration residual sum_{t,bl} ||D - G_p M G_q^H||_F^2 for
// the gains in dj [tile][chanblock] (used to judge a proposed starting point
// against the identity start).  One CTA per chanblock.
__global__ void __launch_bounds__(CT) residual_kernel(const CalParams P, const JonesF64* dj, double* out) {
    const int ch = blockIdx.x;
    const int nt = P.t1 - P.t0;
    const size_t tstride = (size_t)P.nchan * P.nbl;
    const JonesF32* D0 = P.data + ((size_t)P.t0 * P.nchan + ch) * P.nbl;
    const JonesF32* M0 = P.model + ((size_t)P.t0 * P.nchan + ch) * P.nbl;
    double acc = 0.0;
    for (int bl = threadIdx.x; bl < P.nbl; bl += CT) {
        int p, q;
        baseline_to_tiles(bl, P.ntiles, p, q);
        const J2 gp = load_j(dj[(size_t)p * P.nchan + ch]);
        const J2 gqh = herm(load_j(dj[(size_t)q * P.nchan + ch]));
        for (int t = 0; t < nt; t++) {
            const J2 r = load_vis(D0 + t * tstride + bl) - (gp * load_vis(M0 + t * tstride + bl)) * gqh;
            acc += cnorm(r.a) + cnorm(r.b) + cnorm(r.c) + cnorm(r.d);
        }
    }
    __shared__ double red[CT / 32];
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < CT / 32; w++) s += red[w];
        out[ch] = s;
    }
}

// Device-side judge of a proposed start: one pass over the timeblock forms
// the calibration residuals of the proposal dprop and of the identity start
// together; the proposal is kept (use[ch] = 1) where its residual is finite
// and no larger, and the chosen start is written to dstart [tile][chanblock].
__global__ void __launch_bounds__(CT) judge_kernel(const CalParams P, const JonesF64* dprop, JonesF64* dstart,
                                                   int* use) {
    const int ch = blockIdx.x;
    const int nt = P.t1 - P.t0;
    const size_t tstride = (size_t)P.nchan * P.nbl;
    const JonesF32* D0 = P.data + ((size_t)P.t0 * P.nchan + ch) * P.nbl;
    const JonesF32* M0 = P.model + ((size_t)P.t0 * P.nchan + ch) * P.nbl;
    double acc_p = 0.0, acc_i = 0.0;
    for (int bl = threadIdx.x; bl < P.nbl; bl += CT) {
        int p, q;
        baseline_to_tiles(bl, P.ntiles, p, q);
        const J2 gp = load_j(dprop[(size_t)p * P.nchan + ch]);
        const J2 gqh = herm(load_j(dprop[(size_t)q * P.nchan + ch]));
        for (int t = 0; t < nt; t++) {
            const J2 d = load_vis(D0 + t * tstride + bl), m = load_vis(M0 + t * tstride + bl);
            const J2 r = d - (gp * m) * gqh;
            const J2 ri = d - m;
            acc_p += cnorm(r.a) + cnorm(r.b) + cnorm(r.c) + cnorm(r.d);
            acc_i += cnorm(ri.a) + cnorm(ri.b) + cnorm(ri.c) + cnorm(ri.d);
        }
    }
    __shared__ double red[2][CT / 32];
    __shared__ int keep;
    for (int o = 16; o > 0; o >>= 1) {
        acc_p += __shfl_xor_sync(0xffffffffu, acc_p, o);
        acc_i += __shfl_xor_sync(0xffffffffu, acc_i, o);
    }
    if ((threadIdx.x & 31) == 0) {
        red[0][threadIdx.x >> 5] = acc_p;
        red[1][threadIdx.x >> 5] = acc_i;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double sp = 0.0, si = 0.0;
        for (int w = 0; w < CT / 32; w++) {
            sp += red[0][w];
            si += red[1][w];
        }
        keep = isfinite(sp) && sp <= si;
        if (use) use[ch] = keep;
    }
    __syncthreads();
    for (int t = threadIdx.x; t < P.ntiles; t += CT) {
        const size_t i = (size_t)t * P.nchan + ch;
        dstart[i] = keep ? dprop[i] : JonesF64{1.0, 0.0, 0.0, 0.0, 0.0, 0.0, 1.0, 0.0};
    }
}

int launch_judge(const JonesF32* d_data, const JonesF32* d_model, int t0, int t1, int nchan, int nbl, int ntiles,
                 const JonesF64* d_prop, JonesF64* d_start, int* d_use, cudaStream_t s) {
    CalParams P = {};
    P.data = d_data;
    P.model = d_model;
    P.t0 = t0;
    P.t1 = t1;
    P.nchan = nchan;
    P.nbl = nbl;
    P.ntiles = ntiles;
    judge_kernel<<<nchan, CT, 0, s>>>(P, d_prop, d_start, d_use);
    count_launches(1);
    HDC_CUDA_RET_INT(cudaGetLastError());
    return HDC_OK;
}

static size_t smem_base_bytes(int n, int form) {
    const size_t base = (size_t)n * (3 * sizeof(J2) + 2 * sizeof(Herm) + 4 * sizeof(double)) +
                        sizeof(int) * (size_t)((n + 1) & ~1);
    // collapsed forms: column partial sums; FP32 form: group 1's accumulators
    return base + (form != HDC_CAL_PLAIN ? 16 * 16 * 12 * sizeof(double) : 0) +
           (form == HDC_CAL_COLLAPSED_F32 ? (size_t)n * (sizeof(J2) + sizeof(Herm)) : 0);
}

constexpr size_t SMEM_LIMIT = 227 * 1024;
constexpr size_t RING_SLOT = (size_t)NCOV * BLK * sizeof(float);

// ring depth of the FP32 collapsed form: 3 slots where they fit, else 2,
// else direct loads
static int ring_depth(int n, int form) {
    if (form != HDC_CAL_COLLAPSED_F32) return 0;
    for (int r = 3; r >= 2; r--)
        if (smem_base_bytes(n, form) + 16 + r * RING_SLOT <= SMEM_LIMIT) return r;
    return 0;
}

static size_t smem_bytes(int n, int form) {
    const int r = ring_depth(n, form);
    return smem_base_bytes(n, form) + (r ? 16 + r * RING_SLOT : 0);
}

template <int FORM>
static int launch_mitchcal_form(const CalParams& P, int nblocks, cudaStream_t s) {
    const size_t sm = smem_bytes(P.ntiles, FORM);
    HDC_CUDA_RET_INT(
        cudaFuncSetAttribute(mitchcal_kernel<FORM>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    mitchcal_kernel<FORM><<<nblocks, cal_threads(FORM), sm, s>>>(P);
    count_launches(1);
    HDC_CUDA_RET_INT(cudaGetLastError());
    return HDC_OK;
}

// Launch without setting the shared-memory attribute (inside a stream
// capture, after prepare_mitchcal has set it).
static void launch_mitchcal_captured(const CalParams& P, int form, int nblocks, cudaStream_t s) {
    const size_t sm = smem_bytes(P.ntiles, form);
    if (form == HDC_CAL_COLLAPSED)
        mitchcal_kernel<1><<<nblocks, cal_threads(1), sm, s>>>(P);
    else if (form == HDC_CAL_COLLAPSED_F32)
        mitchcal_kernel<2><<<nblocks, cal_threads(2), sm, s>>>(P);
    else
        mitchcal_kernel<0><<<nblocks, cal_threads(0), sm, s>>>(P);
    count_launches(1);
}

static int prepare_mitchcal(int ntiles, int form) {
    const int sm = (int)smem_bytes(ntiles, form);
    if (form == HDC_CAL_COLLAPSED)
        HDC_CUDA_RET_INT(cudaFuncSetAttribute(mitchcal_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
    else if (form == HDC_CAL_COLLAPSED_F32)
        HDC_CUDA_RET_INT(cudaFuncSetAttribute(mitchcal_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
    else
        HDC_CUDA_RET_INT(cudaFuncSetAttribute(mitchcal_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
    return HDC_OK;
}

__global__ void identity_kernel(JonesF64* dj, size_t n) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dj[i] = JonesF64{1.0, 0.0, 0.0, 0.0, 0.0, 0.0, 1.0, 0.0};
}

static void launch_collapse(const CalParams& P, int form, void* cov, cudaStream_t s) {
    const dim3 grid(2 * P.nblk, P.nchan);
    if (form == HDC_CAL_COLLAPSED)
        collapse_kernel<double><<<grid, BLK / 2, 0, s>>>(P, static_cast<double*>(cov));
    else
        collapse_kernel<float><<<grid, BLK / 2, 0, s>>>(P, static_cast<float*>(cov));
    count_launches(1);
}

// A non-blocking stream per device on which the multi-timeblock graph is
// captured (capture is not possible on the legacy default stream).
static std::mutex g_cs_mu;
static cudaStream_t g_cs[16] = {nullptr};

static cudaStream_t capture_stream() {
    std::lock_guard<std::mutex> lk(g_cs_mu);
    int d = 0;
    if (cudaGetDevice(&d) != cudaSuccess || d < 0 || d >= 16) return nullptr;
    if (!g_cs[d] && cudaStreamCreateWithFlags(&g_cs[d], cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    return g_cs[d];
}

static int launch_mitchcal(const CalParams& P, int form, int nblocks, cudaStream_t s) {
    if (form == HDC_CAL_COLLAPSED) return launch_mitchcal_form<1>(P, nblocks, s);
    if (form == HDC_CAL_COLLAPSED_F32) return launch_mitchcal_form<2>(P, nblocks, s);
    return launch_mitchcal_form<0>(P, nblocks, s);
}

// Grow-only per-device buffer for the collapsed covariances.
static std::mutex g_cov_mu;
static void* g_cov[16] = {nullptr};
static size_t g_cov_size[16] = {0};

static void* covariance_buffer(size_t bytes) {
    std::lock_guard<std::mutex> lk(g_cov_mu);
    int d = 0;
    if (cudaGetDevice(&d) != cudaSuccess || d < 0 || d >= 16) return nullptr;
    if (g_cov_size[d] < bytes) {
        if (g_cov[d]) {
            cudaDeviceSynchronize();  // queued work may still read the old buffer
            cudaFree(g_cov[d]);
            g_cov[d] = nullptr;
            g_cov_size[d] = 0;
        }
        if (cudaMalloc(&g_cov[d], bytes) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        g_cov_size[d] = bytes;
    }
    return g_cov[d];
}

// Retry failed chanblocks from interpolated neighbours (mod.rs:468-614):
// res holds the first pass's results (read back); P.results/P.di_jones point
// at this timeblock's device results and solutions; for the collapsed forms
// P.cov must hold this timeblock's covariances.
static int retry_failed(CalParams P, int form, std::vector<HdcCalResult>& res, int* d_list, int2* d_pairs,
                        cudaStream_t s) {
    int rc = HDC_OK;
    int total = 0;
    for (auto& r : res) total += r.converged;
    if (total > 0 && total != P.nchan) {
        int new_conv = 1;
        while (new_conv > 0 && total != P.nchan) {
            std::vector<int2> pairs;
            int left = -1;
            bool in_fail = false;
            for (int c = 0; c < P.nchan; c++) {
                const bool conv = res[c].converged != 0;
                if (!in_fail && conv)
                    left = c;
                else if (!in_fail && !conv)
                    in_fail = true;
                else if (in_fail && conv) {
                    in_fail = false;
                    pairs.push_back(make_int2(left, c));
                    left = c;
                }
            }
            std::vector<int> list;
            for (int c = 0; c < P.nchan; c++)
                if (!res[c].converged) list.push_back(c);
            if (!pairs.empty()) {
                cudaMemcpyAsync(d_pairs, pairs.data(), sizeof(int2) * pairs.size(), cudaMemcpyHostToDevice, s);
                retry_seed_kernel<<<(P.ntiles + 127) / 128, 128, 0, s>>>(P.di_jones, P.nchan, P.ntiles, d_pairs,
                                                                        (int)pairs.size());
                count_launches(1);
            }
            cudaMemcpyAsync(d_list, list.data(), sizeof(int) * list.size(), cudaMemcpyHostToDevice, s);
            P.chan_list = d_list;
            rc = launch_mitchcal(P, form, (int)list.size(), s);
            if (rc) return rc;
            if (cudaMemcpyAsync(res.data(), P.results, sizeof(HdcCalResult) * P.nchan, cudaMemcpyDeviceToHost,
                                s) != cudaSuccess ||
                cudaStreamSynchronize(s) != cudaSuccess) {
                set_error("calibration retry: %s", cudaGetErrorString(cudaGetLastError()));
                return HDC_ERR_CUDA;
            }
            for (int c : list)
                if (std::fabs(res[c].max_precision) > 1e100) res[c].max_precision = NAN;
            int tmp = 0;
            for (auto& r : res) tmp += r.converged;
            new_conv = tmp - total;
            total = tmp;
        }
    }
    return rc;
}

}  // namespace hdc

using namespace hdc;

// calibrate_timeblock's body: the first pass over every chanblock (or over
// the listed ones, whose results alone are written), then -- with `retry` --
// the retry of failed chanblocks from interpolated neighbours.
static int calibrate_timeblock_impl(const JonesF32* d_data_tfb, const JonesF32* d_model_tfb, int num_timesteps,
                                    int timeblock_start, int timeblock_end, int num_chanblocks, int num_baselines,
                                    JonesF64* d_di_jones, int max_iterations, double stop_threshold,
                                    double min_threshold, int pols, HdcCalResult* h_results, int form, bool retry,
                                    const int* h_list, int num_listed, cudaStream_t s) {
    const int ntiles = (int)((1.0 + std::sqrt(1.0 + 8.0 * num_baselines)) / 2.0 + 0.5);
    if (ntiles * (ntiles - 1) / 2 != num_baselines || ntiles > CT || num_chanblocks <= 0 ||
        timeblock_start < 0 || timeblock_end > num_timesteps || timeblock_start >= timeblock_end || !h_results ||
        pols < 0 || pols > 4) {
        set_error("hdc_calibrate_timeblock: invalid arguments (baselines %d -> %d tiles, max %d)", num_baselines,
                  ntiles, CT);
        return HDC_ERR_ARG;
    }
    if (form != HDC_CAL_PLAIN && form != HDC_CAL_COLLAPSED && form != HDC_CAL_COLLAPSED_F32) {
        set_error("hdc_calibrate_timeblock: unknown form %d", form);
        return HDC_ERR_ARG;
    }
    HdcCalResult* d_res = nullptr;
    int* d_list = nullptr;
    int2* d_pairs = nullptr;
    int rc = HDC_OK;
    auto cleanup = [&]() {
        if (d_res) cudaFree(d_res);
        if (d_list) cudaFree(d_list);
        if (d_pairs) cudaFree(d_pairs);
    };
    if (cudaMalloc(&d_res, sizeof(HdcCalResult) * num_chanblocks) != cudaSuccess ||
        cudaMalloc(&d_list, sizeof(int) * num_chanblocks) != cudaSuccess ||
        cudaMalloc(&d_pairs, sizeof(int2) * (num_chanblocks + 1)) != cudaSuccess) {
        cudaGetLastError();
        cleanup();
        set_error("hdc_calibrate_timeblock: device allocation failed");
        return HDC_ERR_ALLOC;
    }
    CalParams P;
    P.data = d_data_tfb;
    P.model = d_model_tfb;
    P.t0 = timeblock_start;
    P.t1 = timeblock_end;
    P.nchan = num_chanblocks;
    P.nbl = num_baselines;
    P.ntiles = ntiles;
    P.di_jones = d_di_jones;
    P.chan_list = nullptr;
    P.max_iter = max_iterations;
    P.stop = stop_threshold;
    P.min_thr = min_threshold;
    P.pols = pols;
    P.results = d_res;
    P.cov = nullptr;
    P.nblk = cov_blocks(ntiles);
    P.nring = ring_depth(ntiles, form);
    P.err = device_error_word();
    if (form != HDC_CAL_PLAIN) {
        const size_t elem = form == HDC_CAL_COLLAPSED ? sizeof(double) : sizeof(float);
        void* cov = covariance_buffer(elem * NCOV * BLK * (size_t)num_chanblocks * P.nblk);
        if (!cov) {
            cleanup();
            set_error("hdc_calibrate_timeblock: covariance allocation failed");
            return HDC_ERR_ALLOC;
        }
        P.cov = cov;
        launch_collapse(P, form, cov, s);
        if (cudaGetLastError() != cudaSuccess) {
            cleanup();
            set_error("hdc_calibrate_timeblock: collapse launch failed");
            return HDC_ERR_CUDA;
        }
    }
    int nblocks = num_chanblocks;
    if (h_list) {
        for (int k = 0; k < num_listed; k++)
            if (h_list[k] < 0 || h_list[k] >= num_chanblocks) {
                cleanup();
                set_error("hdc_calibrate_chanblocks: chanblock %d of the list is outside 0..%d", h_list[k],
                          num_chanblocks - 1);
                return HDC_ERR_ARG;
            }
        if (num_listed == 0) {
            cleanup();
            return HDC_OK;
        }
        if (cudaMemcpyAsync(d_list, h_list, sizeof(int) * num_listed, cudaMemcpyHostToDevice, s) != cudaSuccess) {
            cleanup();
            set_error("hdc_calibrate_chanblocks: %s", cudaGetErrorString(cudaGetLastError()));
            return HDC_ERR_CUDA;
        }
        P.chan_list = d_list;
        nblocks = num_listed;
    }
    rc = launch_mitchcal(P, form, nblocks, s);
    if (rc) {
        cleanup();
        return rc;
    }
    std::vector<HdcCalResult> res(num_chanblocks);
    if (cudaMemcpyAsync(res.data(), d_res, sizeof(HdcCalResult) * num_chanblocks, cudaMemcpyDeviceToHost, s) !=
            cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess) {
        cleanup();
        set_error("hdc_calibrate_timeblock: %s", cudaGetErrorString(cudaGetLastError()));
        return HDC_ERR_CUDA;
    }
    if (form == HDC_CAL_COLLAPSED_F32 && take_device_error(s)) {
        cleanup();
        set_error("hdc_calibrate_timeblock: a covariance copy did not arrive in time");
        return HDC_ERR_TIMEOUT;
    }
    if (retry) {
        rc = retry_failed(P, form, res, d_list, d_pairs, s);
        if (rc) {
            cleanup();
            return rc;
        }
    }
    if (h_list) {
        for (int k = 0; k < num_listed; k++) {
            HdcCalResult r = res[h_list[k]];
            if (std::fabs(r.max_precision) > 1e100) r.max_precision = NAN;
            h_results[h_list[k]] = r;
        }
    } else {
        for (int c = 0; c < num_chanblocks; c++) h_results[c] = res[c];
    }
    cleanup();
    return HDC_OK;
}

extern "C" int hdc_calibrate_timeblock(const JonesF32* d_data_tfb, const JonesF32* d_model_tfb, int num_timesteps,
                                       int timeblock_start, int timeblock_end, int num_chanblocks, int num_baselines,
                                       JonesF64* d_di_jones, int max_iterations, double stop_threshold,
                                       double min_threshold, int pols, HdcCalResult* h_results, int form,
                                       hdcStream_t stream) {
    return calibrate_timeblock_impl(d_data_tfb, d_model_tfb, num_timesteps, timeblock_start, timeblock_end,
                                    num_chanblocks, num_baselines, d_di_jones, max_iterations, stop_threshold,
                                    min_threshold, pols, h_results, form, true, nullptr, 0, (cudaStream_t)stream);
}

extern "C" int hdc_calibrate_chanblocks(const JonesF32* d_data_tfb, const JonesF32* d_model_tfb, int num_timesteps,
                                        int timeblock_start, int timeblock_end, int num_chanblocks,
                                        int num_baselines, JonesF64* d_di_jones, int max_iterations,
                                        double stop_threshold, double min_threshold, int pols,
                                        const int* h_chanblock_list, int num_listed, HdcCalResult* h_results,
                                        int form, hdcStream_t stream) {
    if (h_chanblock_list == nullptr && num_listed != 0) {
        set_error("hdc_calibrate_chanblocks: a count without a list");
        return HDC_ERR_ARG;
    }
    return calibrate_timeblock_impl(d_data_tfb, d_model_tfb, num_timesteps, timeblock_start, timeblock_end,
                                    num_chanblocks, num_baselines, d_di_jones, max_iterations, stop_threshold,
                                    min_threshold, pols, h_results, form, false, h_chanblock_list, num_listed,
                                    (cudaStream_t)stream);
}

// All timeblocks of an observation (calibrate_timeblocks, mod.rs:272-361):
// the first pass of every timeblock (identity start, collapse for the
// collapsed forms, the persistent MitchCal kernel over all chanblocks) is
// captured once into a CUDA graph and launched as one unit; the host reads
// every timeblock's results once, then runs the reference's retry of failed
// chanblocks per timeblock where it applies (outside the graph: its shape
// depends on which chanblocks failed).
extern "C" int hdc_calibrate_timeblocks(const JonesF32* d_data_tfb, const JonesF32* d_model_tfb, int num_timesteps,
                                        const int* h_timeblock_bounds, int num_timeblocks, int num_chanblocks,
                                        int num_baselines, JonesF64* d_di_jones, int max_iterations,
                                        double stop_threshold, double min_threshold, int pols,
                                        HdcCalResult* h_results, int form, hdcStream_t stream) {
    cudaStream_t s = (cudaStream_t)stream;
    const int ntiles = (int)((1.0 + std::sqrt(1.0 + 8.0 * num_baselines)) / 2.0 + 0.5);
    bool ok = ntiles * (ntiles - 1) / 2 == num_baselines && ntiles <= CT && num_chanblocks > 0 &&
              num_timeblocks > 0 && h_timeblock_bounds && h_results && pols >= 0 && pols <= 4 &&
              (form == HDC_CAL_PLAIN || form == HDC_CAL_COLLAPSED || form == HDC_CAL_COLLAPSED_F32);
    for (int k = 0; ok && k < num_timeblocks; k++) {
        const int a = h_timeblock_bounds[2 * k], b = h_timeblock_bounds[2 * k + 1];
        ok = a >= 0 && b <= num_timesteps && a < b;
    }
    if (!ok) {
        set_error("hdc_calibrate_timeblocks: invalid arguments");
        return HDC_ERR_ARG;
    }
    const size_t nres = (size_t)num_timeblocks * num_chanblocks;
    const size_t nsol = (size_t)ntiles * num_chanblocks;
    HdcCalResult* d_res = nullptr;
    int* d_list = nullptr;
    int2* d_pairs = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    auto cleanup = [&]() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        if (d_res) cudaFree(d_res);
        if (d_list) cudaFree(d_list);
        if (d_pairs) cudaFree(d_pairs);
    };
    if (cudaMalloc(&d_res, sizeof(HdcCalResult) * nres) != cudaSuccess ||
        cudaMalloc(&d_list, sizeof(int) * num_chanblocks) != cudaSuccess ||
        cudaMalloc(&d_pairs, sizeof(int2) * (num_chanblocks + 1)) != cudaSuccess) {
        cudaGetLastError();
        cleanup();
        set_error("hdc_calibrate_timeblocks: device allocation failed");
        return HDC_ERR_ALLOC;
    }
    void* cov = nullptr;
    const int nblk = cov_blocks(ntiles), nring = ring_depth(ntiles, form);
    int* errw = device_error_word();
    if (form != HDC_CAL_PLAIN) {
        const size_t elem = form == HDC_CAL_COLLAPSED ? sizeof(double) : sizeof(float);
        cov = covariance_buffer(elem * NCOV * BLK * (size_t)num_chanblocks * nblk);
        if (!cov) {
            cleanup();
            set_error("hdc_calibrate_timeblocks: covariance allocation failed");
            return HDC_ERR_ALLOC;
        }
    }
    int rc = prepare_mitchcal(ntiles, form);
    cudaStream_t cs = capture_stream();
    if (rc || !cs) {
        cleanup();
        if (!rc) set_error("hdc_calibrate_timeblocks: no capture stream");
        return rc ? rc : HDC_ERR_CUDA;
    }
    auto params = [&](int k) {
        CalParams P = {};
        P.data = d_data_tfb;
        P.model = d_model_tfb;
        P.t0 = h_timeblock_bounds[2 * k];
        P.t1 = h_timeblock_bounds[2 * k + 1];
        P.nchan = num_chanblocks;
        P.nbl = num_baselines;
        P.ntiles = ntiles;
        P.di_jones = d_di_jones + (size_t)k * nsol;
        P.chan_list = nullptr;
        P.max_iter = max_iterations;
        P.stop = stop_threshold;
        P.min_thr = min_threshold;
        P.pols = pols;
        P.results = d_res + (size_t)k * num_chanblocks;
        P.cov = cov;
        P.nblk = nblk;
        P.nring = nring;
        P.err = errw;
        return P;
    };
    cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
        for (int k = 0; k < num_timeblocks; k++) {
            const CalParams P = params(k);
            identity_kernel<<<(unsigned)((nsol + 255) / 256), 256, 0, cs>>>(P.di_jones, nsol);
            count_launches(1);
            if (form != HDC_CAL_PLAIN) launch_collapse(P, form, cov, cs);
            launch_mitchcal_captured(P, form, num_chanblocks, cs);
        }
        const cudaError_t le = cudaGetLastError();
        e = cudaStreamEndCapture(cs, &graph);
        if (e == cudaSuccess) e = le;
    }
    if (e == cudaSuccess) e = cudaGraphInstantiate(&exec, graph, 0);
    if (e == cudaSuccess) e = cudaGraphLaunch(exec, s);
    std::vector<HdcCalResult> res(nres);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(res.data(), d_res, sizeof(HdcCalResult) * nres, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        cleanup();
        set_error("hdc_calibrate_timeblocks: %s", cudaGetErrorString(e));
        return HDC_ERR_CUDA;
    }
    if (form == HDC_CAL_COLLAPSED_F32 && take_device_error(s)) {
        cleanup();
        set_error("hdc_calibrate_timeblocks: a covariance copy did not arrive in time");
        return HDC_ERR_TIMEOUT;
    }
    for (int k = 0; k < num_timeblocks; k++) {
        std::vector<HdcCalResult> rk(res.begin() + (size_t)k * num_chanblocks,
                                     res.begin() + (size_t)(k + 1) * num_chanblocks);
        int conv = 0;
        for (auto& r : rk) conv += r.converged;
        if (conv > 0 && conv != num_chanblocks) {
            const CalParams P = params(k);
            if (form != HDC_CAL_PLAIN) launch_collapse(P, form, cov, s);  // this timeblock's covariances
            rc = retry_failed(P, form, rk, d_list, d_pairs, s);
            if (rc) {
                cleanup();
                return rc;
            }
        }
        for (int c = 0; c < num_chanblocks; c++) h_results[(size_t)k * num_chanblocks + c] = rk[c];
    }
    cleanup();
    return HDC_OK;
}

extern "C" int hdc_calibration_residuals(const JonesF32* d_data_tfb, const JonesF32* d_model_tfb, int num_timesteps,
                                         int timeblock_start, int timeblock_end, int num_chanblocks, int num_baselines,
                                         const JonesF64* d_di_jones, double* h_residuals, hdcStream_t stream) {
    cudaStream_t s = (cudaStream_t)stream;
    const int ntiles = (int)((1.0 + std::sqrt(1.0 + 8.0 * num_baselines)) / 2.0 + 0.5);
    if (ntiles * (ntiles - 1) / 2 != num_baselines || timeblock_start < 0 || timeblock_end > num_timesteps ||
        timeblock_start >= timeblock_end || num_chanblocks <= 0 || !h_residuals) {
        set_error("hdc_calibration_residuals: invalid arguments");
        return HDC_ERR_ARG;
    }
    double* d_out = nullptr;
    HDC_CUDA_RET_INT(cudaMalloc(&d_out, sizeof(double) * num_chanblocks));
    CalParams P = {};
    P.data = d_data_tfb;
    P.model = d_model_tfb;
    P.t0 = timeblock_start;
    P.t1 = timeblock_end;
    P.nchan = num_chanblocks;
    P.nbl = num_baselines;
    P.ntiles = ntiles;
    residual_kernel<<<num_chanblocks, CT, 0, s>>>(P, d_di_jones, d_out);
    count_launches(1);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(h_residuals, d_out, sizeof(double) * num_chanblocks, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaFree(d_out);
    if (e != cudaSuccess) {
        set_error("hdc_calibration_residuals: %s", cudaGetErrorString(e));
        return HDC_ERR_CUDA;
    }
    return HDC_OK;
}
