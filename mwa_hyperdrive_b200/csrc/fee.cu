// MWA FEE beam on the device: per-tile Jones matrices from the
// spherical-wave expansion of the dipoles' embedded element patterns.
//
// The reference takes them from mwa_hyperbeam 0.11.0 (a crates.io
// dependency, not part of the reference tree): FEEBeam::gpu_prepare and
// FEEBeamGpu::calc_jones_device_pair_inner, called from beam/fee.rs:307-349
// and read by the predict kernels as [uniq tile][uniq freq][direction]
// (model/gpu.rs:889-910, gpu/model.cu:114-123).  The model is that of
// Sokolowski et al. 2017 (PASA 34, e062).  For one polarisation with the
// beamformed coefficients Q1_mn, Q2_mn (the file's s = 1 and s = 2 modes,
// summed over the 16 dipoles with each dipole's amplitude and delay phase
// exp(-2 pi i f tau), tau = delay x 435 ps):
//   sigma_T = sum_mn K_mn e^{i m phi} (P1sin (|m| Q2 u - m Q1) + Q2 P1)
//   sigma_P = sum_mn K_mn e^{i m phi} j (P1sin (m Q2 - |m| Q1 u) - Q1 P1)
//   K_mn = C_mn (-m/|m|)^m j^n / sqrt(n (n + 1)),
//   C_mn = sqrt((2n + 1)/2 (n - |m|)! / (n + |m|)!)
// with u = cos theta, theta = za, phi = pi/2 - az, P1sin = P_n^|m|(u) /
// sin theta and P1 = dP_n^|m|(cos theta) / d theta (associated Legendre
// functions with the Condon-Shortley phase; (-m/|m|)^m is 1 for m <= 0).
// The polarisation's Jones row is (sigma_T, -sigma_P); rows X then Y.  With
// norm_to_zenith every element is divided by the magnitude of the same
// element of the zenith-pointed beam at the zenith, taken at the azimuth
// where it peaks (phi = 0, -pi/2, pi/2, 0).  With a latitude the matrix is
// rotated by the parallactic angle + pi/2 (ERFA ae2hd and hd2pa, as marlu's
// AzEl::to_hadec and HADec::get_parallactic_angle).
//
// Device layout.  K_mn is folded into the coefficients on the host, and the
// records of a (tile, frequency) set are stored in the order the kernel
// visits them (|m| outer, n inner), every set laid out for the beam's largest
// degree.  The modes +m and -m of one degree share P1sin, P1 and
// e^{-i m phi} = conj(e^{i m phi}), so they are stored as the sums and
// differences of their coefficients and added together:
//   e (a q1+ + b q2+) + conj(e) (-a q1- + b q2-)
//     = Re(e) (a M1 + b P2) + i Im(e) (a P1 + b M2),  P = q+ + q-, M = q+ - q-
// (a = -|m| P1sin, b = |m| u P1sin + P1), which with Re(e) a, Re(e) b,
// Im(e) a and Im(e) b formed once is 16 fused multiply-adds per polarisation
// for the two modes.  A thread sums one set at two directions, so every
// record it loads (all threads of a block read the same one: one L1
// broadcast per warp) serves both.  Per direction and |m| it runs one upward
// Legendre recurrence in n of R_n^|m| = P_n^|m| / sin^|m| theta (a
// polynomial in u, finite at the zenith), one degree ahead, for
//   P1sin = sin^{|m|-1} R_n,
//   P1 = sin^{|m|-1} ((n - |m| + 1) R_{n+1} - (n + 1) u R_n)
// (the m = 0 modes: P1 = P_n^1 = sin theta R_n^1), with no division.  The
// recurrence constants come from a small table.  The work is FP64
// arithmetic; the roofline counts the published sum's 56 FLOPs per mode per
// direction (both polarisations).

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "common.cuh"

namespace hdc {

constexpr int FEE_MAX_N = 64;              // largest mode degree n supported
constexpr double FEE_DELAY_STEP = 435e-12; // seconds per delay step
constexpr uint32_t FEE_DEAD_DELAY = 32;    // delay value marking a dead dipole
constexpr int FEE_BLOCK = 128;

// One 64-byte coefficient record (K_mn folded in).  The records of a set are
// stored in the order the kernel visits them: for |m| = 1 .. nmax, for
// n = |m| .. nmax: (for |m| = 1 only) the m = 0 mode of degree n as
// (q1 X, q2 X, q1 Y, q2 Y), then the pair +|m|, -|m| of degree n as two
// records, X then Y, each (P1, M1, P2, M2) with P = q(+m) + q(-m) and
// M = q(+m) - q(-m).
struct FeeMode {
    double2 c0, c1, c2, c3;
};

// Records of a set whose largest degree is nmax: n = 1..nmax, m = -n..n.
inline int fee_num_modes(int nmax) { return nmax * (nmax + 2); }

// Per (n, |m|) constants of the column recurrence: n + 1 and n - |m| + 1 (the
// derivative identity) and the coefficients that take R^|m| from degrees
// n, n + 1 to n + 2: (2n+3)/(n+2-|m|) and (n+1+|m|)/(n+2-|m|).
struct FeeRec {
    double c1, c2, al, be;
};

struct FeeSums {
    cplx tx, px, ty, py;  // sigma_T and sigma_P / j of the X and Y rows
};

__device__ __forceinline__ FeeMode ld_mode(const FeeMode* __restrict__ p) {
    return FeeMode{__ldg(&p->c0), __ldg(&p->c1), __ldg(&p->c2), __ldg(&p->c3)};
}

// An m = 0 mode (e = 1, a = 0, b = P1 = P_n^1): sigma_T += b q2,
// sigma_P / j += b q1.
__device__ __forceinline__ void fee_m0_add(const FeeMode& r, double b, FeeSums& s) {
    s.tx.re = fma(b, r.c1.x, s.tx.re);
    s.tx.im = fma(b, r.c1.y, s.tx.im);
    s.px.re = fma(b, r.c0.x, s.px.re);
    s.px.im = fma(b, r.c0.y, s.px.im);
    s.ty.re = fma(b, r.c3.x, s.ty.re);
    s.ty.im = fma(b, r.c3.y, s.ty.im);
    s.py.re = fma(b, r.c2.x, s.py.re);
    s.py.im = fma(b, r.c2.y, s.py.im);
}

// The pair +m, -m of one polarisation, record (P1, M1, P2, M2), with
// ra = Re(e) a, rb = Re(e) b, ia = Im(e) a, ib = Im(e) b (e = e^{i |m| phi},
// a = -|m| P1sin):
//   sigma_T     += Re(e) (a M1 + b P2) + i Im(e) (a P1 + b M2)
//   sigma_P / j += Re(e) (b P1 + a M2) + i Im(e) (b M1 + a P2)
// 16 fused multiply-adds.
__device__ __forceinline__ void fee_pair_add(const FeeMode& r, double ra, double rb, double ia, double ib, cplx& t,
                                             cplx& ph) {
    const double2 p1 = r.c0, m1 = r.c1, p2 = r.c2, m2 = r.c3;
    t.re = fma(ra, m1.x, fma(rb, p2.x, fma(-ia, p1.y, fma(-ib, m2.y, t.re))));
    t.im = fma(ra, m1.y, fma(rb, p2.y, fma(ia, p1.x, fma(ib, m2.x, t.im))));
    ph.re = fma(rb, p1.x, fma(ra, m2.x, fma(-ib, m1.y, fma(-ia, p2.y, ph.re))));
    ph.im = fma(rb, p1.y, fma(ra, m2.y, fma(ib, m1.x, fma(ia, p2.x, ph.im))));
}

// The mode sums of one coefficient set at D directions (theta[k], phi[k]).
// For each |m| one column of R_n^|m| = P_n^|m| / sin^|m| theta runs one
// degree ahead, and with x = cos theta, s = sin theta:
//   P1sin = s^{|m|-1} R_n,
//   P1 = dP_n^|m|/d theta = s^{|m|-1} ((n - |m| + 1) R_{n+1} - (n + 1) x R_n)
// (from (1 - x^2) dP_n^m/dx = (n + 1) x P_n^m - (n - m + 1) P_{n+1}^m), and
// the m = 0 modes take P1 = P_n^1 = s R_n^1 from the |m| = 1 column: one
// recurrence per (n, |m|), no division, exact at the zenith.  Every record
// and table entry a thread loads serves its D directions.  (Measured and
// not kept, on 4600 directions x 600 sets at degree 16: three Legendre
// columns per |m|, 3.3 ms; the coefficient records read one mode ahead in
// registers, 3.5 ms; four unique frequencies per thread at one direction,
// 3.3 ms; three directions per thread, 2.3 ms; this form, 1.74 ms.)
template <int D>
__device__ void fee_sums(const double (&theta)[D], const double (&phi)[D], const FeeMode* __restrict__ q, int nmax,
                         const FeeRec* __restrict__ rec, FeeSums (&out)[D]) {
    double s[D], x[D], sm1[D];
    cplx e1[D], em[D];
    FeeSums acc[D];
#pragma unroll
    for (int k = 0; k < D; k++) {
        double sph, cph;
        sincos(theta[k], &s[k], &x[k]);
        sincos(phi[k], &sph, &cph);
        e1[k] = cplx{cph, sph};
        em[k] = e1[k];  // e^{i |m| phi}, |m| = 1
        sm1[k] = 1.0;   // s^{|m|-1}
        acc[k] = FeeSums{{0, 0}, {0, 0}, {0, 0}, {0, 0}};
    }
    double rd = -1.0;  // R_|m|^|m| = (-1)^|m| (2|m|-1)!!
    const FeeMode* p = q;
    for (int ma = 1; ma <= nmax; ma++) {
        double cur[D], nxt[D];  // R_n and R_{n+1} of column |m|
#pragma unroll
        for (int k = 0; k < D; k++) {
            cur[k] = rd;
            nxt[k] = x[k] * (2.0 * ma + 1.0) * rd;
        }
        const FeeRec* r = rec + ma * (FEE_MAX_N + 1) + ma;  // row n = ma, column |m|
        for (int n = ma; n <= nmax; n++, r += FEE_MAX_N + 1) {
            const double2 c01 = __ldg(reinterpret_cast<const double2*>(r));  // (n + 1, n - |m| + 1)
            const double2 c23 = __ldg(reinterpret_cast<const double2*>(r) + 1);  // (al, be)
            const double4 c = make_double4(c01.x, c01.y, c23.x, c23.y);
            FeeMode m0;
            if (ma == 1) m0 = ld_mode(p++);
            const FeeMode rx = ld_mode(p), ry = ld_mode(p + 1);
            p += 2;
#pragma unroll
            for (int k = 0; k < D; k++) {
                const double p1sin = sm1[k] * cur[k];
                const double p1 = sm1[k] * fma(c.y, nxt[k], -c.x * x[k] * cur[k]);
                const double a = -ma * p1sin;
                const double b = fma(ma * x[k], p1sin, p1);
                if (ma == 1) fee_m0_add(m0, s[k] * cur[k], acc[k]);
                const double ra = em[k].re * a, rb = em[k].re * b, ia = em[k].im * a, ib = em[k].im * b;
                fee_pair_add(rx, ra, rb, ia, ib, acc[k].tx, acc[k].px);
                fee_pair_add(ry, ra, rb, ia, ib, acc[k].ty, acc[k].py);
                // R_{n+2} = al x R_{n+1} - be R_n
                const double t = fma(c.z * x[k], nxt[k], -c.w * cur[k]);
                cur[k] = nxt[k];
                nxt[k] = t;
            }
        }
        rd *= -(2.0 * ma + 1.0);
#pragma unroll
        for (int k = 0; k < D; k++) {
            sm1[k] *= s[k];
            em[k] = em[k] * e1[k];
        }
    }
#pragma unroll
    for (int k = 0; k < D; k++) out[k] = acc[k];
}

__device__ __forceinline__ J2 fee_jones(const FeeSums& s) {
    // rows (sigma_T, -sigma_P) with sigma_P = j (sigma_P / j)
    return J2{s.tx, cplx{-s.px.im, s.px.re}, s.ty, cplx{-s.py.im, s.py.re}};
}

// Rotation by the parallactic angle + pi/2 of direction (az, za) at latitude
// lat: ERFA ae2hd (Az/El -> HA/Dec), then hd2pa.
__device__ __forceinline__ J2 fee_parallactic(const J2& j, double az, double za, double lat) {
    double sa, ca, se, ce, sp, cp;
    sincos(az, &sa, &ca);
    sincos(FRAC_PI_2 - za, &se, &ce);
    sincos(lat, &sp, &cp);
    const double x = -ca * ce * sp + se * cp;
    const double y = -sa * ce;
    const double z = ca * ce * cp + se * sp;
    const double r = sqrt(x * x + y * y);
    const double ha = r != 0.0 ? atan2(y, x) : 0.0;
    const double dec = atan2(z, r);
    double sh, ch, sd, cd;
    sincos(ha, &sh, &ch);
    sincos(dec, &sd, &cd);
    const double sqsz = cp * sh;
    const double cqsz = sp * cd - cp * sd * ch;
    const double pa = (sqsz != 0.0 || cqsz != 0.0) ? atan2(sqsz, cqsz) : 0.0;
    double sr, cr;
    sincos(pa + FRAC_PI_2, &sr, &cr);
    return J2{j.a * cr - j.b * sr, j.a * sr + j.b * cr, j.c * cr - j.d * sr, j.c * sr + j.d * cr};
}

struct FeeArgs {
    const FeeMode* sets;  // [uniq tile][uniq freq][stride], every set laid out for degree nmax
    int stride;
    int nmax;
    const double* norm;   // [uniq freq][4], or NULL
    const FeeRec* rec;    // [FEE_MAX_N + 1][FEE_MAX_N + 1], (n, |m|)
    int n_uniq_freq;
    int n_dirs;
    JonesF64* out;        // [uniq tile][uniq freq][n_dirs]
};

// D directions (d0 + k * FEE_BLOCK) of one (unique tile blockIdx.z, unique
// frequency blockIdx.y) set per thread; a block covers D * FEE_BLOCK
// directions.  RADEC: directions from (RA, Dec) at the LST and latitude
// given (the modeller's components; rotation always applied); otherwise from
// (az, za) arrays, rotated when d_lat is set.  Directions past the end repeat
// the last one and are not written.
template <int D, bool RADEC>
__global__ void __launch_bounds__(FEE_BLOCK, 4) fee_jones_kernel(FeeArgs a, const double* __restrict__ az_in,
                                                             const double* __restrict__ za_in,
                                                             const double2* __restrict__ radec, double lst,
                                                             double lat_v, const double* __restrict__ d_lat) {
    const int d0 = blockIdx.x * (D * FEE_BLOCK) + threadIdx.x;
    const int uf = blockIdx.y, u = blockIdx.z;
    if (d0 >= a.n_dirs) return;
    double az[D], za[D], theta[D], phi[D];
    const bool rot = RADEC || d_lat != nullptr;
    const double lat = RADEC ? lat_v : (d_lat ? *d_lat : 0.0);
#pragma unroll
    for (int k = 0; k < D; k++) {
        const int d = min(d0 + k * FEE_BLOCK, a.n_dirs - 1);
        if (RADEC) {
            const double2 rd = radec[d];
            double el;
            hadec_to_azel(lst - rd.x, rd.y, lat_v, az[k], el);
            za[k] = FRAC_PI_2 - el;
        } else {
            az[k] = az_in[d];
            za[k] = za_in[d];
        }
        theta[k] = za[k];
        phi[k] = FRAC_PI_2 - az[k];
    }
    const size_t set = (size_t)u * a.n_uniq_freq + uf;
    FeeSums sums[D];
    fee_sums<D>(theta, phi, a.sets + set * a.stride, a.nmax, a.rec, sums);
#pragma unroll
    for (int k = 0; k < D; k++) {
        const int d = d0 + k * FEE_BLOCK;
        if (d >= a.n_dirs) break;
        J2 j = fee_jones(sums[k]);
        if (a.norm) {
            const double* nm = a.norm + 4 * uf;
            j.a = cplx{j.a.re / nm[0], j.a.im / nm[0]};
            j.b = cplx{j.b.re / nm[1], j.b.im / nm[1]};
            j.c = cplx{j.c.re / nm[2], j.c.im / nm[2]};
            j.d = cplx{j.d.re / nm[3], j.d.im / nm[3]};
        }
        if (rot) j = fee_parallactic(j, az[k], za[k], lat);
        a.out[set * a.n_dirs + d] = store_j(j);
    }
}

// Directions per thread.  The kernel is bounded to 128 registers so that 4
// blocks (16 warps) fit an SM: with a little spilling that measured faster
// (1.74 ms against 2.06 on the bench workload) than 158 registers at 3.
constexpr int FEE_DIRS_PER_THREAD = 2;

template <bool RADEC>
cudaError_t fee_launch(const FeeArgs& a, int n_uniq_tile, const double* az, const double* za, const double2* radec,
                       double lst, double lat, const double* d_lat, cudaStream_t s) {
    constexpr int D = FEE_DIRS_PER_THREAD;
    dim3 g((a.n_dirs + D * FEE_BLOCK - 1) / (D * FEE_BLOCK), a.n_uniq_freq, n_uniq_tile);
    fee_jones_kernel<D, RADEC><<<g, FEE_BLOCK, 0, s>>>(a, az, za, radec, lst, lat, d_lat);
    return cudaGetLastError();
}

// Zenith normalisation: |element k| of the zenith-pointed beam at the zenith,
// at the azimuth where that element peaks (phi = 0, -pi/2, pi/2, 0).
__global__ void fee_norm_kernel(const FeeMode* __restrict__ ideal, int stride, int nmax,
                                const FeeRec* __restrict__ rec, int n_uniq_freq, double* __restrict__ norm) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 4 * n_uniq_freq) return;
    const int uf = t >> 2, k = t & 3;
    const double theta[1] = {0.0};
    const double phi[1] = {(k == 1) ? -FRAC_PI_2 : (k == 2) ? FRAC_PI_2 : 0.0};
    FeeSums s[1];
    fee_sums<1>(theta, phi, ideal + (size_t)uf * stride, nmax, rec, s);
    const J2 j = fee_jones(s[0]);
    const cplx e = k == 0 ? j.a : k == 1 ? j.b : k == 2 ? j.c : j.d;
    norm[t] = hypot(e.re, e.im);
}

}  // namespace hdc

struct HdcFeeBeam {
    int device = 0;
    int ntiles = 0, nfreqs = 0, n_uniq_tile = 0, n_uniq_freq = 0, stride = 0, nmax = 1;
    hdc::FeeMode* d_sets = nullptr;
    double* d_norm = nullptr;
    hdc::FeeRec* d_rec = nullptr;
    int* d_tile_map = nullptr;
    int* d_freq_map = nullptr;
    std::vector<int> tile_map, freq_map;  // host copies
};

namespace hdc {
namespace {

using zc = std::complex<double>;

void fee_release(HdcFeeBeam* b) {
    cudaFree(b->d_sets);
    cudaFree(b->d_norm);
    cudaFree(b->d_rec);
    cudaFree(b->d_tile_map);
    cudaFree(b->d_freq_map);
    b->d_sets = nullptr;
    b->d_tile_map = b->d_freq_map = nullptr;
    b->d_norm = nullptr;
    b->d_rec = nullptr;
}

// K_mn = C_mn (-m/|m|)^m j^n / sqrt(n (n + 1)).
zc fee_factor(int m, int n) {
    static const zc jpow[4] = {zc(1, 0), zc(0, 1), zc(-1, 0), zc(0, -1)};
    const int a = std::abs(m);
    double ratio = 1.0;  // (n - |m|)! / (n + |m|)!
    for (int t = n - a + 1; t <= n + a; t++) ratio /= (double)t;
    const double c_mn = std::sqrt(0.5 * (2.0 * n + 1.0) * ratio);
    const double sgn = (m > 0 && (m & 1)) ? -1.0 : 1.0;
    return jpow[n & 3] * (c_mn * sgn / std::sqrt((double)n * (n + 1.0)));
}

// The beamformed coefficients of one set (file frequency k, one tile's
// amplitudes [32] and delays [16], dead dipoles already zeroed) as the
// fee_num_modes(nmax) records of the kernel's order in out.
void fee_set(const HdcFeeCoeffs* f, int k, const double* amps, const uint32_t* delays, int nmax, FeeMode* out) {
    const int nm = f->num_freq_modes[k];
    const size_t dense = (size_t)(nmax + 1) * (nmax + 1);  // (n, m) at n^2 + n + m
    std::vector<zc> q1[2], q2[2];
    for (int p = 0; p < 2; p++) {
        q1[p].assign(dense, zc(0, 0));
        q2[p].assign(dense, zc(0, 0));
        zc w[16];
        for (int d = 0; d < 16; d++) {
            const double ph = -TAU * (double)f->freqs_hz[k] * (double)delays[d] * FEE_DELAY_STEP;
            w[d] = std::polar(amps[16 * p + d], ph);
        }
        const double* qk = f->q + (((size_t)k * 2 + p) * 16) * (size_t)f->num_modes * 2;
        for (int col = 0; col < nm; col++) {
            const int s = f->modes[col], m = f->modes[f->num_modes + col], n = f->modes[2 * f->num_modes + col];
            zc acc(0, 0);
            for (int d = 0; d < 16; d++) {
                const double* c = qk + ((size_t)d * f->num_modes + col) * 2;
                acc += w[d] * zc(c[0], c[1]);
            }
            const size_t i = (size_t)n * n + n + m;
            (s == 1 ? q1[p] : q2[p])[i] += acc * fee_factor(m, n);
        }
    }
    auto d2 = [](zc z) { return make_double2(z.real(), z.imag()); };
    FeeMode* o = out;
    for (int ma = 1; ma <= nmax; ma++)
        for (int n = ma; n <= nmax; n++) {
            if (ma == 1) {
                const size_t i0 = (size_t)n * n + n;
                *o++ = FeeMode{d2(q1[0][i0]), d2(q2[0][i0]), d2(q1[1][i0]), d2(q2[1][i0])};
            }
            const size_t ip = (size_t)n * n + n + ma, im = (size_t)n * n + n - ma;
            for (int p = 0; p < 2; p++)
                *o++ = FeeMode{d2(q1[p][ip] + q1[p][im]), d2(q1[p][ip] - q1[p][im]), d2(q2[p][ip] + q2[p][im]),
                               d2(q2[p][ip] - q2[p][im])};
        }
}

int fee_check_file(const HdcFeeCoeffs* f) {
    if (!f || f->num_freqs < 1 || !f->freqs_hz || f->num_modes < 1 || !f->modes || !f->num_freq_modes || !f->q) {
        set_error("hdc_fee_beam_new: incomplete coefficient arrays");
        return HDC_ERR_ARG;
    }
    for (int k = 0; k < f->num_freqs; k++)
        if (f->num_freq_modes[k] < 1 || f->num_freq_modes[k] > f->num_modes) {
            set_error("hdc_fee_beam_new: frequency %d has %d modes of %d", k, f->num_freq_modes[k], f->num_modes);
            return HDC_ERR_ARG;
        }
    for (int c = 0; c < f->num_modes; c++) {
        const int s = f->modes[c], m = f->modes[f->num_modes + c], n = f->modes[2 * f->num_modes + c];
        if ((s != 1 && s != 2) || n < 1 || n > FEE_MAX_N || std::abs(m) > n) {
            set_error("hdc_fee_beam_new: mode column %d (s %d, m %d, n %d) is outside s in {1, 2}, 1 <= n <= %d, "
                      "|m| <= n", c, s, m, n, FEE_MAX_N);
            return HDC_ERR_ARG;
        }
    }
    return HDC_OK;
}

}  // namespace

// Directions from (RA, Dec) at an LST (the modeller's per-timestep beam).
int fee_launch_radec(const HdcFeeBeam* b, const double2* d_radec, int n, double lst, double lat, JonesF64* d_out,
                     cudaStream_t s) {
    if (n <= 0) return HDC_OK;
    FeeArgs a{b->d_sets, b->stride, b->nmax, b->d_norm, b->d_rec, b->n_uniq_freq, n, d_out};
    HDC_CUDA_RET_INT(fee_launch<true>(a, b->n_uniq_tile, nullptr, nullptr, d_radec, lst, lat, nullptr, s));
    count_launches(1);
    return HDC_OK;
}

int fee_num_tiles(const HdcFeeBeam* b) { return b->ntiles; }
int fee_num_freqs(const HdcFeeBeam* b) { return b->nfreqs; }
int fee_device(const HdcFeeBeam* b) { return b->device; }

}  // namespace hdc

using namespace hdc;

extern "C" int hdc_fee_beam_new(const HdcFeeCoeffs* file, const uint32_t* h_freqs_hz, int num_freqs,
                                const uint32_t* h_delays, const double* h_amps, int num_tiles, int num_amps,
                                int norm_to_zenith, HdcFeeBeam** out) {
    if (!out) {
        set_error("hdc_fee_beam_new: NULL output");
        return HDC_ERR_ARG;
    }
    *out = nullptr;
    int rc = fee_check_file(file);
    if (rc) return rc;
    if (!h_freqs_hz || num_freqs < 1 || !h_delays || !h_amps || num_tiles < 1 || (num_amps != 16 && num_amps != 32)) {
        set_error("hdc_fee_beam_new: invalid arguments (num_freqs %d, num_tiles %d, num_amps %d)", num_freqs,
                  num_tiles, num_amps);
        return HDC_ERR_ARG;
    }
    // channels -> the file's closest frequency (the first on a tie), unique in order of first appearance
    std::vector<int> fmap(num_freqs), ufile;
    for (int f = 0; f < num_freqs; f++) {
        int best = 0;
        long long bd = -1;
        for (int k = 0; k < file->num_freqs; k++) {
            const long long dd = std::llabs((long long)file->freqs_hz[k] - (long long)h_freqs_hz[f]);
            if (bd < 0 || dd < bd) {
                bd = dd;
                best = k;
            }
        }
        auto it = std::find(ufile.begin(), ufile.end(), best);
        fmap[f] = (int)(it - ufile.begin());
        if (it == ufile.end()) ufile.push_back(best);
    }
    // tiles -> unique (delays, amplitudes), dead dipoles (delay 32) at amplitude 0 and delay 0
    std::vector<int> tmap(num_tiles);
    std::vector<std::vector<double>> uamp;
    std::vector<std::vector<uint32_t>> udel;
    for (int t = 0; t < num_tiles; t++) {
        std::vector<double> a(32);
        std::vector<uint32_t> dl(16);
        for (int d = 0; d < 16; d++) {
            const uint32_t v = h_delays[16 * (size_t)t + d];
            if (v > FEE_DEAD_DELAY) {
                set_error("hdc_fee_beam_new: tile %d dipole %d has delay %u (at most 32)", t, d, v);
                return HDC_ERR_ARG;
            }
            const bool dead = v == FEE_DEAD_DELAY;
            dl[d] = dead ? 0u : v;
            const double ax = h_amps[(size_t)num_amps * t + d];
            const double ay = h_amps[(size_t)num_amps * t + (num_amps == 32 ? 16 + d : d)];
            a[d] = dead ? 0.0 : ax;
            a[16 + d] = dead ? 0.0 : ay;
        }
        int found = -1;
        for (size_t u = 0; u < uamp.size() && found < 0; u++)
            if (uamp[u] == a && udel[u] == dl) found = (int)u;
        if (found < 0) {
            found = (int)uamp.size();
            uamp.push_back(a);
            udel.push_back(dl);
        }
        tmap[t] = found;
    }
    const int nu = (int)uamp.size(), nuf = (int)ufile.size();
    // every set is laid out for the largest degree of all the unique
    // frequencies (zero coefficients above a frequency's own): one stride and
    // one loop for all sets
    int nmax = 1;
    for (int i = 0; i < nuf; i++) {
        const int k = ufile[i];
        for (int c = 0; c < file->num_freq_modes[k]; c++) nmax = std::max(nmax, (int)file->modes[2 * file->num_modes + c]);
    }
    const int stride = fee_num_modes(nmax);
    std::vector<FeeMode> sets((size_t)nu * nuf * stride);
    for (int u = 0; u < nu; u++)
        for (int i = 0; i < nuf; i++)
            fee_set(file, ufile[i], uamp[u].data(), udel[u].data(), nmax, sets.data() + ((size_t)u * nuf + i) * stride);
    // the column recurrence's constants per (n, |m|), |m| <= n
    std::vector<FeeRec> rec((size_t)(FEE_MAX_N + 1) * (FEE_MAX_N + 1), FeeRec{0.0, 0.0, 0.0, 0.0});
    for (int n = 1; n <= FEE_MAX_N; n++)
        for (int ma = 1; ma <= n; ma++)
            rec[(size_t)n * (FEE_MAX_N + 1) + ma] =
                FeeRec{n + 1.0, n - ma + 1.0, (2.0 * n + 3.0) / (n + 2.0 - ma), (n + 1.0 + ma) / (n + 2.0 - ma)};

    HdcFeeBeam* b = new HdcFeeBeam();
    cudaGetDevice(&b->device);
    b->ntiles = num_tiles;
    b->nfreqs = num_freqs;
    b->n_uniq_tile = nu;
    b->n_uniq_freq = nuf;
    b->stride = stride;
    b->nmax = nmax;
    b->tile_map = tmap;
    b->freq_map = fmap;
    auto fail = [&](cudaError_t e, const char* what) {
        set_error("hdc_fee_beam_new: %s: %s", what, cudaGetErrorString(e));
        fee_release(b);
        delete b;
        return e == cudaErrorMemoryAllocation ? HDC_ERR_ALLOC : HDC_ERR_CUDA;
    };
    cudaError_t e;
    if ((e = cudaMalloc(&b->d_sets, sizeof(FeeMode) * sets.size())) != cudaSuccess) return fail(e, "cudaMalloc");
    if ((e = cudaMalloc(&b->d_rec, sizeof(FeeRec) * rec.size())) != cudaSuccess) return fail(e, "cudaMalloc");
    if ((e = cudaMalloc(&b->d_tile_map, sizeof(int) * num_tiles)) != cudaSuccess) return fail(e, "cudaMalloc");
    if ((e = cudaMalloc(&b->d_freq_map, sizeof(int) * num_freqs)) != cudaSuccess) return fail(e, "cudaMalloc");
    if ((e = cudaMemcpy(b->d_sets, sets.data(), sizeof(FeeMode) * sets.size(), cudaMemcpyHostToDevice)) != cudaSuccess)
        return fail(e, "cudaMemcpy");
    if ((e = cudaMemcpy(b->d_rec, rec.data(), sizeof(FeeRec) * rec.size(), cudaMemcpyHostToDevice)) != cudaSuccess)
        return fail(e, "cudaMemcpy");
    if ((e = cudaMemcpy(b->d_tile_map, tmap.data(), sizeof(int) * num_tiles, cudaMemcpyHostToDevice)) != cudaSuccess)
        return fail(e, "cudaMemcpy");
    if ((e = cudaMemcpy(b->d_freq_map, fmap.data(), sizeof(int) * num_freqs, cudaMemcpyHostToDevice)) != cudaSuccess)
        return fail(e, "cudaMemcpy");
    if (norm_to_zenith) {
        // the zenith-pointed beam of every unique frequency: all delays 0, amplitudes 1
        std::vector<FeeMode> ideal((size_t)nuf * stride);
        const std::vector<double> ones(32, 1.0);
        const std::vector<uint32_t> zeros(16, 0u);
        for (int i = 0; i < nuf; i++)
            fee_set(file, ufile[i], ones.data(), zeros.data(), nmax, ideal.data() + (size_t)i * stride);
        FeeMode* d_ideal = nullptr;
        if ((e = cudaMalloc(&d_ideal, sizeof(FeeMode) * ideal.size())) != cudaSuccess) return fail(e, "cudaMalloc");
        if ((e = cudaMalloc(&b->d_norm, sizeof(double) * 4 * nuf)) != cudaSuccess) {
            cudaFree(d_ideal);
            return fail(e, "cudaMalloc");
        }
        e = cudaMemcpy(d_ideal, ideal.data(), sizeof(FeeMode) * ideal.size(), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) {
            fee_norm_kernel<<<(4 * nuf + 127) / 128, 128>>>(d_ideal, stride, nmax, b->d_rec, nuf, b->d_norm);
            count_launches(1);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaDeviceSynchronize();
        cudaFree(d_ideal);
        if (e != cudaSuccess) return fail(e, "zenith normalisation");
        // every element divides by its norm: a zero or non-finite one (a
        // coefficient set without that element at the zenith) is refused
        std::vector<double> h_norm((size_t)4 * nuf);
        if ((e = cudaMemcpy(h_norm.data(), b->d_norm, sizeof(double) * h_norm.size(), cudaMemcpyDeviceToHost)) !=
            cudaSuccess)
            return fail(e, "cudaMemcpy");
        for (size_t i = 0; i < h_norm.size(); i++)
            if (!(h_norm[i] > 0.0) || !std::isfinite(h_norm[i])) {
                set_error("hdc_fee_beam_new: the zenith-pointed beam's element %d at %u Hz is %g at the zenith; it "
                          "cannot normalise", (int)(i % 4), file->freqs_hz[ufile[i / 4]], h_norm[i]);
                fee_release(b);
                delete b;
                return HDC_ERR_ARG;
            }
    }
    *out = b;
    return HDC_OK;
}

extern "C" void hdc_fee_beam_free(HdcFeeBeam* b) {
    if (!b) return;
    int cur = 0;
    cudaGetDevice(&cur);
    if (cur != b->device) cudaSetDevice(b->device);
    fee_release(b);
    if (cur != b->device) cudaSetDevice(cur);
    delete b;
}

extern "C" int hdc_fee_beam_num_unique_tiles(const HdcFeeBeam* b) { return b ? b->n_uniq_tile : 0; }
extern "C" int hdc_fee_beam_num_unique_freqs(const HdcFeeBeam* b) { return b ? b->n_uniq_freq : 0; }
extern "C" const int* hdc_fee_beam_tile_map(const HdcFeeBeam* b) { return b ? b->d_tile_map : nullptr; }
extern "C" const int* hdc_fee_beam_freq_map(const HdcFeeBeam* b) { return b ? b->d_freq_map : nullptr; }

extern "C" int hdc_fee_beam_host_maps(const HdcFeeBeam* b, int* h_tile_map, int* h_freq_map) {
    if (!b) return HDC_ERR_ARG;
    if (h_tile_map) std::copy(b->tile_map.begin(), b->tile_map.end(), h_tile_map);
    if (h_freq_map) std::copy(b->freq_map.begin(), b->freq_map.end(), h_freq_map);
    return HDC_OK;
}

extern "C" int hdc_fee_calc_jones(const HdcFeeBeam* b, const double* d_az_rad, const double* d_za_rad,
                                  int num_directions, const double* d_latitude_rad, int iau_order, JonesF64* d_jones,
                                  hdcStream_t stream) {
    if (!b || num_directions < 0 || (num_directions > 0 && (!d_az_rad || !d_za_rad || !d_jones))) {
        set_error("hdc_fee_calc_jones: invalid arguments");
        return HDC_ERR_ARG;
    }
    if (iau_order) {
        set_error("hdc_fee_calc_jones: iau_order = 1 is not supported (the reference asks for 0)");
        return HDC_ERR_UNSUPPORTED;
    }
    int dev = 0;
    HDC_CUDA_RET_INT(cudaGetDevice(&dev));
    if (dev != b->device) {
        set_error("hdc_fee_calc_jones: the beam was prepared on device %d, the current device is %d", b->device, dev);
        return HDC_ERR_ARG;
    }
    if (num_directions == 0) return HDC_OK;
    FeeArgs a{b->d_sets, b->stride, b->nmax, b->d_norm, b->d_rec, b->n_uniq_freq, num_directions, d_jones};
    HDC_CUDA_RET_INT(fee_launch<false>(a, b->n_uniq_tile, d_az_rad, d_za_rad, nullptr, 0.0, 0.0, d_latitude_rad,
                                       (cudaStream_t)stream));
    count_launches(1);
    return HDC_OK;
}
