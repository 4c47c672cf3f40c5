// ORACLE — test infrastructure only. Nothing in the product links or calls
// this file; only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
// arm load it, as the checker.
//
// A CPU, FP64 restatement of mwa_hyperdrive's algorithms on the sky-model
// predict / DI-calibration / peel path.  Every function cites the reference
// file:line it follows (paths relative to the mwa_hyperdrive project root).
// The reference is Rust and cannot be built in this environment (no cargo, no
// vendored crates), so there is no compiled-reference twin; parity is pinned
// against the reference's own known-answer tests (tests/golden/*).
//
// Arithmetic conventions mirror the reference's Rust code: complex multiply
// and divide are the naive num_complex formulas, no FMA contraction
// (compiled with -ffp-contract=off), f64 accumulation with an f32 demotion at
// the same points as the reference.
//
// Third-party maths restated here (crates not present in the reference tree,
// pinned in its Cargo.lock): marlu 0.17.1 (Jones algebra, RADec->LMN,
// HADec->AzEl, XYZ->UVW), num-complex 0.4 (complex division).

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr double VEL_C = 299792458.0;
constexpr double TAU = 6.283185307179586;
constexpr double FRAC_PI_2 = 1.5707963267948966;
constexpr double LN_2 = 0.6931471805599453;
constexpr double SQRT_FRAC_PI_SQ_2_LN_2 = 2.6682231283184983;
constexpr double SBF_C = 5000.0;
constexpr int SBF_L = 10001;
constexpr int SBF_N = 101;
constexpr double SBF_DX = 0.01;
// model/cpu.rs:36-37
const double GAUSSIAN_EXP_CONST = -(FRAC_PI_2 * FRAC_PI_2) / LN_2;
const double SHAPELET_CONST = SQRT_FRAC_PI_SQ_2_LN_2 / SBF_DX;
constexpr double DEFAULT_SPEC_INDEX = -0.8;  // constants.rs

struct c64 {
    double re, im;
};
inline c64 cadd(c64 a, c64 b) { return {a.re + b.re, a.im + b.im}; }
inline c64 csub(c64 a, c64 b) { return {a.re - b.re, a.im - b.im}; }
inline c64 cmul(c64 a, c64 b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
inline c64 cscale(c64 a, double s) { return {a.re * s, a.im * s}; }
inline c64 cconj(c64 a) { return {a.re, -a.im}; }
inline double cnorm_sqr(c64 a) { return a.re * a.re + a.im * a.im; }
// num_complex Div (naive): (a * conj(b)) / |b|^2
inline c64 cdiv(c64 a, c64 b) {
    double n = cnorm_sqr(b);
    double re = a.re * b.re + a.im * b.im;
    double im = a.im * b.re - a.re * b.im;
    return {re / n, im / n};
}
inline c64 cis(double x) { return {std::cos(x), std::sin(x)}; }

struct J64 {
    c64 j[4];
};
inline J64 jzero() { return J64{{{0, 0}, {0, 0}, {0, 0}, {0, 0}}}; }
inline J64 jidentity() { return J64{{{1, 0}, {0, 0}, {0, 0}, {1, 0}}}; }
inline J64 jadd(const J64& a, const J64& b) {
    J64 r;
    for (int k = 0; k < 4; k++) r.j[k] = cadd(a.j[k], b.j[k]);
    return r;
}
inline J64 jsub(const J64& a, const J64& b) {
    J64 r;
    for (int k = 0; k < 4; k++) r.j[k] = csub(a.j[k], b.j[k]);
    return r;
}
// marlu Jones Mul<Jones>
inline J64 jmul(const J64& a, const J64& b) {
    J64 r;
    r.j[0] = cadd(cmul(a.j[0], b.j[0]), cmul(a.j[1], b.j[2]));
    r.j[1] = cadd(cmul(a.j[0], b.j[1]), cmul(a.j[1], b.j[3]));
    r.j[2] = cadd(cmul(a.j[2], b.j[0]), cmul(a.j[3], b.j[2]));
    r.j[3] = cadd(cmul(a.j[2], b.j[1]), cmul(a.j[3], b.j[3]));
    return r;
}
inline J64 jmulc(const J64& a, c64 c) {
    J64 r;
    for (int k = 0; k < 4; k++) r.j[k] = cmul(a.j[k], c);
    return r;
}
inline J64 jscale(const J64& a, double s) {
    J64 r;
    for (int k = 0; k < 4; k++) r.j[k] = cscale(a.j[k], s);
    return r;
}
// conjugate transpose (marlu Jones::h)
inline J64 jh(const J64& a) {
    J64 r;
    r.j[0] = cconj(a.j[0]);
    r.j[1] = cconj(a.j[2]);
    r.j[2] = cconj(a.j[1]);
    r.j[3] = cconj(a.j[3]);
    return r;
}
// marlu Jones::inv: inv_det = 1/(ad - bc); [d, -b, -c, a] * inv_det
inline J64 jinv(const J64& a) {
    c64 det = csub(cmul(a.j[0], a.j[3]), cmul(a.j[1], a.j[2]));
    c64 inv_det = cdiv(c64{1.0, 0.0}, det);
    J64 r;
    r.j[0] = cmul(inv_det, a.j[3]);
    r.j[1] = cmul(cscale(inv_det, -1.0), a.j[1]);
    r.j[2] = cmul(cscale(inv_det, -1.0), a.j[2]);
    r.j[3] = cmul(inv_det, a.j[0]);
    return r;
}
inline bool jany_nan(const J64& a) {
    for (int k = 0; k < 4; k++)
        if (std::isnan(a.j[k].re) || std::isnan(a.j[k].im)) return true;
    return false;
}
inline J64 jnan() {
    J64 r;
    for (int k = 0; k < 4; k++) r.j[k] = {NAN, NAN};
    return r;
}
inline J64 from_f32(const float* p) {
    J64 r;
    for (int k = 0; k < 4; k++) r.j[k] = {(double)p[2 * k], (double)p[2 * k + 1]};
    return r;
}
inline J64 from_f64(const double* p) {
    J64 r;
    for (int k = 0; k < 4; k++) r.j[k] = {p[2 * k], p[2 * k + 1]};
    return r;
}
inline void to_f64(const J64& a, double* p) {
    for (int k = 0; k < 4; k++) {
        p[2 * k] = a.j[k].re;
        p[2 * k + 1] = a.j[k].im;
    }
}
inline void to_f32(const J64& a, float* p) {
    for (int k = 0; k < 4; k++) {
        p[2 * k] = (float)a.j[k].re;
        p[2 * k + 1] = (float)a.j[k].im;
    }
}
// gpu/common.cuh `JonesF32 * C64`: the complex factor is demoted to f32 and
// the product is formed in f32.
inline void jf32_mul_c64(const float* a, c64 b, float* out) {
    float bx = (float)b.re, by = (float)b.im;
    for (int k = 0; k < 4; k++) {
        float re = a[2 * k], im = a[2 * k + 1];
        out[2 * k] = re * bx - im * by;
        out[2 * k + 1] = re * by + im * bx;
    }
}
// Rust f64::signum
inline double rsignum(double x) {
    if (std::isnan(x)) return NAN;
    return std::signbit(x) ? -1.0 : 1.0;
}
// Rust `f as usize` (saturating; NaN -> 0)
inline long long rs_as_usize(double x) {
    if (!(x > 0.0)) return 0;
    if (x >= 9.0e18) return (long long)9.0e18;
    return (long long)x;
}

}  // namespace

extern "C" {

// ---------------------------------------------------------------------------
// Sky-model description (struct of arrays). The same layout as the product's
// HdcSkyModel, defined independently here.
// comp_type: 0 point, 1 Gaussian, 2 shapelet.
// flux_type: 0 list, 1 power law, 2 curved power law.
// fds: 5 doubles per entry (freq [Hz], I, Q, U, V); for (curved) power laws
// fd_count == 1 and the entry is the reference flux density.
// ---------------------------------------------------------------------------
typedef struct OrSky {
    int num_components;
    const int* comp_type;
    const double* ra;
    const double* dec;
    const double* maj;
    const double* min;
    const double* pa;
    const int* flux_type;
    const double* si;
    const double* q;
    const int* fd_start;
    const int* fd_count;
    const double* fds;
    const int* coeff_start;
    const int* coeff_count;
    const int* coeff_n1;
    const int* coeff_n2;
    const double* coeff_value;
} OrSky;

typedef struct OrFD {
    double freq, i, q, u, v;
} OrFD;

}  // extern "C"

namespace {

OrFD fd_at(const OrSky* s, int idx) {
    const double* p = s->fds + 5 * idx;
    return OrFD{p[0], p[1], p[2], p[3], p[4]};
}
OrFD fd_scale(OrFD a, double r) { return OrFD{a.freq, a.i * r, a.q * r, a.u * r, a.v * r}; }

// srclist/types/flux_density/mod.rs:273-275
double calc_flux_ratio(double desired_freq_hz, double cat_freq_hz, double spec_index) {
    return std::pow(desired_freq_hz / cat_freq_hz, spec_index);
}

// srclist/types/flux_density/mod.rs:158-270 (FluxDensityType::estimate_at_freq)
OrFD estimate_at_freq(const OrSky* s, int c, double freq_hz) {
    int ft = s->flux_type[c];
    int start = s->fd_start[c];
    int count = s->fd_count[c];
    if (ft == 1) {
        OrFD fd = fd_at(s, start);
        double ratio = calc_flux_ratio(freq_hz, fd.freq, s->si[c]);
        OrFD n = fd_scale(fd, ratio);
        n.freq = freq_hz;
        return n;
    }
    if (ft == 2) {
        OrFD fd = fd_at(s, start);
        OrFD pl = fd_scale(fd, calc_flux_ratio(freq_hz, fd.freq, s->si[c]));
        pl.freq = freq_hz;
        double lr = std::log(freq_hz / fd.freq);
        double curved = std::exp(s->q[c] * (lr * lr));
        return fd_scale(pl, curved);
    }
    // list
    double spec_index;
    OrFD smaller;
    if (count == 1) {
        spec_index = DEFAULT_SPEC_INDEX;
        smaller = fd_at(s, start);
    } else {
        OrFD p0 = fd_at(s, start), p1 = fd_at(s, start + 1);
        for (int w = 0; w + 1 < count; w++) {
            OrFD w0 = fd_at(s, start + w), w1 = fd_at(s, start + w + 1);
            p0 = w0;
            p1 = w1;
            if (std::fabs(w0.freq - freq_hz) < 1e-3) return w0;
            if (std::fabs(w1.freq - freq_hz) < 1e-3) return w1;
            if (freq_hz < w1.freq) break;
        }
        OrFD fd1 = p0, fd2 = p1;
        if (rsignum(fd1.i) != rsignum(fd2.i)) {
            double run = fd2.freq - fd1.freq;
            double is = (fd2.i - fd1.i) / run, qs = (fd2.q - fd1.q) / run;
            double us = (fd2.u - fd1.u) / run, vs = (fd2.v - fd1.v) / run;
            double df = freq_hz - fd1.freq;
            return OrFD{freq_hz, fd1.i + is * df, fd1.q + qs * df, fd1.u + us * df, fd1.v + vs * df};
        }
        // FluxDensity::calc_spec_index (flux_density/mod.rs:47-49)
        spec_index = std::log(fd2.i / fd1.i) / std::log(fd2.freq / fd1.freq);
        smaller = (fd2.freq < freq_hz) ? fd2 : fd1;
    }
    double ratio = calc_flux_ratio(freq_hz, smaller.freq, spec_index);
    OrFD out = smaller;
    out.freq = freq_hz;
    return fd_scale(out, ratio);
}

// flux_density/mod.rs:58-65 (to_inst_stokes; X = EW)
J64 to_inst_stokes(OrFD f) {
    J64 r;
    r.j[0] = {f.i - f.q, 0.0};
    r.j[1] = {f.u, -f.v};
    r.j[2] = {f.u, f.v};
    r.j[3] = {f.i + f.q, 0.0};
    return r;
}

// marlu RADec::to_lmn + LMN::prepare_for_rime (used at components/mod.rs:214)
void lmn_rime(double ra, double dec, double pc_ra, double pc_dec, double out[3]) {
    double d_ra = ra - pc_ra;
    double s_d_ra = std::sin(d_ra), c_d_ra = std::cos(d_ra);
    double s_dec = std::sin(dec), c_dec = std::cos(dec);
    double pc_s = std::sin(pc_dec), pc_c = std::cos(pc_dec);
    double l = c_dec * s_d_ra;
    double m = s_dec * pc_c - c_dec * pc_s * c_d_ra;
    double n = s_dec * pc_s + c_dec * pc_c * c_d_ra;
    out[0] = TAU * l;
    out[1] = TAU * m;
    out[2] = TAU * (n - 1.0);
}

// marlu UVW::from_xyz_inner (same formula as params/peel/mod.rs:1482-1530)
void uvw_from_xyz(const double* xyz, double s_ha, double c_ha, double s_dec, double c_dec, double out[3]) {
    double x = xyz[0], y = xyz[1], z = xyz[2];
    out[0] = s_ha * x + c_ha * y;
    out[1] = -s_dec * c_ha * x + s_dec * s_ha * y + c_dec * z;
    out[2] = c_dec * c_ha * x - c_dec * s_ha * y + s_dec * z;
}

// marlu xyzs_to_cross_uvws: tile UVWs, then tile1 - tile2 for p < q
void xyzs_to_cross_uvws(const double* xyzs, int ntiles, double ha, double dec, double* uvws) {
    double s_ha = std::sin(ha), c_ha = std::cos(ha), s_dec = std::sin(dec), c_dec = std::cos(dec);
    std::vector<double> t(3 * (size_t)ntiles);
    for (int i = 0; i < ntiles; i++) uvw_from_xyz(xyzs + 3 * i, s_ha, c_ha, s_dec, c_dec, &t[3 * i]);
    size_t b = 0;
    for (int i = 0; i < ntiles; i++)
        for (int j = i + 1; j < ntiles; j++, b++)
            for (int k = 0; k < 3; k++) uvws[3 * b + k] = t[3 * i + k] - t[3 * j + k];
}

// marlu HADec::to_azel (ERFA hd2ae)
void hadec_to_azel(double ha, double dec, double lat, double* az, double* el) {
    double s_ha = std::sin(ha), c_ha = std::cos(ha);
    double s_dec = std::sin(dec), c_dec = std::cos(dec);
    double s_lat = std::sin(lat), c_lat = std::cos(lat);
    double x = -s_ha * c_dec;
    double y = -c_ha * c_dec * s_lat + s_dec * c_lat;
    double z = c_ha * c_dec * c_lat + s_dec * s_lat;
    double r = std::hypot(x, y);
    double a = (r == 0.0) ? 0.0 : std::atan2(x, y);
    *az = (a < 0.0) ? a + TAU : a;
    *el = std::atan2(z, r);
}

// Analytic 4x4 dipole-array tile beam with a ground plane (a model of this
// project; the reference has no analytic beam). J = A(az,za,f) R(az)^T
// diag(cos za, 1) R(az), A = AFx(l) AFy(m) GP(za)/|GP(0)|.
J64 analytic_beam(double az, double el, double freq) {
    double za = FRAC_PI_2 - el;
    if (el <= 0.0) return jzero();
    double k = TAU * freq / VEL_C;
    double sza = std::sin(za), cza = std::cos(za);
    double saz = std::sin(az), caz = std::cos(az);
    double l = sza * saz, m = sza * caz;
    double afx = 0.5 * (std::cos(k * 0.55 * l) + std::cos(k * 1.65 * l));
    double afy = 0.5 * (std::cos(k * 0.55 * m) + std::cos(k * 1.65 * m));
    const double h = 0.278;
    // GP = 1 - exp(-2 i k h cos za); |GP(0)| = 2 |sin(k h)|
    double ph = 2.0 * k * h * cza;
    c64 gp = {1.0 - std::cos(ph), std::sin(ph)};
    double gp0 = 2.0 * std::fabs(std::sin(k * h));
    double a = afx * afy / gp0;
    c64 amp = cscale(gp, a);
    double p00 = cza * saz * saz + caz * caz;
    double p01 = (cza - 1.0) * saz * caz;
    double p11 = cza * caz * caz + saz * saz;
    J64 r;
    r.j[0] = cscale(amp, p00);
    r.j[1] = cscale(amp, p01);
    r.j[2] = cscale(amp, p01);
    r.j[3] = cscale(amp, p11);
    return r;
}

// The same tile with each dipole's own amplitude g [2][16] (X dipoles then
// Y; dipole d at east (d % 4 - 1.5) 1.1 m, north (d / 4 - 1.5) 1.1 m; this
// project's model, used for per-tile beams): J = diag(ax, ay) R(az)^T
// diag(cos za, 1) R(az), ax = AF(g_x) GP / |GP(0)|, AF(g) = (1/16) sum_d g_d
// exp(i k (x_d l + y_d m)).  With unit gains it is analytic_beam.
J64 analytic_beam_tile(double az, double el, double freq, const double* g) {
    if (el <= 0.0) return jzero();
    double za = FRAC_PI_2 - el;
    double k = TAU * freq / VEL_C;
    double sza = std::sin(za), cza = std::cos(za);
    double saz = std::sin(az), caz = std::cos(az);
    double l = sza * saz, m = sza * caz;
    c64 afx = {0.0, 0.0}, afy = {0.0, 0.0};
    for (int d = 0; d < 16; d++) {
        double x = (d % 4 - 1.5) * 1.1, y = (d / 4 - 1.5) * 1.1;
        c64 e = cis(k * (x * l + y * m));
        afx = cadd(afx, cscale(e, g[d]));
        afy = cadd(afy, cscale(e, g[16 + d]));
    }
    const double h = 0.278;
    double ph = 2.0 * k * h * cza;
    c64 gp = {1.0 - std::cos(ph), std::sin(ph)};
    double gp0 = 2.0 * std::fabs(std::sin(k * h));
    c64 ax = cscale(cmul(afx, gp), 1.0 / (16.0 * gp0)), ay = cscale(cmul(afy, gp), 1.0 / (16.0 * gp0));
    double p00 = cza * saz * saz + caz * caz;
    double p01 = (cza - 1.0) * saz * caz;
    double p11 = cza * caz * caz + saz * saz;
    J64 r;
    r.j[0] = cscale(ax, p00);
    r.j[1] = cscale(ax, p01);
    r.j[2] = cscale(ay, p01);
    r.j[3] = cscale(ay, p11);
    return r;
}

std::vector<double> g_sbf;  // shapelet basis table, built on first use

// The reference regenerates its table with make_shapelet_basis_values.py:
// B_n(x) = exp(-x^2/2) H_n(x) / sqrt(2^n n!) on linspace(-50, 50, 10001),
// H_n the physicists' Hermite polynomial (three-term recurrence).
void build_sbf() {
    if (!g_sbf.empty()) return;
    g_sbf.assign((size_t)SBF_N * SBF_L, 0.0);
    for (int ix = 0; ix < SBF_L; ix++) {
        // numpy linspace: start + i*step, last point exact
        double step = 100.0 / (SBF_L - 1);
        double x = (ix == SBF_L - 1) ? 50.0 : -50.0 + ix * step;
        double g = std::exp(-0.5 * (x * x));
        double hm1 = 1.0, h = 2.0 * x;
        for (int n = 0; n < SBF_N; n++) {
            double hn;
            if (n == 0)
                hn = 1.0;
            else if (n == 1)
                hn = 2.0 * x;
            else {
                double hp = 2.0 * x * h - 2.0 * (n - 1) * hm1;
                hm1 = h;
                h = hp;
                hn = hp;
            }
            double norm = 1.0 / std::sqrt(std::pow(2.0, n) * std::tgamma(n + 1.0));
            g_sbf[(size_t)n * SBF_L + ix] = g * norm * hn;
        }
    }
}

struct CompTables {
    // per type: component indices into the sky model, in sky-model order
    std::vector<int> idx[3];
    std::vector<double> lmn[3];       // [c][3] (2*pi scaled, n-1)
    std::vector<J64> fds[3];          // [f][c]
};

void build_tables(const OrSky* s, const double* freqs, int nf, double pc_ra, double pc_dec, CompTables& t) {
    for (int c = 0; c < s->num_components; c++) t.idx[s->comp_type[c]].push_back(c);
    for (int ty = 0; ty < 3; ty++) {
        int nc = (int)t.idx[ty].size();
        t.lmn[ty].resize(3 * (size_t)nc);
        t.fds[ty].resize((size_t)nf * nc);
        for (int k = 0; k < nc; k++) {
            int c = t.idx[ty][k];
            lmn_rime(s->ra[c], s->dec[c], pc_ra, pc_dec, &t.lmn[ty][3 * k]);
            for (int f = 0; f < nf; f++) t.fds[ty][(size_t)f * nc + k] = to_inst_stokes(estimate_at_freq(s, c, freqs[f]));
        }
    }
}

inline void bl_to_tiles(int ntiles, std::vector<int>& t1, std::vector<int>& t2) {
    t1.clear();
    t2.clear();
    for (int i = 0; i < ntiles; i++)
        for (int j = i + 1; j < ntiles; j++) {
            t1.push_back(i);
            t2.push_back(j);
        }
}

}  // namespace

extern "C" {

int or_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void or_set_num_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

// model/shapelets.rs (table values); writes SBF_N*SBF_L doubles.
void or_shapelet_basis(double* out) {
    build_sbf();
    std::memcpy(out, g_sbf.data(), g_sbf.size() * sizeof(double));
}

// components/mod.rs:323-346 get_instrumental_flux_densities for all
// components of the sky model in order; out: [nf][nc] JonesF64.
void or_inst_flux(const OrSky* s, const double* freqs, int nf, double* out) {
    int nc = s->num_components;
    for (int f = 0; f < nf; f++)
        for (int c = 0; c < nc; c++) to_f64(to_inst_stokes(estimate_at_freq(s, c, freqs[f])), out + 8 * ((size_t)f * nc + c));
}

void or_estimate_at_freq(const OrSky* s, int c, double freq, double* out5) {
    OrFD f = estimate_at_freq(s, c, freq);
    out5[0] = f.freq;
    out5[1] = f.i;
    out5[2] = f.q;
    out5[3] = f.u;
    out5[4] = f.v;
}

void or_lmn_rime(double ra, double dec, double pc_ra, double pc_dec, double* out3) { lmn_rime(ra, dec, pc_ra, pc_dec, out3); }

void or_xyzs_to_cross_uvws(const double* xyzs, int ntiles, double ha, double dec, double* uvws) {
    xyzs_to_cross_uvws(xyzs, ntiles, ha, dec, uvws);
}

void or_hadec_to_azel(double ha, double dec, double lat, double* az, double* el) { hadec_to_azel(ha, dec, lat, az, el); }

void or_analytic_beam(double az, double el, double freq, double* out8) { to_f64(analytic_beam(az, el, freq), out8); }

// Per-tile beam table of the components of type comp_type in sky-model
// order: out [uniq][nuf][n_type] JonesF64 from gains [uniq][2][16] at the
// unique frequencies ufreqs, for the given LST and latitude (the explicit
// per-tile layout of OrBeam kind 2).
void or_tile_beam_table(const OrSky* s, int comp_type, double lst, double lat, const double* gains, int nuniq,
                        const double* ufreqs, int nuf, double* out) {
    std::vector<int> idx;
    for (int c = 0; c < s->num_components; c++)
        if (s->comp_type[c] == comp_type) idx.push_back(c);
    const int n = (int)idx.size();
    for (int k = 0; k < n; k++) {
        double az, el;
        hadec_to_azel(lst - s->ra[idx[k]], s->dec[idx[k]], lat, &az, &el);
        for (int u = 0; u < nuniq; u++)
            for (int f = 0; f < nuf; f++)
                to_f64(analytic_beam_tile(az, el, ufreqs[f], gains + 32 * u), out + 8 * (((size_t)u * nuf + f) * n + k));
    }
}

// ---------------------------------------------------------------------------
// Predictor: SkyModellerCpu::model_points / model_gaussians / model_shapelets
// (model/cpu.rs:249-352, 371-495, 518-726) and model_timestep_with
// (model/cpu.rs:787-812).
//
// beam_kind: 0 none (identity), 1 analytic dipole array (shared by all tiles),
// 2 explicit per-tile Jones supplied per component type in `beam_jones[ty]`
// with layout [uniq_tile][uniq_freq][n_type] and maps tile_map[tile],
// freq_map[freq].
// out_mode: 0 -> accumulate into JonesF32 vis (reference demotion per type,
// cpu.rs:348); 1 -> accumulate into JonesF64 vis (pure f64, no demotion).
// ---------------------------------------------------------------------------
typedef struct OrBeam {
    int kind;
    const double* beam_jones[3];
    const int* tile_map;
    const int* freq_map;
    int num_unique_freqs;
} OrBeam;

}  // extern "C"

namespace {

// Beam Jones for component k of type ty, unique tile/freq indices (ut, uf).
struct BeamEval {
    const OrBeam* beam;
    int ntype;
    int ty;
    std::vector<J64> analytic;  // [f][k] when kind == 1
    J64 get(int tile, int f, int k) const {
        if (!beam || beam->kind == 0) return jidentity();
        if (beam->kind == 1) return analytic[(size_t)f * ntype + k];
        int ut = beam->tile_map[tile], uf = beam->freq_map[f];
        return from_f64(beam->beam_jones[ty] + 8 * (((size_t)ut * beam->num_unique_freqs + uf) * ntype + k));
    }
};

void prepare_beam(BeamEval& be, const OrBeam* beam, int ty, const OrSky* s, const std::vector<int>& idx, const double* freqs,
                  int nf, double lst, double lat) {
    be.beam = beam;
    be.ty = ty;
    be.ntype = (int)idx.size();
    if (beam && beam->kind == 1) {
        be.analytic.resize((size_t)nf * be.ntype);
        for (int k = 0; k < be.ntype; k++) {
            int c = idx[k];
            double az, el;
            hadec_to_azel(lst - s->ra[c], s->dec[c], lat, &az, &el);
            for (int f = 0; f < nf; f++) be.analytic[(size_t)f * be.ntype + k] = analytic_beam(az, el, freqs[f]);
        }
    }
}

void accumulate_out(void* vis, int out_mode, size_t i, const J64& acc) {
    if (out_mode == 0) {
        float* p = (float*)vis + 8 * i;
        float tmp[8];
        to_f32(acc, tmp);
        for (int k = 0; k < 8; k++) p[k] += tmp[k];
    } else {
        double* p = (double*)vis + 8 * i;
        for (int k = 0; k < 8; k++) p[k] += (k & 1) ? acc.j[k / 2].im : acc.j[k / 2].re;
    }
}

void model_type(int ty, const OrSky* s, const CompTables& t, const BeamEval& be, const double* uvws,
                const double* shapelet_uvws /*[bl][nshape][3]*/, const double* freqs, int nf, int ntiles, void* vis,
                int out_mode) {
    const std::vector<int>& idx = t.idx[ty];
    int nc = (int)idx.size();
    if (nc == 0) return;
    int nbl = ntiles * (ntiles - 1) / 2;
    std::vector<int> t1, t2;
    bl_to_tiles(ntiles, t1, t2);
    const double* sbf = g_sbf.data();
    static const c64 I_POWER[4] = {{1.0, 0.0}, {0.0, 1.0}, {-1.0, 0.0}, {0.0, -1.0}};

#pragma omp parallel for schedule(static)
    for (int b = 0; b < nbl; b++) {
        std::vector<c64> envelopes(ty == 2 ? nc : 0);
        for (int f = 0; f < nf; f++) {
            double freq = freqs[f];
            double u, v, w;
            double one_on_lambda = freq / VEL_C;
            if (ty == 2) {
                // cpu.rs:642-643: uvw * one_on_lambda
                u = uvws[3 * b] * one_on_lambda;
                v = uvws[3 * b + 1] * one_on_lambda;
                w = uvws[3 * b + 2] * one_on_lambda;
            } else {
                // cpu.rs:330: uvw * *freq / VEL_C
                u = uvws[3 * b] * freq / VEL_C;
                v = uvws[3 * b + 1] * freq / VEL_C;
                w = uvws[3 * b + 2] * freq / VEL_C;
            }
            if (ty == 2) {
                for (int k = 0; k < nc; k++) {
                    int c = idx[k];
                    double su = shapelet_uvws[3 * ((size_t)b * nc + k)] * one_on_lambda;
                    double sv = shapelet_uvws[3 * ((size_t)b * nc + k) + 1] * one_on_lambda;
                    double s_pa = std::sin(s->pa[c]), c_pa = std::cos(s->pa[c]);
                    double x = su * s_pa + sv * c_pa;
                    double y = su * c_pa - sv * s_pa;
                    double const_x = s->maj[c] * SHAPELET_CONST;
                    double const_y = -s->min[c] * SHAPELET_CONST;
                    double x_pos = x * const_x + SBF_C;
                    double y_pos = y * const_y + SBF_C;
                    long long xi = rs_as_usize(std::floor(x_pos));
                    long long yi = rs_as_usize(std::floor(y_pos));
                    // The reference reads unchecked; indices past the table end
                    // are clamped here (and in the product) to stay in bounds.
                    if (xi > SBF_L - 2) xi = SBF_L - 2;
                    if (yi > SBF_L - 2) yi = SBF_L - 2;
                    c64 env = {0.0, 0.0};
                    for (int q = 0; q < s->coeff_count[c]; q++) {
                        int ci = s->coeff_start[c] + q;
                        int n1 = s->coeff_n1[ci], n2 = s->coeff_n2[ci];
                        double f_hat = s->coeff_value[ci];
                        double x_low = sbf[(size_t)SBF_L * n1 + xi];
                        double x_high = sbf[(size_t)SBF_L * n1 + xi + 1];
                        double u_value = x_low + (x_high - x_low) * (x_pos - std::floor(x_pos));
                        double y_low = sbf[(size_t)SBF_L * n2 + yi];
                        double y_high = sbf[(size_t)SBF_L * n2 + yi + 1];
                        double v_value = y_low + (y_high - y_low) * (y_pos - std::floor(y_pos));
                        c64 term = cscale(cscale(cscale(I_POWER[(n1 + n2) % 4], f_hat), u_value), v_value);
                        env = cadd(env, term);
                    }
                    envelopes[k] = env;
                }
            }
            J64 acc = jzero();
            for (int k = 0; k < nc; k++) {
                int c = idx[k];
                const double* lmn = &t.lmn[ty][3 * k];
                J64 fd = t.fds[ty][(size_t)f * nc + k];
                J64 b1 = be.get(t1[b], f, k), b2 = be.get(t2[b], f, k);
                J64 bsb = jmul(jmul(b1, fd), jh(b2));
                double arg = u * lmn[0] + v * lmn[1] + w * lmn[2];
                J64 term = jmulc(bsb, cis(arg));
                if (ty == 1) {
                    double s_pa = std::sin(s->pa[c]), c_pa = std::cos(s->pa[c]);
                    double k_x = u * s_pa + v * c_pa;
                    double k_y = u * c_pa - v * s_pa;
                    double maj = s->maj[c], mn = s->min[c];
                    double env = std::exp(GAUSSIAN_EXP_CONST * (maj * maj * (k_x * k_x) + mn * mn * (k_y * k_y)));
                    term = jscale(term, env);
                } else if (ty == 2) {
                    term = jmulc(term, envelopes[k]);
                }
                acc = jadd(acc, term);
            }
            accumulate_out(vis, out_mode, (size_t)f * nbl + b, acc);
        }
    }
}

// model/mod.rs:264-285
void mask_pols_f32(float* vis, size_t n, int pols) {
    if (pols == 0) return;
    for (size_t i = 0; i < n; i++) {
        float* p = vis + 8 * i;
        bool keep[4] = {false, false, false, false};
        if (pols == 1) keep[0] = true;                                    // XX
        if (pols == 2) keep[3] = true;                                    // YY
        if (pols == 3) keep[0] = keep[3] = true;                          // XX_YY
        if (pols == 4) keep[0] = keep[1] = keep[3] = true;                // XX_YY_XY
        for (int k = 0; k < 4; k++)
            if (!keep[k]) p[2 * k] = p[2 * k + 1] = 0.0f;
    }
}

}  // namespace

extern "C" {

// ShapeletComponentParams::get_shapelet_uvws (components/mod.rs:279-298) for
// the shapelet components (in sky-model order). out: [nbl][nshape][3].
void or_shapelet_uvws(const OrSky* s, const double* xyzs, int ntiles, double lst, double* out) {
    std::vector<int> idx;
    for (int c = 0; c < s->num_components; c++)
        if (s->comp_type[c] == 2) idx.push_back(c);
    int nsh = (int)idx.size(), nbl = ntiles * (ntiles - 1) / 2;
    std::vector<double> tmp(3 * (size_t)nbl);
    for (int k = 0; k < nsh; k++) {
        int c = idx[k];
        xyzs_to_cross_uvws(xyzs, ntiles, lst - s->ra[c], s->dec[c], tmp.data());
        for (int b = 0; b < nbl; b++)
            for (int q = 0; q < 3; q++) out[3 * ((size_t)b * nsh + k) + q] = tmp[3 * b + q];
    }
}

// One type of the predictor with caller-supplied baseline UVWs, as the
// reference's model tests call SkyModellerCpu::model_points etc. directly.
// comp_type selects points/Gaussians/shapelets.
int or_model_type(int comp_type, const OrSky* s, const double* xyzs, int ntiles, const double* freqs, int nf, double pc_ra,
                  double pc_dec, double lst, double lat, const double* uvws, const OrBeam* beam, void* vis, int out_mode) {
    build_sbf();
    CompTables t;
    build_tables(s, freqs, nf, pc_ra, pc_dec, t);
    BeamEval be;
    prepare_beam(be, beam, comp_type, s, t.idx[comp_type], freqs, nf, lst, lat);
    std::vector<double> suv;
    if (comp_type == 2) {
        int nbl = ntiles * (ntiles - 1) / 2;
        suv.resize(3 * (size_t)nbl * t.idx[2].size() + 3);
        or_shapelet_uvws(s, xyzs, ntiles, lst, suv.data());
    }
    model_type(comp_type, s, t, be, uvws, suv.data(), freqs, nf, ntiles, vis, out_mode);
    return 0;
}

// SkyModeller::model_timestep_with without precession (model/cpu.rs:787-812):
// UVWs from the tile XYZs at the phase centre's hour angle (lst - ra), then
// points, Gaussians, shapelets, then mask_pols (f32 mode). uvws_out may be NULL.
int or_model_timestep(const OrSky* s, const double* xyzs, int ntiles, const double* freqs, int nf, double pc_ra,
                      double pc_dec, double lst, double lat, const OrBeam* beam, int pols, void* vis, int out_mode,
                      double* uvws_out) {
    build_sbf();
    int nbl = ntiles * (ntiles - 1) / 2;
    std::vector<double> uvws(3 * (size_t)nbl + 3);
    xyzs_to_cross_uvws(xyzs, ntiles, lst - pc_ra, pc_dec, uvws.data());
    CompTables t;
    build_tables(s, freqs, nf, pc_ra, pc_dec, t);
    std::vector<double> suv(3 * (size_t)nbl * t.idx[2].size() + 3);
    or_shapelet_uvws(s, xyzs, ntiles, lst, suv.data());
    for (int ty = 0; ty < 3; ty++) {
        BeamEval be;
        prepare_beam(be, beam, ty, s, t.idx[ty], freqs, nf, lst, lat);
        model_type(ty, s, t, be, uvws.data(), suv.data(), freqs, nf, ntiles, vis, out_mode);
    }
    if (out_mode == 0) mask_pols_f32((float*)vis, (size_t)nf * nbl, pols);
    if (uvws_out) std::memcpy(uvws_out, uvws.data(), sizeof(double) * 3 * nbl);
    return 0;
}

// SkyModeller::model_timestep_autos_with (model/cpu.rs:854-935), no
// precession. vis: [nf][ntiles] JonesF32 (accumulated).
int or_model_autos(const OrSky* s, int ntiles, const double* freqs, int nf, double lst, double lat, const OrBeam* beam,
                   float* vis) {
    CompTables t;
    build_tables(s, freqs, nf, 0.0, 0.0, t);
    for (int ty = 0; ty < 3; ty++) {
        int nc = (int)t.idx[ty].size();
        if (nc == 0) continue;
        BeamEval be;
        prepare_beam(be, beam, ty, s, t.idx[ty], freqs, nf, lst, lat);
        for (int tile = 0; tile < ntiles; tile++)
            for (int f = 0; f < nf; f++) {
                J64 acc = jzero();
                for (int k = 0; k < nc; k++) {
                    J64 b = be.get(tile, f, k);
                    acc = jadd(acc, jmul(jmul(b, t.fds[ty][(size_t)f * nc + k]), jh(b)));
                }
                float tmp[8];
                to_f32(acc, tmp);
                float* p = vis + 8 * ((size_t)f * ntiles + tile);
                for (int q = 0; q < 8; q++) p[q] += tmp[q];
            }
    }
    return 0;
}

// ---------------------------------------------------------------------------
// DI calibration: di_calibrate/mod.rs
// ---------------------------------------------------------------------------
typedef struct OrCalResult {
    int num_iterations;
    int converged;
    double max_precision;
    int num_failed;
} OrCalResult;

}  // extern "C"

namespace {

// di_calibrate/mod.rs:900-968 (calibration_loop; MitchCal eq. 11).
// data/model: [nt][nchan_total][nbl], we read chanblock `ch` only.
void calibration_loop(const float* data, const float* model, int nt, int nchan, int ch, int nbl, int ntiles,
                      const J64* di_jones, J64* top, J64* bot) {
    for (int t = 0; t < nt; t++) {
        int i1 = 0, i2 = 0;
        for (int b = 0; b < nbl; b++) {
            i2 += 1;
            if (i2 == ntiles) {
                i1 += 1;
                i2 = i1 + 1;
            }
            size_t off = 8 * (((size_t)t * nchan + ch) * nbl + b);
            J64 D = from_f32(data + off);
            J64 M = from_f32(model + off);
            {
                J64 J2 = di_jones[i2];
                J64 Z = jmul(J2, jh(M));
                top[i1] = jadd(top[i1], jmul(D, Z));
                bot[i1] = jadd(bot[i1], jmul(jh(Z), Z));
            }
            {
                J64 J1 = di_jones[i1];
                J64 Z = jmul(J1, M);
                top[i2] = jadd(top[i2], jmul(jh(D), Z));
                bot[i2] = jadd(bot[i2], jmul(jh(Z), Z));
            }
        }
    }
}

J64 div_func(const J64& top, const J64& bot, int pols) {
    if (pols == 1) {
        J64 r = jzero();
        r.j[0] = cdiv(top.j[0], bot.j[0]);
        return r;
    }
    if (pols == 2) {
        J64 r = jzero();
        r.j[3] = cdiv(top.j[3], bot.j[3]);
        return r;
    }
    return jmul(top, jinv(bot));
}

// di_calibrate/mod.rs:640-893 (calibrate). di_jones: [ntiles] in/out.
OrCalResult calibrate(const float* data, const float* model, int nt, int nchan, int ch, int nbl, J64* di_jones, int ntiles,
                      int max_iterations, double stop_threshold, double min_threshold, int pols) {
    std::vector<J64> old_jones(ntiles, jzero()), top(ntiles), bot(ntiles);
    std::vector<double> precisions(4 * (size_t)ntiles, 0.0);
    std::vector<char> failed(ntiles, 0);
    int iteration = 0;
    while (iteration < max_iterations) {
        iteration += 1;
        std::fill(top.begin(), top.end(), jzero());
        std::fill(bot.begin(), bot.end(), jzero());
        calibration_loop(data, model, nt, nchan, ch, nbl, ntiles, di_jones, top.data(), bot.data());

        if (iteration == 1) {
            bool eq = true, zeros = true;
            for (int i = 0; i < ntiles; i++) {
                J64 diff = jsub(top[i], bot[i]);
                for (int k = 0; k < 8; k++) {
                    double d = (k & 1) ? diff.j[k / 2].im : diff.j[k / 2].re;
                    if (std::fabs(d) > stop_threshold) {
                        eq = false;
                        zeros = false;
                        break;
                    }
                }
                if (!eq && !zeros) break;
                if (zeros) {
                    for (int k = 0; k < 8; k++) {
                        double d = (k & 1) ? top[i].j[k / 2].im : top[i].j[k / 2].re;
                        if (std::fabs(d) > 2.220446049250313e-16) {
                            zeros = false;
                            break;
                        }
                    }
                }
                if (zeros) {
                    for (int k = 0; k < 8; k++) {
                        double d = (k & 1) ? bot[i].j[k / 2].im : bot[i].j[k / 2].re;
                        if (std::fabs(d) > 2.220446049250313e-16) {
                            zeros = false;
                            break;
                        }
                    }
                }
                if (!eq && !zeros) break;
            }
            if (eq) {
                if (zeros) std::fill(failed.begin(), failed.end(), 1);
                break;
            }
        }

        for (int i = 0; i < ntiles; i++) {
            if (failed[i]) continue;
            J64 div = div_func(top[i], bot[i], pols);
            if (jany_nan(div)) {
                failed[i] = 1;
                di_jones[i] = jzero();
                old_jones[i] = jzero();
            } else {
                di_jones[i] = div;
            }
        }

        int num_failed = 0;
        for (int i = 0; i < ntiles; i++) num_failed += failed[i];
        if (ntiles - num_failed <= 4) break;

        if (iteration % 2 == 0) {
            for (int i = 0; i < ntiles; i++) {
                if (failed[i]) continue;
                J64 diff = jsub(di_jones[i], old_jones[i]);
                for (int k = 0; k < 4; k++) precisions[4 * i + k] = cnorm_sqr(diff.j[k]);
                di_jones[i] = jscale(jadd(di_jones[i], old_jones[i]), 0.5);
            }
            bool all_below = true;
            for (size_t k = 0; k < precisions.size(); k++)
                if (!(precisions[k] < stop_threshold)) {
                    all_below = false;
                    break;
                }
            if (all_below) break;
        }
        for (int i = 0; i < ntiles; i++) old_jones[i] = di_jones[i];
    }

    for (int i = 0; i < ntiles; i++)
        if (failed[i]) di_jones[i] = jnan();

    double max_precision = -1.7976931348623157e308;  // f64::MIN
    for (int i = 0; i < ntiles; i++) {
        if (failed[i]) continue;
        // Rust f64::max ignores NaN
        for (int k = 3; k >= 0; k--) {
            double p = precisions[4 * i + k];
            max_precision = std::isnan(p) ? max_precision : (std::isnan(max_precision) ? p : std::max(max_precision, p));
        }
    }
    int num_failed = 0;
    for (int i = 0; i < ntiles; i++) num_failed += failed[i];
    bool converged;
    if (ntiles - num_failed <= 4 || max_precision > min_threshold) {
        for (int i = 0; i < ntiles; i++) di_jones[i] = jnan();
        converged = false;
    } else {
        converged = true;
    }
    return OrCalResult{iteration, converged ? 1 : 0, max_precision, num_failed};
}

}  // namespace

extern "C" {

// calibrate() for one chanblock; di_jones [ntiles] JonesF64 in/out.
int or_calibrate(const float* data, const float* model, int nt, int nchan, int ch, int nbl, double* di_jones, int max_iter,
                 double stop, double min, int pols, OrCalResult* res) {
    int ntiles = (int)((1.0 + std::sqrt(1.0 + 8.0 * nbl)) / 2.0 + 0.5);
    std::vector<J64> dj(ntiles);
    for (int i = 0; i < ntiles; i++) dj[i] = from_f64(di_jones + 8 * i);
    *res = calibrate(data, model, nt, nchan, ch, nbl, dj.data(), ntiles, max_iter, stop, min, pols);
    for (int i = 0; i < ntiles; i++) to_f64(dj[i], di_jones + 8 * i);
    return 0;
}

// calibrate_timeblock (di_calibrate/mod.rs:387-618) over a timestep range
// [t0, t1) of data/model [nt_total][nchanblocks][nbl]. di_jones: [ntiles]
// [nchanblocks] (this timeblock's slice) in/out. results: [nchanblocks].
// Chanblocks are taken as unflagged indices 0..nchanblocks-1.
int or_calibrate_timeblock(const float* data, const float* model, int nt_total, int t0, int t1, int nchanblocks, int nbl,
                           double* di_jones, int max_iter, double stop, double min, int pols, OrCalResult* results) {
    int ntiles = (int)((1.0 + std::sqrt(1.0 + 8.0 * nbl)) / 2.0 + 0.5);
    (void)nt_total;
    const float* d0 = data + 8 * (size_t)t0 * nchanblocks * nbl;
    const float* m0 = model + 8 * (size_t)t0 * nchanblocks * nbl;
    int nt = t1 - t0;
    // di_jones_rev[chanblock][tile]
    std::vector<J64> rev((size_t)nchanblocks * ntiles);
    for (int i = 0; i < ntiles; i++)
        for (int c = 0; c < nchanblocks; c++) rev[(size_t)c * ntiles + i] = from_f64(di_jones + 8 * ((size_t)i * nchanblocks + c));

#pragma omp parallel for schedule(dynamic, 1)
    for (int c = 0; c < nchanblocks; c++)
        results[c] = calibrate(d0, m0, nt, nchanblocks, c, nbl, &rev[(size_t)c * ntiles], ntiles, max_iter, stop, min, pols);

    int total_converged = 0;
    for (int c = 0; c < nchanblocks; c++) total_converged += results[c].converged;
    if (total_converged > 0 && total_converged != nchanblocks) {
        int new_converged = 1;
        while (new_converged > 0 && total_converged != nchanblocks) {
            // pairs of converged chanblocks around runs of failures
            std::vector<std::pair<int, int>> pairs;  // -1 = None
            int left = -1;
            bool in_failures = false;
            for (int c = 0; c < nchanblocks; c++) {
                bool conv = results[c].converged != 0;
                if (!in_failures && conv)
                    left = c;
                else if (!in_failures && !conv)
                    in_failures = true;
                else if (in_failures && conv) {
                    in_failures = false;
                    pairs.push_back({left, c});
                    left = c;
                }
            }
            // Note: a trailing failure run is only recorded as (Some(l), None)
            // if the reference loop records it; the reference only pushes
            // pairs when a converged chanblock follows a failure run
            // (mod.rs:486-497), so trailing runs are not re-seeded.
            for (auto& p : pairs) {
                int l = p.first, r = p.second;
                if (l >= 0 && r >= 0) {
                    for (int i = l + 1; i < r; i++) {
                        double lw = (double)(r - i), rw = (double)(i - l);
                        for (int tt = 0; tt < ntiles; tt++) {
                            J64 a = jscale(rev[(size_t)l * ntiles + tt], lw);
                            J64 b = jscale(rev[(size_t)r * ntiles + tt], rw);
                            // (&left * lw + &right * rw) / (r - l)
                            J64 sum = jadd(a, b);
                            double d = (double)(r - l);
                            J64 out;
                            for (int k = 0; k < 4; k++) out.j[k] = {sum.j[k].re / d, sum.j[k].im / d};
                            rev[(size_t)i * ntiles + tt] = out;
                        }
                    }
                } else if (l < 0 && r >= 0) {
                    for (int i = 0; i < r; i++)
                        for (int tt = 0; tt < ntiles; tt++) rev[(size_t)i * ntiles + tt] = rev[(size_t)r * ntiles + tt];
                }
            }
#pragma omp parallel for schedule(dynamic, 1)
            for (int c = 0; c < nchanblocks; c++) {
                if (results[c].converged) continue;
                OrCalResult nr = calibrate(d0, m0, nt, nchanblocks, c, nbl, &rev[(size_t)c * ntiles], ntiles, max_iter, stop,
                                           min, pols);
                if (std::fabs(nr.max_precision) > 1e100) nr.max_precision = NAN;
                results[c] = nr;
            }
            int tmp = 0;
            for (int c = 0; c < nchanblocks; c++) tmp += results[c].converged;
            new_converged = tmp - total_converged;
            total_converged = tmp;
        }
    }
    for (int i = 0; i < ntiles; i++)
        for (int c = 0; c < nchanblocks; c++) to_f64(rev[(size_t)c * ntiles + i], di_jones + 8 * ((size_t)i * nchanblocks + c));
    return 0;
}

// ---------------------------------------------------------------------------
// Peel kernels, restating the reference GPU kernels' semantics
// (gpu/peel.cu). Arrays are [t][f][bl] JonesF32 / f32 weights, UVW f64.
// ---------------------------------------------------------------------------

// peel.cu:17-48 xyzs_to_uvws: xyzs [t][tile], lmsts [t], uvws [t][bl].
// Differences the XYZs first, then rotates (unlike xyzs_to_cross_uvws).
int or_xyzs_to_uvws(const double* xyzs, const double* lmsts, double* uvws, double pc_ra, double pc_dec, int ntiles, int nbl,
                    int nt) {
    std::vector<int> t1, t2;
    bl_to_tiles(ntiles, t1, t2);
    double s_dec = std::sin(pc_dec), c_dec = std::cos(pc_dec);
    for (int t = 0; t < nt; t++) {
        double ha = lmsts[t] - pc_ra;
        double s_ha = std::sin(ha), c_ha = std::cos(ha);
        for (int b = 0; b < nbl; b++) {
            const double* a = xyzs + 3 * ((size_t)t * ntiles + t1[b]);
            const double* c = xyzs + 3 * ((size_t)t * ntiles + t2[b]);
            double x = a[0] - c[0], y = a[1] - c[1], z = a[2] - c[2];
            double* o = uvws + 3 * ((size_t)t * nbl + b);
            o[0] = s_ha * x + c_ha * y;
            o[1] = -s_dec * c_ha * x + s_dec * s_ha * y + c_dec * z;
            o[2] = c_dec * c_ha * x - c_dec * s_ha * y + s_dec * z;
        }
    }
    return 0;
}

// peel.cu:56-102 rotate (in place), f64 internal.
int or_rotate(float* vis, int nt, int nbl, int nf, const double* uvws_from, const double* uvws_to, const double* lambdas) {
#pragma omp parallel for schedule(static)
    for (int b = 0; b < nbl; b++)
        for (int f = 0; f < nf; f++)
            for (int t = 0; t < nt; t++) {
                double arg = -TAU * (uvws_to[3 * ((size_t)t * nbl + b) + 2] - uvws_from[3 * ((size_t)t * nbl + b) + 2]);
                double x = arg / lambdas[f];
                c64 rot = {std::cos(x), std::sin(x)};
                float* p = vis + 8 * (((size_t)t * nf + f) * nbl + b);
                to_f32(jmulc(from_f32(p), rot), p);
            }
    return 0;
}

// peel.cu:111-176 average (time and frequency); low: [f_lo][bl].
int or_average(const float* hi, const float* w, float* lo, int nt, int nbl, int nf, int favg) {
#pragma omp parallel for schedule(static)
    for (int b = 0; b < nbl; b++)
        for (int f = 0; f < nf; f += favg) {
            J64 sum = jzero();
            double ws = 0.0;
            for (int t = 0; t < nt; t++)
                for (int fc = f; fc < f + favg; fc++) {
                    size_t step = ((size_t)t * nf + fc) * nbl + b;
                    double wt = w[step];
                    sum = jadd(sum, jscale(from_f32(hi + 8 * step), wt));
                    ws += wt;
                }
            double d = ws > 0.0 ? ws : 1.0;
            J64 out;
            for (int k = 0; k < 4; k++) out.j[k] = {sum.j[k].re / d, sum.j[k].im / d};
            to_f32(out, lo + 8 * ((size_t)(f / favg) * nbl + b));
        }
    return 0;
}

typedef struct OrIono {
    double alpha, beta, gain;
} OrIono;

// peel.cu:437-486 + 250-432 + 657-717: iono_loop on low-res [f][bl] arrays,
// uvws [bl]. Updates `consts` (starts from the caller's value) for
// num_iterations, stopping early only when gain < 0 (peel.cu:711).
int or_iono_loop(const float* resid, const float* weights, const float* model, float* model_rot, OrIono* consts, int nbl,
                 int nf, int niter, const double* uvws, const double* lambdas, double convergence) {
    for (int it = 0; it < niter; it++) {
        double sums[7] = {0, 0, 0, 0, 0, 0, 0};
        for (int f = 0; f < nf; f++) {
            double fs[7] = {0, 0, 0, 0, 0, 0, 0};
            for (int b = 0; b < nbl; b++) {
                double u = uvws[3 * b], v = uvws[3 * b + 1];
                double arg = -TAU * (u * consts->alpha + v * consts->beta);
                double x = arg * lambdas[f];
                c64 rot = cscale(c64{std::cos(x), std::sin(x)}, consts->gain);
                size_t step = (size_t)f * nbl + b;
                // peel.cu:479: vis_out = vis * (complex * gain), JonesF32 * C64
                float mr32[8];
                jf32_mul_c64(model + 8 * step, rot, mr32);
                std::memcpy(model_rot + 8 * step, mr32, sizeof(mr32));
                double wt = weights[step];
                const float* r = resid + 8 * step;
                double ri_re = (double)r[0] + (double)r[6];
                double ri_im = (double)r[1] + (double)r[7];
                double mi_re = (double)mr32[0] + (double)mr32[6];
                double mi_im = (double)mr32[1] + (double)mr32[7];
                double mr = mi_re * (ri_im - mi_im);
                double mm = mi_re * mi_re;
                fs[0] += wt * mm * u * u;
                fs[1] += wt * mm * u * v;
                fs[2] += wt * mm * v * v;
                fs[3] += wt * mr * u;
                fs[4] += wt * mr * v;
                fs[5] += wt * mi_re * ri_re;
                fs[6] += wt * mm;
            }
            double lam = lambdas[f], lam2 = lam * lam;
            sums[0] += fs[0] * lam2;
            sums[1] += fs[1] * lam2;
            sums[2] += fs[2] * lam2;
            sums[3] += fs[3] * -lam;
            sums[4] += fs[4] * -lam;
            sums[5] += fs[5];
            sums[6] += fs[6];
        }
        double a_uu = sums[0], a_uv = sums[1], a_vv = sums[2], A_u = sums[3], A_v = sums[4], s_vm = sums[5], s_mm = sums[6];
        double denom = TAU * (a_uu * a_vv - a_uv * a_uv);
        consts->alpha += convergence * (A_u * a_vv - A_v * a_uv) / denom;
        consts->beta += convergence * (A_v * a_uu - A_u * a_uv) / denom;
        consts->gain *= 1. + convergence * (s_vm / s_mm - 1);
        if (consts->gain < 0.0) break;
    }
    return 0;
}

// peel.cu:488-557 subtract_iono: residual += m*old - m*new, uvws [t][bl].
int or_subtract_iono(float* resid, const float* model, OrIono c, OrIono old, const double* uvws, const double* lambdas,
                     int nt, int nbl, int nf) {
#pragma omp parallel for schedule(static)
    for (int b = 0; b < nbl; b++)
        for (int t = 0; t < nt; t++) {
            double u = uvws[3 * ((size_t)t * nbl + b)], v = uvws[3 * ((size_t)t * nbl + b) + 1];
            double arg = -TAU * (u * c.alpha + v * c.beta);
            double old_arg = -TAU * (u * old.alpha + v * old.beta);
            for (int f = 0; f < nf; f++) {
                double lam = lambdas[f];
                c64 cn = {std::cos(arg * lam), std::sin(arg * lam)};
                c64 co = {std::cos(old_arg * lam), std::sin(old_arg * lam)};
                size_t step = ((size_t)t * nf + f) * nbl + b;
                J64 r = from_f32(resid + 8 * step);
                J64 m = from_f32(model + 8 * step);
                r = jadd(r, jmulc(m, cscale(co, old.gain)));
                r = jsub(r, jmulc(m, cscale(cn, c.gain)));
                to_f32(r, resid + 8 * step);
            }
        }
    return 0;
}

// peel.cu:559-592 add_model: residual += model * cis(arg*lambda) * gain.
int or_add_model(float* resid, const float* model, OrIono c, const double* lambdas, const double* uvws, int nt, int nf,
                 int nbl) {
#pragma omp parallel for schedule(static)
    for (int b = 0; b < nbl; b++)
        for (int t = 0; t < nt; t++) {
            double u = uvws[3 * ((size_t)t * nbl + b)], v = uvws[3 * ((size_t)t * nbl + b) + 1];
            double arg = -TAU * (u * c.alpha + v * c.beta);
            for (int f = 0; f < nf; f++) {
                c64 cx;
                if (c.alpha == 0.0 && c.beta == 0.0)
                    cx = {1.0, 0.0};
                else
                    cx = {std::cos(arg * lambdas[f]), std::sin(arg * lambdas[f])};
                size_t step = ((size_t)t * nf + f) * nbl + b;
                float* p = resid + 8 * step;
                float tmp[8];
                jf32_mul_c64(model + 8 * step, cscale(cx, c.gain), tmp);
                for (int k = 0; k < 8; k++) p[k] += tmp[k];
            }
        }
    return 0;
}

// ---------------------------------------------------------------------------
// Peel CPU helpers (params/peel/mod.rs)
// ---------------------------------------------------------------------------

// mod.rs:960-1076 iono_fit: low-res [t][f][bl], tile_uvs [t][tile][2].
// Returns alpha, beta, s_vm, s_mm.
void or_iono_fit(const float* resid, const float* weights, const float* model, const double* lambdas, const double* tile_uvs,
                 int nt, int nf, int ntiles, double* out4) {
    int nbl = ntiles * (ntiles - 1) / 2;
    double a_uu = 0, a_uv = 0, a_vv = 0, A_u = 0, A_v = 0, s_vm = 0, s_mm = 0;
    for (int t = 0; t < nt; t++)
        for (int f = 0; f < nf; f++) {
            double lambda = lambdas[f], lambda_2 = lambda * lambda;
            int i1 = 0, i2 = 0;
            const double* uv1 = tile_uvs + 2 * ((size_t)t * ntiles + i1);
            double ab[7] = {0, 0, 0, 0, 0, 0, 0};
            for (int b = 0; b < nbl; b++) {
                i2 += 1;
                if (i2 == ntiles) {
                    i1 += 1;
                    i2 = i1 + 1;
                    uv1 = tile_uvs + 2 * ((size_t)t * ntiles + i1);
                }
                size_t step = ((size_t)t * nf + f) * nbl + b;
                float wt32 = weights[step];
                if (wt32 > 0.0f) {
                    const double* uv2 = tile_uvs + 2 * ((size_t)t * ntiles + i2);
                    double u = uv1[0] - uv2[0], v = uv1[1] - uv2[1];
                    const float* r = resid + 8 * step;
                    const float* m = model + 8 * step;
                    // Complex<f32> additions
                    float ri_re = r[0] + r[6], ri_im = r[1] + r[7];
                    float mi_re = m[0] + m[6], mi_im = m[1] + m[7];
                    double model_i_re = (double)mi_re;
                    double mr = model_i_re * ((double)ri_im - (double)mi_im);
                    double mm = model_i_re * model_i_re;
                    double svm = model_i_re * (double)ri_re;
                    double wt = (double)wt32;
                    ab[0] += wt * mm * u * u;
                    ab[1] += wt * mm * u * v;
                    ab[2] += wt * mm * v * v;
                    ab[3] += wt * mr * u;
                    ab[4] += wt * mr * v;
                    ab[5] += wt * svm;
                    ab[6] += wt * mm;
                }
            }
            a_uu += ab[0] * lambda_2;
            a_uv += ab[1] * lambda_2;
            a_vv += ab[2] * lambda_2;
            A_u += ab[3] * -lambda;
            A_v += ab[4] * -lambda;
            s_vm += ab[5];
            s_mm += ab[6];
        }
    double denom = TAU * (a_uu * a_vv - a_uv * a_uv);
    out4[0] = (A_u * a_vv - A_v * a_uv) / denom;
    out4[1] = (A_v * a_uu - A_u * a_uv) / denom;
    out4[2] = s_vm;
    out4[3] = s_mm;
}

// mod.rs:854-893 apply_iono_fb (per timestep slab [f][bl]); tile_uvs [tile][2]
void or_apply_iono_fb(const float* vis, float* out, const double* tile_uvs, int ntiles, int nf, OrIono c,
                      const double* lambdas) {
    int nbl = ntiles * (ntiles - 1) / 2;
    int i1 = 0, i2 = 0;
    for (int b = 0; b < nbl; b++) {
        i2 += 1;
        if (i2 == ntiles) {
            i1 += 1;
            i2 = i1 + 1;
        }
        double u = tile_uvs[2 * i1] - tile_uvs[2 * i2], v = tile_uvs[2 * i1 + 1] - tile_uvs[2 * i2 + 1];
        double arg = -TAU * (u * c.alpha + v * c.beta);
        for (int f = 0; f < nf; f++) {
            c64 rot = cscale(cis(arg * lambdas[f]), c.gain);
            size_t step = (size_t)f * nbl + b;
            to_f32(jmulc(from_f32(vis + 8 * step), rot), out + 8 * step);
        }
    }
}

// mod.rs:605-642 get_weights_rts: tile_uvs [t][tile][2] -> weights [t][f][bl]
void or_weights_rts(const double* tile_uvs, int nt, int ntiles, const double* lambdas, int nf, double sigma, float* out) {
    int nbl = ntiles * (ntiles - 1) / 2;
    for (int t = 0; t < nt; t++) {
        int i1 = 0, i2 = 0;
        for (int b = 0; b < nbl; b++) {
            i2 += 1;
            if (i2 == ntiles) {
                i1 += 1;
                i2 = i1 + 1;
            }
            const double* a = tile_uvs + 2 * ((size_t)t * ntiles + i1);
            const double* c = tile_uvs + 2 * ((size_t)t * ntiles + i2);
            double u0 = a[0] - c[0], v0 = a[1] - c[1];
            for (int f = 0; f < nf; f++) {
                double u = u0 / lambdas[f], v = v0 / lambdas[f];
                double uv_sq = u * u + v * v;
                double e = std::exp(-uv_sq / (2.0 * sigma * sigma));
                out[((size_t)t * nf + f) * nbl + b] = (float)(1.0 - e);
            }
        }
    }
}

// params/di_calibration.rs:578-625 (CalVis::scale_by_weights): data and model
// [t][f][bl] times f64(weight) * baseline weight (cycled over baselines),
// stored back as FP32; a product <= 0 zeroes both.
int or_scale_by_weights(float* data, float* model, const float* weights, int nt, int nf, int nbl,
                        const double* bl_weights) {
    const size_t n = (size_t)nt * nf * nbl;
    for (size_t i = 0; i < n; i++) {
        const double w = (double)weights[i] * (bl_weights ? bl_weights[i % nbl] : 1.0);
        if (w <= 0.0) {
            for (int k = 0; k < 8; k++) data[8 * i + k] = model[8 * i + k] = 0.0f;
        } else {
            to_f32(jscale(from_f32(data + 8 * i), w), data + 8 * i);
            to_f32(jscale(from_f32(model + 8 * i), w), model + 8 * i);
        }
    }
    return 0;
}

// averaging/mod.rs:537-600 (vis_average) and 606-648
// (vis_average_weights_non_zero): all nt timesteps into one; channel chunks
// of ceil(nf / (nout + nflag)) channels with the flagged chunk indices
// skipped; per output the FP64 sums in (t, f) order.
int or_vis_average(const float* from, const float* wfrom, int nt, int nf, int nbl, const int* flagged, int nflag,
                   float* to, float* wto, int nout) {
    const int nchunks = nout + nflag;
    const int avg_freq = (int)std::ceil((double)nf / (double)nchunks);
    int o = 0;
    for (int c = 0; c < nchunks && o < nout; c++) {
        bool skip = false;
        for (int k = 0; k < nflag; k++) skip |= flagged[k] == c;
        if (skip) continue;
        const int f0 = c * avg_freq, f1 = std::min(f0 + avg_freq, nf);
        for (int b = 0; b < nbl; b++) {
            J64 ws = jzero(), s = jzero();
            double wsum = 0.0, fsum = 0.0;
            bool all_flagged = true;
            for (int t = 0; t < nt; t++)
                for (int f = f0; f < f1; f++) {
                    const size_t i = ((size_t)t * nf + f) * nbl + b;
                    const J64 v = from_f32(from + 8 * i);
                    s = jadd(s, v);
                    const double wa = std::fabs((double)wfrom[i]);
                    if (wfrom[i] > 0.0f) {
                        all_flagged = false;
                        ws = jadd(ws, jscale(v, wa));
                        wsum += wa;
                    } else {
                        fsum += wa;
                    }
                }
            J64 r;
            float wr;
            if (all_flagged || wsum <= 0.0) {
                const double len = (double)nt * (f1 - f0);
                for (int k = 0; k < 4; k++) r.j[k] = {s.j[k].re / len, s.j[k].im / len};
                wr = (float)-fsum;
            } else {
                for (int k = 0; k < 4; k++) r.j[k] = {ws.j[k].re / wsum, ws.j[k].im / wsum};
                wr = (float)wsum;
            }
            to_f32(r, to + 8 * ((size_t)o * nbl + b));
            wto[(size_t)o * nbl + b] = wr;
        }
        o++;
    }
    return o == nout ? 0 : 1;
}

// di_calibrate/mod.rs:89-176 (into_cal_sols): [tb][unflagged tile][unflagged
// chanblock] model->data gains to [tb][tile][chanblock] data->model
// solutions; inverted as marlu Jones::inv (jinv) or, for XX / YY only data,
// Complex::inv of that entry; NaN where a tile or chanblock is flagged.
int or_into_cal_sols(const double* in, int ntb, int nut, int nuc, const int* ftiles, int nft, const int* fchans,
                     int nfc, int pols, double* out) {
    const int ntt = nut + nft, ntc = nuc + nfc;
    std::vector<char> tf(ntt, 0), cf(ntc, 0);
    for (int k = 0; k < nft; k++) tf[ftiles[k]] = 1;
    for (int k = 0; k < nfc; k++) cf[fchans[k]] = 1;
    for (int tb = 0; tb < ntb; tb++) {
        int ut = 0;
        for (int t = 0; t < ntt; t++) {
            int uc = 0;
            for (int c = 0; c < ntc; c++) {
                double* o = out + 8 * (((size_t)tb * ntt + t) * ntc + c);
                if (tf[t] || cf[c]) {
                    for (int k = 0; k < 8; k++) o[k] = NAN;
                    continue;
                }
                const double* p = in + 8 * (((size_t)tb * nut + ut) * nuc + uc);
                J64 j;
                for (int k = 0; k < 4; k++) j.j[k] = {p[2 * k], p[2 * k + 1]};
                J64 r = jzero();
                if (pols == 1) {
                    const double n = cnorm_sqr(j.j[0]);
                    r.j[0] = {j.j[0].re / n, -j.j[0].im / n};
                } else if (pols == 2) {
                    const double n = cnorm_sqr(j.j[3]);
                    r.j[3] = {j.j[3].re / n, -j.j[3].im / n};
                } else {
                    r = jinv(j);
                }
                for (int k = 0; k < 4; k++) o[2 * k] = r.j[k].re, o[2 * k + 1] = r.j[k].im;
                uc++;
            }
            if (!tf[t]) ut++;
        }
    }
    return 0;
}


// ---------------------------------------------------------------------------
// peel_cpu (params/peel/mod.rs:1121-1475), the reference's CPU peel loop, with
// its helpers vis_rotate_tfb (:783-825), apply_iono_tfb (:829-893),
// vis_average_tfb (:648-707), weights_average (:709-755), iono_fit
// (:960-1076, or_iono_fit above) and unpeel_model (:897-956).  No precession
// (the tile XYZs are used at every timestep with the given LMSTs, as
// `no_precession`).  Arrays [t][f][bl] JonesF32 / f32 weights; the modeller is
// SkyModellerCpu at the observation phase centre (model_timestep_with, f32
// output).  num_passes and num_loops are the loop counts as used (the
// reference destructures PeelLoopParams::get() with the two swapped,
// mod.rs:1138 vs :218-224: a caller reproducing that passes them swapped).
// The loops over timesteps run in parallel where the reference uses rayon
// (vis_rotate_tfb, unpeel_model); everything else is sequential as there.
// ---------------------------------------------------------------------------
}  // extern "C"

namespace {

// tile (u, v, w) of every tile at hour angle ha, declination dec
void tile_uvws(const double* xyzs, int ntiles, double ha, double dec, double* out /*[tile][3]*/) {
    const double s_ha = std::sin(ha), c_ha = std::cos(ha), s_dec = std::sin(dec), c_dec = std::cos(dec);
    for (int i = 0; i < ntiles; i++) uvw_from_xyz(xyzs + 3 * i, s_ha, c_ha, s_dec, c_dec, out + 3 * i);
}

// vis_rotate_fb: rot = vis * cis(-tau ((w1_to - w2_to) - (w1_from - w2_from)) / lambda)
void rotate_fb(const float* vis, float* out, const double* tuvw_from, const double* tuvw_to, int ntiles, int nf,
               const double* lambdas) {
    const int nbl = ntiles * (ntiles - 1) / 2;
    int i1 = 0, i2 = 0;
    for (int b = 0; b < nbl; b++) {
        i2 += 1;
        if (i2 == ntiles) {
            i1 += 1;
            i2 = i1 + 1;
        }
        const double w_diff = (tuvw_to[3 * i1 + 2] - tuvw_to[3 * i2 + 2]) - (tuvw_from[3 * i1 + 2] - tuvw_from[3 * i2 + 2]);
        const double arg = -TAU * w_diff;
        for (int f = 0; f < nf; f++) {
            const size_t step = (size_t)f * nbl + b;
            to_f32(jmulc(from_f32(vis + 8 * step), cis(arg / lambdas[f])), out + 8 * step);
        }
    }
}

// apply_iono_fb over tile (u, v, w) triples
void iono_fb(const float* vis, float* out, const double* tuvw, int ntiles, int nf, OrIono c, const double* lambdas) {
    const int nbl = ntiles * (ntiles - 1) / 2;
    int i1 = 0, i2 = 0;
    for (int b = 0; b < nbl; b++) {
        i2 += 1;
        if (i2 == ntiles) {
            i1 += 1;
            i2 = i1 + 1;
        }
        const double u = tuvw[3 * i1] - tuvw[3 * i2], v = tuvw[3 * i1 + 1] - tuvw[3 * i2 + 1];
        const double arg = -TAU * (u * c.alpha + v * c.beta);
        for (int f = 0; f < nf; f++) {
            const c64 rot = cscale(cis(arg * lambdas[f]), c.gain);
            const size_t step = (size_t)f * nbl + b;
            to_f32(jmulc(from_f32(vis + 8 * step), rot), out + 8 * step);
        }
    }
}

// vis_average_tfb into one low-res timestep: [nt][nf][nbl] -> [nf / favg][nbl]
// (weights assumed capped at zero; an output with no weight is left as is)
void average_tfb(const float* from, const float* w, float* to, int nt, int nf, int nbl, int favg) {
    const int nlo = (nf + favg - 1) / favg;
    for (int fl = 0; fl < nlo; fl++)
        for (int b = 0; b < nbl; b++) {
            J64 sum = jzero();
            double ws = 0.0;
            for (int t = 0; t < nt; t++)
                for (int f = fl * favg; f < std::min(nf, (fl + 1) * favg); f++) {
                    const size_t step = ((size_t)t * nf + f) * nbl + b;
                    sum = jadd(sum, jscale(from_f32(from + 8 * step), (double)w[step]));
                    ws += (double)w[step];
                }
            if (ws > 0.0) to_f32(jscale(sum, 1.0 / ws), to + 8 * ((size_t)fl * nbl + b));
        }
}

}  // namespace

extern "C" {

int or_peel_cpu(float* resid, const float* weights, int nt, int nf, const double* freqs, const double* xyzs, int ntiles,
                const double* lmsts, double average_lmst, double pc_ra, double pc_dec, int num_sources,
                const OrSky* const* sources, const double* positions /*[src][2]*/, OrIono* consts, int num_passes,
                int num_loops, double convergence, int favg, double lat) {
    const int nbl = ntiles * (ntiles - 1) / 2;
    const int nlo = (nf + favg - 1) / favg;
    const size_t nvis = (size_t)nt * nf * nbl, slab = (size_t)nf * nbl;
    std::vector<double> lam(nf), lam_lo(nlo);
    for (int f = 0; f < nf; f++) lam[f] = VEL_C / freqs[f];
    // low-res wavelengths from the mean frequency of each channel group
    for (int fl = 0; fl < nlo; fl++) {
        double s = 0.0;
        int n = 0;
        for (int f = fl * favg; f < std::min(nf, (fl + 1) * favg); f++, n++) s += freqs[f];
        lam_lo[fl] = VEL_C / (s / n);
    }
    // tile UVWs at the observation phase centre, per timestep
    std::vector<double> tuvw_obs(3 * (size_t)nt * ntiles), tuvw_src(3 * (size_t)nt * ntiles), tuv_lo(2 * (size_t)ntiles);
    for (int t = 0; t < nt; t++) tile_uvws(xyzs, ntiles, lmsts[t] - pc_ra, pc_dec, &tuvw_obs[3 * (size_t)t * ntiles]);
    std::vector<float> resid_src(8 * nvis), model_obs(8 * nvis), model_src(8 * nvis), model_src_iono(8 * nvis);
    std::vector<float> resid_lo(8 * (size_t)nlo * nbl, 0.f), model_lo(8 * (size_t)nlo * nbl, 0.f);
    // weights_average: the sum over the timeblock and each channel group, >= 0
    std::vector<float> w_lo((size_t)nlo * nbl);
    for (int fl = 0; fl < nlo; fl++)
        for (int b = 0; b < nbl; b++) {
            double s = 0.0;
            for (int t = 0; t < nt; t++)
                for (int f = fl * favg; f < std::min(nf, (fl + 1) * favg); f++) s += (double)weights[((size_t)t * nf + f) * nbl + b];
            w_lo[(size_t)fl * nbl + b] = std::max((float)s, 0.f);
        }
    OrBeam nobeam = {};
    for (int pass = 0; pass < num_passes; pass++) {
        for (int s = 0; s < num_sources; s++) {
            const OrIono old = consts[s];
            const double src_ra = positions[2 * s], src_dec = positions[2 * s + 1];
            // high-res model of this source at the observation phase centre
            std::fill(model_obs.begin(), model_obs.end(), 0.f);
            for (int t = 0; t < nt; t++) {
                or_model_timestep(sources[s], xyzs, ntiles, freqs, nf, pc_ra, pc_dec, lmsts[t], lat, &nobeam, 0,
                                  &model_obs[8 * t * slab], 0, nullptr);
                tile_uvws(xyzs, ntiles, lmsts[t] - src_ra, src_dec, &tuvw_src[3 * (size_t)t * ntiles]);
            }
            {
                std::vector<double> tmp(3 * (size_t)ntiles);
                tile_uvws(xyzs, ntiles, average_lmst - src_ra, src_dec, tmp.data());
                for (int i = 0; i < ntiles; i++) tuv_lo[2 * i] = tmp[3 * i], tuv_lo[2 * i + 1] = tmp[3 * i + 1];
            }
            // rotate residual and model to the source phase centre
#pragma omp parallel for schedule(static)
            for (int t = 0; t < nt; t++) {
                rotate_fb(resid + 8 * t * slab, &resid_src[8 * t * slab], &tuvw_obs[3 * (size_t)t * ntiles],
                          &tuvw_src[3 * (size_t)t * ntiles], ntiles, nf, lam.data());
                rotate_fb(&model_obs[8 * t * slab], &model_src[8 * t * slab], &tuvw_obs[3 * (size_t)t * ntiles],
                          &tuvw_src[3 * (size_t)t * ntiles], ntiles, nf, lam.data());
            }
            for (int t = 0; t < nt; t++)
                iono_fb(&model_src[8 * t * slab], &model_src_iono[8 * t * slab], &tuvw_src[3 * (size_t)t * ntiles], ntiles,
                        nf, consts[s], lam.data());
            for (size_t k = 0; k < 8 * nvis; k++) resid_src[k] += model_src_iono[k];
            average_tfb(resid_src.data(), weights, resid_lo.data(), nt, nf, nbl, favg);
            for (int it = 0; it < num_loops; it++) {
                for (int t = 0; t < nt; t++)
                    iono_fb(&model_src[8 * t * slab], &model_src_iono[8 * t * slab], &tuvw_src[3 * (size_t)t * ntiles],
                            ntiles, nf, consts[s], lam.data());
                average_tfb(model_src_iono.data(), weights, model_lo.data(), nt, nf, nbl, favg);
                double fit[4];
                or_iono_fit(resid_lo.data(), w_lo.data(), model_lo.data(), lam_lo.data(), tuv_lo.data(), 1, nlo, ntiles,
                            fit);
                const double da = fit[0], db = fit[1], dg = fit[2] / fit[3];
                consts[s].alpha += convergence * da;
                consts[s].beta += convergence * db;
                consts[s].gain *= 1. + convergence * (dg - 1.);
                if (std::sqrt(std::pow(da, 2.) + std::pow(db, 2.) + std::pow(dg - 1., 2.)) < 1e-8) break;
            }
            // unpeel_model: the model at the observation phase centre with the
            // source's tile UVs (as the reference does)
            const OrIono c = consts[s];
#pragma omp parallel for schedule(static)
            for (int t = 0; t < nt; t++) {
                const double* tu = &tuvw_src[3 * (size_t)t * ntiles];
                int i1 = 0, i2 = 0;
                for (int b = 0; b < nbl; b++) {
                    i2 += 1;
                    if (i2 == ntiles) {
                        i1 += 1;
                        i2 = i1 + 1;
                    }
                    const double u = tu[3 * i1] - tu[3 * i2], v = tu[3 * i1 + 1] - tu[3 * i2 + 1];
                    const double arg = -TAU * (u * c.alpha + v * c.beta);
                    const double old_arg = -TAU * (u * old.alpha + v * old.beta);
                    for (int f = 0; f < nf; f++) {
                        const size_t step = (size_t)t * slab + (size_t)f * nbl + b;
                        J64 j = from_f32(resid + 8 * step);
                        const J64 m = from_f32(&model_obs[8 * step]);
                        j = jadd(j, jmulc(m, cscale(cis(old_arg * lam[f]), old.gain)));
                        j = jsub(j, jmulc(m, cscale(cis(arg * lam[f]), c.gain)));
                        to_f32(j, resid + 8 * step);
                    }
                }
            }
        }
    }
    return 0;
}

}  // extern "C"
