// Calibration solutions completed on the device (into_cal_sols,
// di_calibrate/mod.rs:89-176): the solver's model->data gains for the
// unflagged tiles and chanblocks, [timeblock][unflagged tile][unflagged
// chanblock], become data->model solutions for every tile and chanblock,
// [timeblock][tile][chanblock]: each Jones matrix inverted (only XX or only
// YY inverted as a complex number for single-polarisation data, the other
// entries zero), NaN wherever a tile or chanblock is flagged.
//
// One thread per output Jones matrix; the flagged tile and chanblock lists
// travel in the launch's parameters.  The inversion is marlu's Jones::inv
// (inv_det = 1 / (ad - bc); [d, -b, -c, a] x inv_det, complex division as
// num_complex's (a conj(b)) / |b|^2) and Complex::inv (conj / |z|^2), with
// no FMA contraction, as the reference computes it in Rust.

#include <cmath>
#include <vector>

#include "common.cuh"
#include "flagtable.cuh"

namespace hdc {
namespace sols {

constexpr int TILE_CAP = 1024;
constexpr int CHAN_CAP = 8000;
constexpr int THREADS = 256;

struct Flags {
    FlagTable<TILE_CAP> tiles;
    FlagTable<CHAN_CAP> chans;
};  // 18 KB of launch parameters (the limit is 32764 bytes)

struct C {
    double re, im;
};
__device__ __forceinline__ C cmul(C a, C b) {
    return {__dsub_rn(__dmul_rn(a.re, b.re), __dmul_rn(a.im, b.im)),
            __dadd_rn(__dmul_rn(a.re, b.im), __dmul_rn(a.im, b.re))};
}
__device__ __forceinline__ C csub(C a, C b) { return {__dsub_rn(a.re, b.re), __dsub_rn(a.im, b.im)}; }
__device__ __forceinline__ double norm_sqr(C b) { return __dadd_rn(__dmul_rn(b.re, b.re), __dmul_rn(b.im, b.im)); }
// (a conj(b)) / |b|^2
__device__ __forceinline__ C cdiv(C a, C b) {
    const double n = norm_sqr(b);
    return {__ddiv_rn(__dadd_rn(__dmul_rn(a.re, b.re), __dmul_rn(a.im, b.im)), n),
            __ddiv_rn(__dsub_rn(__dmul_rn(a.im, b.re), __dmul_rn(a.re, b.im)), n)};
}
// Complex::inv: conj(z) / |z|^2
__device__ __forceinline__ C cinv(C z) {
    const double n = norm_sqr(z);
    return {__ddiv_rn(z.re, n), __ddiv_rn(-z.im, n)};
}

__global__ void __launch_bounds__(THREADS) into_sols_kernel(const JonesF64* __restrict__ in, int ntb, int nut,
                                                            int nuc, int ntt, int ntc, int pols,
                                                            const __grid_constant__ Flags fl,
                                                            JonesF64* __restrict__ out) {
    const size_t g = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= (size_t)ntb * ntt * ntc) return;
    const int c = (int)(g % ntc);
    const int t = (int)((g / ntc) % ntt);
    const int tb = (int)(g / ((size_t)ntc * ntt));
    const int tl = flag_count_le(fl.tiles, t), cl = flag_count_le(fl.chans, c);
    const bool flagged = (tl > 0 && fl.tiles.v[tl - 1] == t) || (cl > 0 && fl.chans.v[cl - 1] == c);
    double2* o = reinterpret_cast<double2*>(out + g);
    if (flagged) {
        const double2 nan2 = make_double2(__longlong_as_double(0x7ff8000000000000LL),
                                          __longlong_as_double(0x7ff8000000000000LL));
        o[0] = nan2, o[1] = nan2, o[2] = nan2, o[3] = nan2;
        return;
    }
    const double2* p = reinterpret_cast<const double2*>(in + ((size_t)tb * nut + (t - tl)) * nuc + (c - cl));
    const double2 q0 = p[0], q1 = p[1], q2 = p[2], q3 = p[3];
    const C a{q0.x, q0.y}, b{q1.x, q1.y}, cc{q2.x, q2.y}, d{q3.x, q3.y};
    C r0{0, 0}, r1{0, 0}, r2{0, 0}, r3{0, 0};
    if (pols == 1) {  // XX only
        r0 = cinv(a);
    } else if (pols == 2) {  // YY only
        r3 = cinv(d);
    } else {
        const C inv_det = cdiv(C{1.0, 0.0}, csub(cmul(a, d), cmul(b, cc)));
        const C neg{-inv_det.re, -inv_det.im};
        r0 = cmul(inv_det, d), r1 = cmul(neg, b), r2 = cmul(neg, cc), r3 = cmul(inv_det, a);
    }
    o[0] = make_double2(r0.re, r0.im), o[1] = make_double2(r1.re, r1.im);
    o[2] = make_double2(r2.re, r2.im), o[3] = make_double2(r3.re, r3.im);
}

}  // namespace sols
}  // namespace hdc

using namespace hdc;

extern "C" int hdc_into_cal_sols(const JonesF64* d_di_jones, int num_timeblocks, int num_unflagged_tiles,
                                 int num_unflagged_chanblocks, const int* h_flagged_tiles, int num_flagged_tiles,
                                 const int* h_flagged_chanblocks, int num_flagged_chanblocks, int pols,
                                 JonesF64* d_out, hdcStream_t stream) {
    if (!d_di_jones || !d_out || num_timeblocks < 1 || num_unflagged_tiles < 0 || num_unflagged_chanblocks < 0 ||
        num_flagged_tiles < 0 || num_flagged_chanblocks < 0 || (num_flagged_tiles > 0 && !h_flagged_tiles) ||
        (num_flagged_chanblocks > 0 && !h_flagged_chanblocks) || pols < 0 || pols > 4) {
        set_error("hdc_into_cal_sols: invalid arguments");
        return HDC_ERR_ARG;
    }
    const long long ntt = (long long)num_unflagged_tiles + num_flagged_tiles;
    const long long ntc = (long long)num_unflagged_chanblocks + num_flagged_chanblocks;
    if (num_flagged_tiles > sols::TILE_CAP || num_flagged_chanblocks > sols::CHAN_CAP || ntt > 65536 ||
        ntc > 65536) {
        set_error("hdc_into_cal_sols: at most %d flagged tiles and %d flagged chanblocks, each of at most 65536",
                  sols::TILE_CAP, sols::CHAN_CAP);
        return HDC_ERR_ARG;
    }
    bool ok_t, ok_c;
    const std::vector<int> ft = sorted_flags(h_flagged_tiles, num_flagged_tiles, (int)ntt, &ok_t);
    const std::vector<int> fc = sorted_flags(h_flagged_chanblocks, num_flagged_chanblocks, (int)ntc, &ok_c);
    if (!ok_t || !ok_c) {
        set_error("hdc_into_cal_sols: a flagged %s index is out of range or repeated", ok_t ? "chanblock" : "tile");
        return HDC_ERR_ARG;
    }
    const size_t n = (size_t)num_timeblocks * ntt * ntc;
    if (n == 0) return HDC_OK;
    static thread_local sols::Flags fl;  // 18 KB: off the stack
    fl.tiles.n = num_flagged_tiles;
    for (int k = 0; k < num_flagged_tiles; k++) fl.tiles.v[k] = (unsigned short)ft[k];
    fl.chans.n = num_flagged_chanblocks;
    for (int k = 0; k < num_flagged_chanblocks; k++) fl.chans.v[k] = (unsigned short)fc[k];
    sols::into_sols_kernel<<<(unsigned)((n + sols::THREADS - 1) / sols::THREADS), sols::THREADS, 0,
                             (cudaStream_t)stream>>>(d_di_jones, num_timeblocks, num_unflagged_tiles,
                                                     num_unflagged_chanblocks, (int)ntt, (int)ntc, pols, fl, d_out);
    count_launches(1);
    HDC_CUDA_RET_INT(cudaGetLastError());
    return HDC_OK;
}
