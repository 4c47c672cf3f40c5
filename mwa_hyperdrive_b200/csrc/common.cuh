// Shared device helpers for libhdc (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/hdc.h"

namespace hdc {

constexpr double VEL_C = 299792458.0;
constexpr double TAU = 6.283185307179586;
constexpr double INV_TAU = 0.15915494309189535;
constexpr double FRAC_PI_2 = 1.5707963267948966;
constexpr double LN_2 = 0.6931471805599453;
constexpr double SQRT_FRAC_PI_SQ_2_LN_2 = 2.6682231283184983;
constexpr double SBF_C = 5000.0;
constexpr int SBF_L = 10001;
constexpr int SBF_N = 101;
constexpr double SBF_DX = 0.01;
constexpr double POWER_LAW_FD_REF_FREQ = 150e6;
// Gaussian envelope exponent constant -(pi/2)^2 / ln 2 and the shapelet
// basis scale sqrt(pi^2 / (2 ln 2)) / SBF_DX (model/cpu.rs:36-37).
constexpr double GAUSSIAN_EXP_CONST = -(FRAC_PI_2 * FRAC_PI_2) / LN_2;
constexpr double SHAPELET_CONST = SQRT_FRAC_PI_SQ_2_LN_2 / SBF_DX;

// Error flags written by kernels (bit mask in a device word).
constexpr int KERR_TIMEOUT = 1;
constexpr int KERR_INDEX = 2;

struct cplx {
    double re, im;
};
__host__ __device__ __forceinline__ cplx operator+(cplx a, cplx b) { return {a.re + b.re, a.im + b.im}; }
__host__ __device__ __forceinline__ cplx operator-(cplx a, cplx b) { return {a.re - b.re, a.im - b.im}; }
__host__ __device__ __forceinline__ cplx operator*(cplx a, cplx b) {
    return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
__host__ __device__ __forceinline__ cplx operator*(cplx a, double s) { return {a.re * s, a.im * s}; }
__host__ __device__ __forceinline__ cplx conj(cplx a) { return {a.re, -a.im}; }

// 2x2 complex matrix [a b; c d] (XX XY YX YY).
struct J2 {
    cplx a, b, c, d;
};
__host__ __device__ __forceinline__ J2 jzero() { return J2{{0, 0}, {0, 0}, {0, 0}, {0, 0}}; }
__host__ __device__ __forceinline__ J2 operator+(const J2& x, const J2& y) {
    return J2{x.a + y.a, x.b + y.b, x.c + y.c, x.d + y.d};
}
__host__ __device__ __forceinline__ J2 operator-(const J2& x, const J2& y) {
    return J2{x.a - y.a, x.b - y.b, x.c - y.c, x.d - y.d};
}
__host__ __device__ __forceinline__ J2 operator*(const J2& x, const J2& y) {
    return J2{x.a * y.a + x.b * y.c, x.a * y.b + x.b * y.d, x.c * y.a + x.d * y.c, x.c * y.b + x.d * y.d};
}
__host__ __device__ __forceinline__ J2 operator*(const J2& x, cplx s) { return J2{x.a * s, x.b * s, x.c * s, x.d * s}; }
__host__ __device__ __forceinline__ J2 operator*(const J2& x, double s) { return J2{x.a * s, x.b * s, x.c * s, x.d * s}; }
// conjugate transpose
__host__ __device__ __forceinline__ J2 herm(const J2& x) { return J2{conj(x.a), conj(x.c), conj(x.b), conj(x.d)}; }

__host__ __device__ __forceinline__ J2 load_j(const JonesF64& j) {
    return J2{{j.j00_re, j.j00_im}, {j.j01_re, j.j01_im}, {j.j10_re, j.j10_im}, {j.j11_re, j.j11_im}};
}
__host__ __device__ __forceinline__ JonesF64 store_j(const J2& x) {
    return JonesF64{x.a.re, x.a.im, x.b.re, x.b.im, x.c.re, x.c.im, x.d.re, x.d.im};
}
__host__ __device__ __forceinline__ J2 load_j32(const JonesF32& j) {
    return J2{{j.j00_re, j.j00_im}, {j.j01_re, j.j01_im}, {j.j10_re, j.j10_im}, {j.j11_re, j.j11_im}};
}

// Vectorised 64-byte Jones load through the read-only path.
__device__ __forceinline__ J2 ldg_j(const JonesF64* p) {
    const double2* q = reinterpret_cast<const double2*>(p);
    double2 a = __ldg(q), b = __ldg(q + 1), c = __ldg(q + 2), d = __ldg(q + 3);
    return J2{{a.x, a.y}, {b.x, b.y}, {c.x, c.y}, {d.x, d.y}};
}

// Upper-triangle baseline index -> (tile1, tile2), tile1 < tile2, with an
// integer fix-up after the closed-form estimate (exact for any n).
__host__ __device__ __forceinline__ void baseline_to_tiles(int bl, int n, int& t1, int& t2) {
    double b = (double)bl;
    double nn = 2.0 * n - 1.0;
    int p = (int)floor((nn - sqrt(nn * nn - 8.0 * b)) * 0.5);
    if (p < 0) p = 0;
    // start(p) = p (2n - p - 1) / 2
    while (p > 0 && (long long)p * (2 * n - p - 1) / 2 > bl) p--;
    while ((long long)(p + 1) * (2 * n - p - 2) / 2 <= bl) p++;
    t1 = p;
    t2 = bl - (int)((long long)p * (2 * n - p - 1) / 2) + p + 1;
}

__host__ __device__ __forceinline__ int baseline_index(int t1, int t2, int n) {
    return (int)((long long)t1 * (2 * n - t1 - 1) / 2) + (t2 - t1 - 1);
}

// ---------------------------------------------------------------------------
// TMA (bulk async copy) + mbarrier helpers, with waits bounded by the global
// timer so that no kernel can spin forever.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint64_t global_timer_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_barrier_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

// 1-D bulk copy global -> shared (TMA engine).  dst/src 16-byte aligned,
// bytes a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

// Prefetch bytes of global memory into L2 (no completion to wait for).
// src 16-byte aligned, bytes a multiple of 16.
__device__ __forceinline__ void prefetch_l2(const void* src, uint32_t bytes) {
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Wait for phase `parity` of `bar`; gives up after `limit_ns` of global
// time, records KERR_TIMEOUT in *err and returns false.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, int* err,
                                                  uint64_t limit_ns = 2000000000ull) {
    if (mbar_try_wait(bar, parity)) return true;
    uint64_t t0 = global_timer_ns();
    while (!mbar_try_wait(bar, parity)) {
        if (global_timer_ns() - t0 > limit_ns) {
            if (err) atomicOr(err, KERR_TIMEOUT);
            return false;
        }
    }
    return true;
}

// As mbar_wait_bounded, but each try suspends the thread in hardware until
// the phase completes or about a millisecond passes (no polling traffic on
// the shared-memory pipe while it waits).
__device__ __forceinline__ bool mbar_wait_sleep(uint64_t* bar, uint32_t parity, int* err,
                                                uint64_t limit_ns = 2000000000ull) {
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = global_timer_ns();
    for (;;) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(ok)
            : "r"(smem_u32(bar)), "r"(parity), "r"(1000000u)
            : "memory");
        if (ok) return true;
        if (global_timer_ns() - t0 > limit_ns) {
            if (err) atomicOr(err, KERR_TIMEOUT);
            return false;
        }
    }
}

// A shared-memory word written with release and read with acquire (CTA
// scope): a slot tag that says which sequence number a ring slot holds.
__device__ __forceinline__ uint32_t ld_acquire_smem(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.acquire.cta.shared::cta.u32 %0, [%1];" : "=r"(v) : "r"(smem_u32(p)) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_smem(uint32_t* p, uint32_t v) {
    asm volatile("st.release.cta.shared::cta.u32 [%0], %1;" ::"r"(smem_u32(p)), "r"(v) : "memory");
}

// Wait (bounded, as mbar_wait_bounded) until *tag == want.
__device__ __forceinline__ bool tag_wait_bounded(const uint32_t* tag, uint32_t want, int* err,
                                                 uint64_t limit_ns = 2000000000ull) {
    if (ld_acquire_smem(tag) == want) return true;
    const uint64_t t0 = global_timer_ns();
    while (ld_acquire_smem(tag) != want) {
        if (global_timer_ns() - t0 > limit_ns) {
            if (err) atomicOr(err, KERR_TIMEOUT);
            return false;
        }
        __nanosleep(32);
    }
    return true;
}

// After a bounded wait of a two-stage bulk-copy pipeline ran out at chunk k,
// chunks [k, issued) may still be in flight: the issuing thread waits for
// each of them (bounded again) so that no copy lands in the shared memory of
// a CTA that has exited.
__device__ __forceinline__ void drain_two_stage(uint64_t* bar, int k, int issued) {
    for (int j = k; j < issued; j++) mbar_wait_bounded(&bar[j & 1], (j >> 1) & 1, nullptr);
}

// ERFA hd2ae (marlu HADec::to_azel).
__device__ __forceinline__ void hadec_to_azel(double ha, double dec, double lat, double& az, double& el) {
    double s_ha, c_ha, s_dec, c_dec, s_lat, c_lat;
    sincos(ha, &s_ha, &c_ha);
    sincos(dec, &s_dec, &c_dec);
    sincos(lat, &s_lat, &c_lat);
    const double x = -s_ha * c_dec;
    const double y = -c_ha * c_dec * s_lat + s_dec * c_lat;
    const double z = c_ha * c_dec * c_lat + s_dec * s_lat;
    const double r = hypot(x, y);
    const double a = (r == 0.0) ? 0.0 : atan2(x, y);
    az = (a < 0.0) ? a + TAU : a;
    el = atan2(z, r);
}

// FP64 phasor exp(2 pi i t) for a phase in turns: exact range reduction to
// r = t - rint(t) in [-1/2, 1/2], then sincospi(2 r).
__device__ __forceinline__ cplx phasor_turns(double t) {
    double r = t - rint(t);
    double s, c;
    sincospi(2.0 * r, &s, &c);
    return {c, s};
}

// FP32 phasor for the tensor-core predict and the chosen form's direct
// kernels: sin and cos of 2 pi z for z in quarter-turns.  q = rint(z) and
// r = z - q are exact in FP64; sin and cos of (pi/2) r come from
// least-squares polynomials in r^2 on |r| <= 1/2 (fitted by
// mwa_hyperdrive_b200/phasor_poly.py, < 0.75 float32 ulp); the quadrant
// q mod 4 swaps and signs them.
constexpr double QMAGIC = 6755399441055744.0;  // 1.5 * 2^52: adding it rounds to an integer held in the low word
constexpr float PS0 = 1.570796371e+00f, PS1 = -6.459634900e-01f, PS2 = 7.968021929e-02f,
                PS3 = -4.602163099e-03f;
constexpr float PC0 = 1.000000000e+00f, PC1 = -1.233700514e+00f, PC2 = 2.536692023e-01f,
                PC3 = -2.086007036e-02f, PC4 = 9.036298725e-04f;

__device__ __forceinline__ void phasor_quarter_f32(double z, float& sn, float& cs) {
    const double zq = __dadd_rn(z, QMAGIC);
    const int q = __double2loint(zq);
    const float r = (float)__dsub_rn(z, __dsub_rn(zq, QMAGIC));
    const float r2 = r * r;
    const float ps = fmaf(fmaf(fmaf(PS3, r2, PS2), r2, PS1), r2, PS0) * r;
    const float pc = fmaf(fmaf(fmaf(fmaf(PC4, r2, PC3), r2, PC2), r2, PC1), r2, PC0);
    // angle = (pi/2)(q + r): odd q swaps sin and cos; sin takes the sign of
    // bit 1 of q, cos that of bit 1 of q + 1 (moved to bit 31 by << 30)
    const bool odd = q & 1;
    const float a = odd ? pc : ps, b = odd ? ps : pc;
    const uint32_t qs = (uint32_t)q << 30;
    sn = __uint_as_float(__float_as_uint(a) ^ (qs & 0x80000000u));
    cs = __uint_as_float(__float_as_uint(b) ^ ((qs + 0x40000000u) & 0x80000000u));
}

}  // namespace hdc

// ---------------------------------------------------------------------------
// Host-side error plumbing
// ---------------------------------------------------------------------------
namespace hdc {
void set_error(const char* fmt, ...);
const char* cuda_msg(cudaError_t e);
// Per-device scratch (grows on demand; used by the drop-in entry points that
// have no workspace argument).  Returns NULL on allocation failure.
void* device_scratch(size_t bytes);
// Stream-ordered allocation from the library's own pool on the current device
// (freed blocks stay mapped for reuse); release with cudaFreeAsync.
cudaError_t pool_malloc_async(void** p, size_t bytes, cudaStream_t s);
// Device word for kernel error flags (per device, zero-initialised).
int* device_error_word();
// Read and clear the device error word (synchronises the stream).
int take_device_error(cudaStream_t s);
// The drop-in layer's own kernel error word (per device), apart from the
// native layer's so that neither sees the other's errors.
int* dropin_error_word();
// Read error word w after the work queued before it on the legacy default
// stream (a synchronous copy), clear it if set and return the static message
// for its bits (NULL when clear); `who` prefixes hdc_last_error().
const char* take_word_sync(int* w, const char* who);
// Shapelet basis table on the current device (SBF_N x SBF_L doubles).
const double* device_shapelet_basis();
const float* device_shapelet_basis_f32();
// FP32 (value, next - value) pairs of the table's orders 0 .. SDN_TABLE - 1,
// position-major: [SBF_L][SDN_TABLE / 2] float4 (one record per position).
constexpr int SDN_TABLE = 6;
const float4* device_shapelet_basis_pairs();
void host_shapelet_basis(double* out);
// Count of kernel launches made by libhdc (diagnostics).
void count_launches(int n);
}  // namespace hdc

#define HDC_CUDA_RET_STR(call)                                     \
    do {                                                           \
        cudaError_t e_ = (call);                                   \
        if (e_ != cudaSuccess) {                                   \
            hdc::set_error("%s: %s", #call, cudaGetErrorString(e_)); \
            return cudaGetErrorString(e_);                         \
        }                                                          \
    } while (0)

#define HDC_CUDA_RET_INT(call)                                     \
    do {                                                           \
        cudaError_t e_ = (call);                                   \
        if (e_ != cudaSuccess) {                                   \
            hdc::set_error("%s: %s", #call, cudaGetErrorString(e_)); \
            return HDC_ERR_CUDA;                                   \
        }                                                          \
    } while (0)
