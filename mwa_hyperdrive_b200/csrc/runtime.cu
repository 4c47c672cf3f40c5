// Runtime support for libhdc: error messages, per-device scratch and error
// words, the shapelet basis table, device information.

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <atomic>
#include <mutex>
#include <vector>

#include "predict.cuh"

namespace hdc {

static thread_local char g_err[1024] = "";

void set_error(const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}

const char* cuda_msg(cudaError_t e) { return cudaGetErrorString(e); }

static std::atomic<long long> g_launches{0};
void count_launches(int n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

// 8 independent FMA chains per thread, `iters` rounds; the result is stored
// only if it equals a value it never takes, so the work is not optimised away.
template <class T>
__global__ void fma_probe_kernel(T seed, int iters, T* sink) {
    T a[8];
#pragma unroll
    for (int k = 0; k < 8; k++) a[k] = seed + (T)(threadIdx.x * 1e-6) + (T)k;
    const T m = (T)0.999999, c = (T)1e-7;
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int k = 0; k < 8; k++) a[k] = fma(a[k], m, c);
    }
    T s = 0;
#pragma unroll
    for (int k = 0; k < 8; k++) s += a[k];
    if (s == (T)-1.2345) *sink = s;
}

namespace {
constexpr int MAX_DEV = 64;
std::mutex g_mu;
void* g_scratch[MAX_DEV] = {};
size_t g_scratch_size[MAX_DEV] = {};
int* g_errword[MAX_DEV] = {};
int* g_dropin_err[MAX_DEV] = {};
double* g_sbf[MAX_DEV] = {};
float* g_sbf32[MAX_DEV] = {};
float4* g_sbfp[MAX_DEV] = {};
cudaMemPool_t g_pool[MAX_DEV] = {};

int cur_dev() {
    int d = 0;
    if (cudaGetDevice(&d) != cudaSuccess) return -1;
    return (d >= 0 && d < MAX_DEV) ? d : -1;
}
}  // namespace

cudaError_t pool_malloc_async(void** p, size_t bytes, cudaStream_t s) {
    cudaMemPool_t pool = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        const int d = cur_dev();
        if (d < 0) return cudaErrorInvalidDevice;
        if (!g_pool[d]) {
            cudaMemPoolProps props = {};
            props.allocType = cudaMemAllocationTypePinned;
            props.location.type = cudaMemLocationTypeDevice;
            props.location.id = d;
            cudaError_t e = cudaMemPoolCreate(&g_pool[d], &props);
            if (e != cudaSuccess) return e;
            // keep freed blocks mapped: the next call reuses them without a
            // new physical mapping (the default pool returns them at every
            // synchronisation)
            uint64_t keep = UINT64_MAX;
            e = cudaMemPoolSetAttribute(g_pool[d], cudaMemPoolAttrReleaseThreshold, &keep);
            if (e != cudaSuccess) return e;
        }
        pool = g_pool[d];
    }
    return cudaMallocFromPoolAsync(p, bytes, pool, s);
}

void* device_scratch(size_t bytes) {
    std::lock_guard<std::mutex> lk(g_mu);
    int d = cur_dev();
    if (d < 0) return nullptr;
    if (bytes == 0) bytes = 256;
    if (g_scratch_size[d] < bytes) {
        if (g_scratch[d]) {
            // Kernels queued on any stream may still read the old buffer.
            cudaDeviceSynchronize();
            cudaFree(g_scratch[d]);
            g_scratch[d] = nullptr;
            g_scratch_size[d] = 0;
        }
        size_t want = bytes + bytes / 4;
        if (cudaMalloc(&g_scratch[d], want) != cudaSuccess) {
            cudaGetLastError();
            set_error("device scratch allocation of %zu bytes failed", want);
            return nullptr;
        }
        g_scratch_size[d] = want;
    }
    return g_scratch[d];
}

int* device_error_word() {
    std::lock_guard<std::mutex> lk(g_mu);
    int d = cur_dev();
    if (d < 0) return nullptr;
    if (!g_errword[d]) {
        if (cudaMalloc(&g_errword[d], sizeof(int)) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        cudaMemset(g_errword[d], 0, sizeof(int));
    }
    return g_errword[d];
}

int* dropin_error_word() {
    std::lock_guard<std::mutex> lk(g_mu);
    int d = cur_dev();
    if (d < 0) return nullptr;
    if (!g_dropin_err[d]) {
        if (cudaMalloc(&g_dropin_err[d], sizeof(int)) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        cudaMemset(g_dropin_err[d], 0, sizeof(int));
    }
    return g_dropin_err[d];
}

const char* take_word_sync(int* w, const char* who) {
    int h = 0;
    cudaError_t e = cudaMemcpy(&h, w, sizeof(int), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) {
        set_error("%s: %s", who, cudaGetErrorString(e));
        return cudaGetErrorString(e);
    }
    if (!h) return NULL;
    cudaMemset(w, 0, sizeof(int));
    const char* msg = kernel_error_string(h);
    set_error("%s: %s", who, msg);
    return msg;
}

int take_device_error(cudaStream_t s) {
    int* w = device_error_word();
    if (!w) return 0;
    int h = 0;
    if (cudaMemcpyAsync(&h, w, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess) return 0;
    cudaStreamSynchronize(s);
    if (h) cudaMemsetAsync(w, 0, sizeof(int), s);
    return h;
}

// Hermite-Gaussian basis B_n(x) = exp(-x^2/2) H_n(x) / sqrt(2^n n!), sampled
// on x = linspace(-50, 50, SBF_L), n = 0..SBF_N-1 -- the table mwa_hyperdrive
// embeds (model/shapelets.rs:11-37, generated by make_shapelet_basis_values.py).
void host_shapelet_basis(double* out) {
    const double step = 100.0 / (SBF_L - 1);
    for (int ix = 0; ix < SBF_L; ix++) {
        const double x = (ix == SBF_L - 1) ? 50.0 : -50.0 + ix * step;
        const double g = std::exp(-0.5 * (x * x));
        double hm1 = 1.0, h = 2.0 * x;
        for (int n = 0; n < SBF_N; n++) {
            double hn;
            if (n == 0) {
                hn = 1.0;
            } else if (n == 1) {
                hn = 2.0 * x;
            } else {
                const double hp = 2.0 * x * h - 2.0 * (n - 1) * hm1;
                hm1 = h;
                h = hp;
                hn = hp;
            }
            const double norm = 1.0 / std::sqrt(std::pow(2.0, n) * std::tgamma(n + 1.0));
            out[(size_t)n * SBF_L + ix] = g * norm * hn;
        }
    }
}

const double* device_shapelet_basis() {
    std::lock_guard<std::mutex> lk(g_mu);
    int d = cur_dev();
    if (d < 0) return nullptr;
    if (!g_sbf[d]) {
        std::vector<double> h((size_t)SBF_N * SBF_L);
        host_shapelet_basis(h.data());
        if (cudaMalloc(&g_sbf[d], h.size() * sizeof(double)) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        cudaMemcpy(g_sbf[d], h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice);
    }
    return g_sbf[d];
}

const float* device_shapelet_basis_f32() {
    std::lock_guard<std::mutex> lk(g_mu);
    int d = cur_dev();
    if (d < 0) return nullptr;
    if (!g_sbf32[d]) {
        std::vector<double> h((size_t)SBF_N * SBF_L);
        host_shapelet_basis(h.data());
        std::vector<float> hf(h.begin(), h.end());
        if (cudaMalloc(&g_sbf32[d], hf.size() * sizeof(float)) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        cudaMemcpy(g_sbf32[d], hf.data(), hf.size() * sizeof(float), cudaMemcpyHostToDevice);
    }
    return g_sbf32[d];
}

const float4* device_shapelet_basis_pairs() {
    std::lock_guard<std::mutex> lk(g_mu);
    int d = cur_dev();
    if (d < 0) return nullptr;
    if (!g_sbfp[d]) {
        std::vector<double> h((size_t)SBF_N * SBF_L);
        host_shapelet_basis(h.data());
        // position-major: the SDN orders' (value, next - value) pairs at one
        // position are one 48-byte record (three float4)
        std::vector<float> hp((size_t)SBF_L * 2 * SDN_TABLE);
        for (int i = 0; i < SBF_L; i++)
            for (int n = 0; n < SDN_TABLE; n++) {
                const size_t k = (size_t)n * SBF_L + i;
                const double nxt = i + 1 < SBF_L ? h[k + 1] : h[k];
                hp[((size_t)i * SDN_TABLE + n) * 2] = (float)h[k];
                hp[((size_t)i * SDN_TABLE + n) * 2 + 1] = (float)(nxt - h[k]);
            }
        if (cudaMalloc(&g_sbfp[d], hp.size() * sizeof(float)) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        cudaMemcpy(g_sbfp[d], hp.data(), hp.size() * sizeof(float), cudaMemcpyHostToDevice);
    }
    return g_sbfp[d];
}

}  // namespace hdc

extern "C" const char* hdc_last_error(void) { return hdc::g_err; }

extern "C" long long hdc_kernel_launches(void) { return hdc::g_launches.load(); }

namespace {
// FMA rate of the current device in GFLOP/s (an FMA counts 2), one timed
// launch of 4 CTAs of 512 threads per SM after a warm-up.
template <class T>
int probe_fma(double* out, const char* what) {
    int d = 0, sms = 0;
    cudaGetDevice(&d);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, d);
    T* sink = nullptr;
    HDC_CUDA_RET_INT(cudaMalloc(&sink, sizeof(T)));
    const int threads = 512, blocks = sms * 4, iters = sizeof(T) == 8 ? 4096 : 16384;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    hdc::fma_probe_kernel<T><<<blocks, threads>>>((T)1, 64, sink);  // warm-up
    cudaEventRecord(e0);
    hdc::fma_probe_kernel<T><<<blocks, threads>>>((T)1, iters, sink);
    cudaEventRecord(e1);
    cudaError_t e = cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(sink);
    hdc::count_launches(2);
    if (e != cudaSuccess) {
        hdc::set_error("%s probe: %s", what, cudaGetErrorString(e));
        return HDC_ERR_CUDA;
    }
    *out = 2.0 * 8.0 * iters * (double)threads * blocks / (ms * 1e-3) / 1e9;
    return HDC_OK;
}
}  // namespace

extern "C" int hdc_probe_fp64_gflops(double* out) { return probe_fma<double>(out, "fp64"); }

extern "C" int hdc_probe_fp32_gflops(double* out) { return probe_fma<float>(out, "fp32"); }

extern "C" int hdc_device_info(char* buf, int buf_len) {
    int d = 0;
    cudaDeviceProp prop;
    if (cudaGetDevice(&d) != cudaSuccess || cudaGetDeviceProperties(&prop, d) != cudaSuccess) {
        cudaGetLastError();
        hdc::set_error("no CUDA device");
        return HDC_ERR_CUDA;
    }
    int rt = 0, drv = 0;
    cudaRuntimeGetVersion(&rt);
    cudaDriverGetVersion(&drv);
    snprintf(buf, (size_t)buf_len, "%s (sm_%d%d, %d SMs, %.1f GiB), CUDA runtime %d.%d, driver %d.%d, libhdc sm_100a",
             prop.name, prop.major, prop.minor, prop.multiProcessorCount,
             (double)prop.totalGlobalMem / (1024.0 * 1024.0 * 1024.0), rt / 1000, (rt % 1000) / 10, drv / 1000,
             (drv % 1000) / 10);
    return HDC_OK;
}

// The reference's device query (gpu/utils.h:28, bound by gpu/utils_bindings.rs
// and called from gpu/utils.rs:35-60 for the solutions' MODELLER string): make
// `device` current and report its name (NUL-terminated, at most 255
// characters), compute capability, global memory [bytes] and the CUDA driver
// and runtime versions as integers (1000 * major + 10 * minor).  NULL on
// success, else the CUDA error string.
extern "C" const char* get_gpu_device_info(int device, char name[256], int* device_major, int* device_minor,
                                           size_t* total_global_mem, int* driver_version, int* runtime_version) {
    cudaError_t e = cudaSetDevice(device);
    cudaDeviceProp prop;
    if (e == cudaSuccess) e = cudaGetDeviceProperties(&prop, device);
    if (e == cudaSuccess) e = cudaDriverGetVersion(driver_version);
    if (e == cudaSuccess) e = cudaRuntimeGetVersion(runtime_version);
    if (e != cudaSuccess) {
        hdc::set_error("get_gpu_device_info: %s", cudaGetErrorString(e));
        return cudaGetErrorString(e);
    }
    snprintf(name, 256, "%s", prop.name);
    *device_major = prop.major;
    *device_minor = prop.minor;
    *total_global_mem = prop.totalGlobalMem;
    return NULL;
}

// Host copy of the shapelet basis table (for tests and for callers that
// upload it themselves as Addresses::d_shapelet_basis_values).
extern "C" int hdc_shapelet_basis(double* h_out) {
    hdc::host_shapelet_basis(h_out);
    return HDC_OK;
}
