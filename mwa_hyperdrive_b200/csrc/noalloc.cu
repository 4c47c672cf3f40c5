// model_points_noalloc: the point-source predict of model_points for callers
// that cannot allocate device memory.
//
// Some hosts own every byte of device memory themselves -- a framework that
// reserves the GPU's memory up front for its own pool, or a streaming
// pipeline that budgets memory once at start-up and must not call cudaMalloc
// in its processing loop, where the call's implicit device-wide
// synchronisation would stall the other work on the GPU.  model_points needs
// scratch for its derived tables (per-channel flux and LMN) and takes it from
// a buffer that grows with cudaMalloc; this entry point uses a fixed array
// compiled into the library instead and never allocates.
//
// The scratch is the file-scope device array below (HDC_NOALLOC_SCRATCH_BYTES,
// 16 MiB), which every GPU that loads the library holds until the process
// exits.  A call needs 64 B per component (LMN and envelope tables, 32 B
// each) plus 64 B per (channel, component) (the flux table), each table
// rounded up to 256 B; larger problems are rejected with an error before
// anything is launched.  After the kernels the call reads its own error word
// (a synchronous read on the legacy default stream), clears it if set and
// returns the message, so a call never leaves an error for the next one.
// The array is shared by all calls on a device and keeps the previous call's
// contents; every call rewrites all of the scratch it reads, so nothing
// needs clearing between calls.  Calls whose kernels overlap on
// the GPU (concurrent calls from several host threads or streams on one
// device) race on the array and must be serialised by the caller.
//
// In host code the array's name is only a host-side stand-in, so its device
// address is looked up with cudaGetSymbolAddress once per device, with that
// device current, the first time the entry point runs on it; that first call
// on a device should come before any stream capture.

#include <mutex>

#include "predict.cuh"

namespace hdc {
size_t points_workspace_bytes(int nc, int nf);
const char* points_with_workspace(const Points* comps, const Addresses* a, const UVW* d_uvws,
                                  const JonesF64* d_beam_jones, JonesF32* d_vis_fb, void* ws, size_t ws_bytes,
                                  int* err_word);
}  // namespace hdc

static __device__ __align__(256) unsigned char g_points_scratch[HDC_NOALLOC_SCRATCH_BYTES];
static __device__ int g_points_err;

namespace {
constexpr int MAX_DEV = 64;
std::mutex g_mu;
void* g_scratch_addr[MAX_DEV] = {};
int* g_err_addr[MAX_DEV] = {};

// Device addresses of the scratch array and error word on device `dev`
// (which must be current).  Looked up once per device.
const char* device_addresses(int dev, void** ws, int** err) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        int* q = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_points_scratch);
        if (e != cudaSuccess) {
            hdc::set_error("model_points_noalloc: cudaGetSymbolAddress: %s", cudaGetErrorString(e));
            return cudaGetErrorString(e);
        }
        e = cudaGetSymbolAddress((void**)&q, g_points_err);
        if (e != cudaSuccess) {
            hdc::set_error("model_points_noalloc: cudaGetSymbolAddress: %s", cudaGetErrorString(e));
            return cudaGetErrorString(e);
        }
        g_scratch_addr[dev] = p;
        g_err_addr[dev] = q;
    }
    *ws = g_scratch_addr[dev];
    *err = g_err_addr[dev];
    return NULL;
}
}  // namespace

extern "C" const char* model_points_noalloc(const Points* comps, const Addresses* a, const UVW* d_uvws,
                                            const JonesF64* d_beam_jones, JonesF32* d_vis_fb) {
    if (!comps || !a) return "model_points_noalloc: NULL argument";
    const int nc = comps->num_power_laws + comps->num_curved_power_laws + comps->num_lists;
    if (nc == 0) return NULL;
    const size_t need = hdc::points_workspace_bytes(nc, a->num_freqs);
    if (need > (size_t)HDC_NOALLOC_SCRATCH_BYTES) {
        hdc::set_error("model_points_noalloc: %d channels x %d components need %zu bytes of scratch; the limit is %u",
                       a->num_freqs, nc, need, (unsigned)HDC_NOALLOC_SCRATCH_BYTES);
        return "model_points_noalloc: channels x components exceed the fixed scratch (16 MiB); use model_points";
    }
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cudaGetErrorString(e);
    if (dev < 0 || dev >= MAX_DEV) return "model_points_noalloc: device index out of range";
    void* ws = nullptr;
    int* err = nullptr;
    const char* r = device_addresses(dev, &ws, &err);
    if (r) return r;
    return hdc::points_with_workspace(comps, a, d_uvws, d_beam_jones, d_vis_fb, ws, (size_t)HDC_NOALLOC_SCRATCH_BYTES,
                                      err);
}
