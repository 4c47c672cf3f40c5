// A small multilayer perceptron with hand-written FP32 CUDA training and
// inference kernels: the learned warm start for DI calibration (this project's
// addition; mwa_hyperdrive has no counterpart).
//
// Layers: y_0 = x; y_l = relu(y_{l-1} W_l^T + b_l) for hidden layers; the
// output layer is linear; if `residual_dim` > 0 the output adds the input
// slice x[:, residual_offset : residual_offset + out_dim] (the net predicts a
// correction to the centre input).  Training minimises the mean squared error
// with Adam.
//
// Kernels: one tiled SGEMM (64x64 output tile per 256-thread CTA, 4x4 per
// thread, K staged through shared memory 16 at a time) with transpose flags
// and a fused bias + ReLU epilogue, a bias-gradient column reduction, the
// ReLU backward mask, the MSE gradient and the Adam update.

#include <cmath>
#include <cstring>
#include <random>
#include <vector>

#include "common.cuh"

namespace hdc {
namespace mlp {

constexpr int TM = 64, TN = 64, TK = 16;

// C[M][N] (row-major, ldc) = op(A) op(B) (+ bias[N]) (relu), where
// op(A)[m][k] = TA ? A[k][m] : A[m][k] (lda) and op(B)[k][n] = TB ? B[n][k] : B[k][n] (ldb).
// beta: 0 overwrite, 1 accumulate.
template <bool TA, bool TB>
__global__ void __launch_bounds__(256) sgemm_kernel(int M, int N, int K, const float* __restrict__ A, int lda,
                                                    const float* __restrict__ B, int ldb, float* __restrict__ C,
                                                    int ldc, const float* __restrict__ bias, int relu, float beta) {
    __shared__ float As[TK][TM + 4];
    __shared__ float Bs[TK][TN + 4];
    const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
    const int m0 = blockIdx.y * TM, n0 = blockIdx.x * TN;
    float acc[4][4] = {};
    for (int k0 = 0; k0 < K; k0 += TK) {
        for (int i = threadIdx.x; i < TK * TM; i += 256) {
            const int kk = i / TM, mm = i % TM;
            const int m = m0 + mm, k = k0 + kk;
            float v = 0.f;
            if (m < M && k < K) v = TA ? A[(size_t)k * lda + m] : A[(size_t)m * lda + k];
            As[kk][mm] = v;
        }
        for (int i = threadIdx.x; i < TK * TN; i += 256) {
            const int kk = i / TN, nn = i % TN;
            const int n = n0 + nn, k = k0 + kk;
            float v = 0.f;
            if (n < N && k < K) v = TB ? B[(size_t)n * ldb + k] : B[(size_t)k * ldb + n];
            Bs[kk][nn] = v;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < TK; kk++) {
            float a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; i++) a[i] = As[kk][ty * 4 + i];
#pragma unroll
            for (int j = 0; j < 4; j++) b[j] = Bs[kk][tx * 4 + j];
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const int m = m0 + ty * 4 + i;
        if (m >= M) continue;
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int n = n0 + tx * 4 + j;
            if (n >= N) continue;
            float v = acc[i][j];
            if (bias) v += bias[n];
            if (relu) v = fmaxf(v, 0.f);
            float* c = C + (size_t)m * ldc + n;
            *c = beta != 0.f ? *c + v : v;
        }
    }
}

template <bool TA, bool TB>
static cudaError_t sgemm(int M, int N, int K, const float* A, int lda, const float* B, int ldb, float* C, int ldc,
                         const float* bias, bool relu, float beta, cudaStream_t s) {
    dim3 grid((N + TN - 1) / TN, (M + TM - 1) / TM);
    sgemm_kernel<TA, TB><<<grid, 256, 0, s>>>(M, N, K, A, lda, B, ldb, C, ldc, bias, relu ? 1 : 0, beta);
    count_launches(1);
    return cudaGetLastError();
}

__global__ void add_residual_kernel(float* y, const float* x, int batch, int out_dim, int in_dim, int offset) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= batch * out_dim) return;
    const int b = i / out_dim, j = i % out_dim;
    y[i] += x[(size_t)b * in_dim + offset + j];
}

// d = 2 (y - t) / (batch * out_dim); loss partial sums per block
__global__ void mse_grad_kernel(const float* y, const float* t, float* d, int n, float scale, double* loss) {
    __shared__ double red[256];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double l = 0.0;
    if (i < n) {
        const float e = y[i] - t[i];
        d[i] = 2.f * e * scale;
        l = (double)e * e;
    }
    red[threadIdx.x] = l;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) atomicAdd(loss, red[0]);
}

__global__ void relu_backward_kernel(float* d, const float* act, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && act[i] <= 0.f) d[i] = 0.f;
}

// db[n] = sum_b d[b][n]
__global__ void bias_grad_kernel(const float* d, float* db, int batch, int n) {
    const int j = blockIdx.x;
    float s = 0.f;
    for (int b = threadIdx.x; b < batch; b += blockDim.x) s += d[(size_t)b * n + j];
    __shared__ float red[256];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) db[j] = red[0];
}

__global__ void adam_kernel(float* p, const float* g, float* m, float* v, int n, float lr, float b1, float b2,
                            float eps, float c1, float c2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

struct Net {
    std::vector<int> dims;  // n_layers + 1
    int residual_offset = -1;
    float *d_params = nullptr, *d_grads = nullptr, *d_m = nullptr, *d_v = nullptr;
    size_t nparams = 0;
    std::vector<size_t> w_off, b_off;
    // activations for training
    std::vector<float*> acts, deltas;
    int cap_batch = 0;
    double* d_loss = nullptr;
    long long step = 0;

    int layers() const { return (int)dims.size() - 1; }

    void free_acts() {
        for (float* p : acts) cudaFree(p);
        for (float* p : deltas) cudaFree(p);
        acts.clear();
        deltas.clear();
        cap_batch = 0;
    }

    int ensure(int batch) {
        if (batch <= cap_batch) return HDC_OK;
        free_acts();
        for (int l = 0; l <= layers(); l++) {
            float *a = nullptr, *d = nullptr;
            if (cudaMalloc(&a, sizeof(float) * (size_t)batch * dims[l]) != cudaSuccess ||
                cudaMalloc(&d, sizeof(float) * (size_t)batch * dims[l]) != cudaSuccess) {
                cudaGetLastError();
                set_error("mlp: activation allocation failed");
                return HDC_ERR_ALLOC;
            }
            acts.push_back(a);
            deltas.push_back(d);
        }
        cap_batch = batch;
        return HDC_OK;
    }

    ~Net() {
        free_acts();
        cudaFree(d_params);
        cudaFree(d_grads);
        cudaFree(d_m);
        cudaFree(d_v);
        cudaFree(d_loss);
    }

    // forward into acts[0..L] (acts[0] = x copy), returns output pointer
    int forward(const float* d_x, int batch, cudaStream_t s) {
        int rc = ensure(batch);
        if (rc) return rc;
        HDC_CUDA_RET_INT(cudaMemcpyAsync(acts[0], d_x, sizeof(float) * (size_t)batch * dims[0],
                                         cudaMemcpyDeviceToDevice, s));
        for (int l = 0; l < layers(); l++) {
            const bool last = l == layers() - 1;
            HDC_CUDA_RET_INT((sgemm<false, true>(batch, dims[l + 1], dims[l], acts[l], dims[l], d_params + w_off[l],
                                                 dims[l], acts[l + 1], dims[l + 1], d_params + b_off[l], !last, 0.f,
                                                 s)));
        }
        if (residual_offset >= 0) {
            const int n = batch * dims.back();
            add_residual_kernel<<<(n + 255) / 256, 256, 0, s>>>(acts.back(), acts[0], batch, dims.back(), dims[0],
                                                                residual_offset);
            count_launches(1);
            HDC_CUDA_RET_INT(cudaGetLastError());
        }
        return HDC_OK;
    }

    // gradients of the mean squared error into d_grads; loss (sum of squares / n) to *loss
    int backward(const float* d_target, int batch, double* h_loss, cudaStream_t s) {
        const int L = layers();
        const int n = batch * dims[L];
        HDC_CUDA_RET_INT(cudaMemsetAsync(d_loss, 0, sizeof(double), s));
        mse_grad_kernel<<<(n + 255) / 256, 256, 0, s>>>(acts[L], d_target, deltas[L], n, 1.f / (float)n, d_loss);
        count_launches(1);
        for (int l = L - 1; l >= 0; l--) {
            // dW_l = delta_{l+1}^T y_l : [out][in];  db_l = colsum(delta_{l+1})
            HDC_CUDA_RET_INT((sgemm<true, false>(dims[l + 1], dims[l], batch, deltas[l + 1], dims[l + 1], acts[l],
                                                 dims[l], d_grads + w_off[l], dims[l], nullptr, false, 0.f, s)));
            bias_grad_kernel<<<dims[l + 1], 256, 0, s>>>(deltas[l + 1], d_grads + b_off[l], batch, dims[l + 1]);
            count_launches(1);
            if (l > 0) {
                // delta_l = (delta_{l+1} W_l) * relu'(y_l)
                HDC_CUDA_RET_INT((sgemm<false, false>(batch, dims[l], dims[l + 1], deltas[l + 1], dims[l + 1],
                                                      d_params + w_off[l], dims[l], deltas[l], dims[l], nullptr, false,
                                                      0.f, s)));
                const int nl = batch * dims[l];
                relu_backward_kernel<<<(nl + 255) / 256, 256, 0, s>>>(deltas[l], acts[l], nl);
                count_launches(1);
            }
        }
        HDC_CUDA_RET_INT(cudaGetLastError());
        if (h_loss) {
            double l = 0.0;
            HDC_CUDA_RET_INT(cudaMemcpyAsync(&l, d_loss, sizeof(double), cudaMemcpyDeviceToHost, s));
            HDC_CUDA_RET_INT(cudaStreamSynchronize(s));
            *h_loss = l / (double)n;
        }
        return HDC_OK;
    }
};

}  // namespace mlp
}  // namespace hdc

using hdc::mlp::Net;

extern "C" int hdc_mlp_new(int num_layers, const int* dims, int residual_offset, unsigned long long seed,
                           HdcMlp** out) {
    if (num_layers < 1 || !dims || !out) return HDC_ERR_ARG;
    Net* n = new Net();
    n->dims.assign(dims, dims + num_layers + 1);
    n->residual_offset = residual_offset;
    if (residual_offset >= 0 && residual_offset + dims[num_layers] > dims[0]) {
        delete n;
        hdc::set_error("mlp: residual slice outside the input");
        return HDC_ERR_ARG;
    }
    size_t off = 0;
    for (int l = 0; l < num_layers; l++) {
        n->w_off.push_back(off);
        off += (size_t)dims[l] * dims[l + 1];
        n->b_off.push_back(off);
        off += dims[l + 1];
    }
    n->nparams = off;
    // He initialisation for hidden layers; the output layer starts at zero so
    // that a residual net begins as the identity map of its centre input.
    std::vector<float> h(off, 0.f);
    std::mt19937_64 rng(seed);
    for (int l = 0; l < num_layers; l++) {
        const bool last = l == num_layers - 1;
        std::normal_distribution<float> nd(0.f, std::sqrt(2.f / dims[l]));
        for (size_t i = 0; i < (size_t)dims[l] * dims[l + 1]; i++) h[n->w_off[l] + i] = last ? 0.f : nd(rng);
    }
    if (cudaMalloc(&n->d_params, sizeof(float) * off) != cudaSuccess ||
        cudaMalloc(&n->d_grads, sizeof(float) * off) != cudaSuccess ||
        cudaMalloc(&n->d_m, sizeof(float) * off) != cudaSuccess || cudaMalloc(&n->d_v, sizeof(float) * off) != cudaSuccess ||
        cudaMalloc(&n->d_loss, sizeof(double)) != cudaSuccess) {
        cudaGetLastError();
        delete n;
        hdc::set_error("mlp: parameter allocation failed");
        return HDC_ERR_ALLOC;
    }
    cudaMemcpy(n->d_params, h.data(), sizeof(float) * off, cudaMemcpyHostToDevice);
    cudaMemset(n->d_m, 0, sizeof(float) * off);
    cudaMemset(n->d_v, 0, sizeof(float) * off);
    cudaMemset(n->d_grads, 0, sizeof(float) * off);
    *out = reinterpret_cast<HdcMlp*>(n);
    return HDC_OK;
}

extern "C" void hdc_mlp_free(HdcMlp* m) { delete reinterpret_cast<Net*>(m); }

namespace hdc {
// input and output widths of a network (for callers that build its inputs)
int mlp_io_dims(HdcMlp* m, int* in, int* out) {
    if (!m) return HDC_ERR_ARG;
    const Net* n = reinterpret_cast<const Net*>(m);
    *in = n->dims.front();
    *out = n->dims.back();
    return HDC_OK;
}
}  // namespace hdc

extern "C" long long hdc_mlp_num_params(HdcMlp* m) { return (long long)reinterpret_cast<Net*>(m)->nparams; }

extern "C" int hdc_mlp_get_params(HdcMlp* hm, float* h_out) {
    Net* n = reinterpret_cast<Net*>(hm);
    HDC_CUDA_RET_INT(cudaMemcpy(h_out, n->d_params, sizeof(float) * n->nparams, cudaMemcpyDeviceToHost));
    return HDC_OK;
}

extern "C" int hdc_mlp_set_params(HdcMlp* hm, const float* h_in) {
    Net* n = reinterpret_cast<Net*>(hm);
    HDC_CUDA_RET_INT(cudaMemcpy(n->d_params, h_in, sizeof(float) * n->nparams, cudaMemcpyHostToDevice));
    return HDC_OK;
}

extern "C" int hdc_mlp_forward(HdcMlp* hm, const float* d_x, int batch, float* d_y, hdcStream_t stream) {
    Net* n = reinterpret_cast<Net*>(hm);
    cudaStream_t s = (cudaStream_t)stream;
    int rc = n->forward(d_x, batch, s);
    if (rc) return rc;
    HDC_CUDA_RET_INT(cudaMemcpyAsync(d_y, n->acts.back(), sizeof(float) * (size_t)batch * n->dims.back(),
                                     cudaMemcpyDeviceToDevice, s));
    return HDC_OK;
}

extern "C" int hdc_mlp_gradients(HdcMlp* hm, const float* d_x, const float* d_target, int batch, float* h_grads,
                                 double* h_loss, hdcStream_t stream) {
    Net* n = reinterpret_cast<Net*>(hm);
    cudaStream_t s = (cudaStream_t)stream;
    int rc = n->forward(d_x, batch, s);
    if (rc) return rc;
    rc = n->backward(d_target, batch, h_loss, s);
    if (rc) return rc;
    if (h_grads) {
        HDC_CUDA_RET_INT(cudaMemcpyAsync(h_grads, n->d_grads, sizeof(float) * n->nparams, cudaMemcpyDeviceToHost, s));
        HDC_CUDA_RET_INT(cudaStreamSynchronize(s));
    }
    return HDC_OK;
}

extern "C" int hdc_mlp_train_step(HdcMlp* hm, const float* d_x, const float* d_target, int batch, float lr,
                                  double* h_loss, hdcStream_t stream) {
    Net* n = reinterpret_cast<Net*>(hm);
    cudaStream_t s = (cudaStream_t)stream;
    int rc = n->forward(d_x, batch, s);
    if (rc) return rc;
    rc = n->backward(d_target, batch, h_loss, s);
    if (rc) return rc;
    n->step++;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - std::pow(b1, (float)n->step), c2 = 1.f - std::pow(b2, (float)n->step);
    const int np = (int)n->nparams;
    hdc::mlp::adam_kernel<<<(np + 255) / 256, 256, 0, s>>>(n->d_params, n->d_grads, n->d_m, n->d_v, np, lr, b1, b2,
                                                           1e-8f, c1, c2);
    hdc::count_launches(1);
    HDC_CUDA_RET_INT(cudaGetLastError());
    return HDC_OK;
}
