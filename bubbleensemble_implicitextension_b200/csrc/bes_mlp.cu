/*
 * bes_mlp.cu -- the surrogate network: a small MLP trained and evaluated
 * with the library's own CUDA kernels (no reference counterpart).
 *
 * Network: n_in -> width (GELU) x depth -> n_out.  Inputs and targets are
 * standardised with caller-given means and deviations; the loss is the mean
 * squared error of the standardised outputs.  Storage and arithmetic:
 *   - master weights and biases in FP32, Adam moments in FP32;
 *   - weights used by the kernels rounded to BF16 after every update;
 *   - layer inputs (activations) stored in BF16, pre-activations in FP32;
 *   - every product accumulated in FP32 (tiled GEMM, 64 x 64 tiles).
 * GELU is the tanh form 0.5 x (1 + tanh(sqrt(2/pi) (x + 0.044715 x^3))).
 * Parameter vector layout (get/set): for each layer, W [fan_out][fan_in]
 * row-major, then b [fan_out].
 */
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/bes.h"

namespace {

constexpr int TILE = 64;
constexpr int KT = 16;

__device__ __forceinline__ float to_f(float v) { return v; }
__device__ __forceinline__ float to_f(__nv_bfloat16 v) { return __bfloat162float(v); }

/* C[M x N] = A[M x K] B[K x N]; A(m,k) = TA ? A[k*lda + m] : A[m*lda + k],
 * B(k,n) = TB ? B[n*ldb + k] : B[k*ldb + n]; FP32 accumulation. */
template <class TypeA, class TypeB, bool TA, bool TB>
__global__ void __launch_bounds__(256) gemm_kernel(int M, int N, int K, const TypeA* __restrict__ A, int lda,
                                                   const TypeB* __restrict__ B, int ldb, float* __restrict__ C,
                                                   int ldc) {
    __shared__ float As[KT][TILE + 1];
    __shared__ float Bs[KT][TILE + 1];
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    const int m0 = blockIdx.y * TILE, n0 = blockIdx.x * TILE;
    float acc[4][4];
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
        for (int b = 0; b < 4; b++) acc[a][b] = 0.f;
    for (int k0 = 0; k0 < K; k0 += KT) {
        /* 64 x 16 tile of A and 16 x 64 tile of B, 4 elements each per thread */
        for (int e = threadIdx.x; e < TILE * KT; e += 256) {
            const int mm = e % TILE, kk = e / TILE;
            const int gm = m0 + mm, gk = k0 + kk;
            float va = 0.f;
            if (gm < M && gk < K) va = to_f(TA ? A[(int64_t)gk * lda + gm] : A[(int64_t)gm * lda + gk]);
            As[kk][mm] = va;
            const int gn = n0 + mm;
            float vb = 0.f;
            if (gn < N && gk < K) vb = to_f(TB ? B[(int64_t)gn * ldb + gk] : B[(int64_t)gk * ldb + gn]);
            Bs[kk][mm] = vb;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < KT; kk++) {
            float a[4], b[4];
#pragma unroll
            for (int r = 0; r < 4; r++) a[r] = As[kk][ty + 16 * r];
#pragma unroll
            for (int c = 0; c < 4; c++) b[c] = Bs[kk][tx + 16 * c];
#pragma unroll
            for (int r = 0; r < 4; r++)
#pragma unroll
                for (int c = 0; c < 4; c++) acc[r][c] = fmaf(a[r], b[c], acc[r][c]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int r = 0; r < 4; r++)
#pragma unroll
        for (int c = 0; c < 4; c++) {
            const int gm = m0 + ty + 16 * r, gn = n0 + tx + 16 * c;
            if (gm < M && gn < N) C[(int64_t)gm * ldc + gn] = acc[r][c];
        }
}

__device__ __forceinline__ float gelu_t(float x) {
    const float c = 0.7978845608028654f; /* sqrt(2/pi) */
    return 0.5f * x * (1.f + tanhf(c * (x + 0.044715f * x * x * x)));
}
__device__ __forceinline__ float gelu_dt(float x) {
    const float c = 0.7978845608028654f;
    const float t = tanhf(c * (x + 0.044715f * x * x * x));
    return 0.5f * (1.f + t) + 0.5f * x * (1.f - t * t) * c * (1.f + 3.f * 0.044715f * x * x);
}

__global__ void normalize_input(const float* __restrict__ x, int batch, int n_in, const float* __restrict__ mean,
                                const float* __restrict__ stdv, __nv_bfloat16* __restrict__ out) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= (int64_t)batch * n_in) return;
    const int f = (int)(i % n_in);
    out[i] = __float2bfloat16_rn((x[i] - mean[f]) / stdv[f]);
}

/* pre += bias; next = bf16(gelu(pre)) (hidden layers) */
__global__ void bias_gelu(float* __restrict__ pre, const float* __restrict__ bias, int batch, int n,
                          __nv_bfloat16* __restrict__ next) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= (int64_t)batch * n) return;
    const float z = pre[i] + bias[i % n];
    pre[i] = z;
    next[i] = __float2bfloat16_rn(gelu_t(z));
}

/* last layer: pre += bias; y = pre * out_std + out_mean */
__global__ void bias_output(float* __restrict__ pre, const float* __restrict__ bias, int batch, int n,
                            const float* __restrict__ omean, const float* __restrict__ ostd, float* __restrict__ y) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= (int64_t)batch * n) return;
    const int f = (int)(i % n);
    const float z = pre[i] + bias[f];
    pre[i] = z;
    if (y) y[i] = z * ostd[f] + omean[f];
}

/* dZ = 2 (z - (t - mean)/std) / (batch n); per-element squared error into err */
__global__ void mse_grad(const float* __restrict__ z, const float* __restrict__ t, int batch, int n,
                         const float* __restrict__ omean, const float* __restrict__ ostd, float* __restrict__ dz,
                         float* __restrict__ err) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= (int64_t)batch * n) return;
    const int f = (int)(i % n);
    const float d = z[i] - (t[i] - omean[f]) / ostd[f];
    dz[i] = 2.f * d / (float)((int64_t)batch * n);
    err[i] = d * d;
}

/* dZ_prev = dX * gelu'(pre_prev) */
__global__ void gelu_back(float* __restrict__ dx, const float* __restrict__ pre, int64_t count) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < count) dx[i] = dx[i] * gelu_dt(pre[i]);
}

/* db[o] = sum_b dZ[b][o] (one warp per output column, fixed order) */
__global__ void column_sum(const float* __restrict__ dz, int batch, int n, float* __restrict__ db) {
    const int o = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (o >= n) return;
    float s = 0.f;
    for (int b = lane; b < batch; b += 32) s += dz[(int64_t)b * n + o];
#pragma unroll
    for (int off = 16; off >= 1; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
    if (lane == 0) db[o] = s;
}

__global__ void sum_errors(const float* __restrict__ err, int64_t count, float* __restrict__ out) {
    __shared__ float part[256];
    float s = 0.f;
    for (int64_t i = threadIdx.x; i < count; i += blockDim.x) s += err[i];
    part[threadIdx.x] = s;
    __syncthreads();
    for (int h = 128; h >= 1; h >>= 1) {
        if (threadIdx.x < h) part[threadIdx.x] += part[threadIdx.x + h];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[0] = part[0] / (float)count;
}

/* Adam on the FP32 master parameters, then the BF16 copies of the weights */
__global__ void adam_update(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, int64_t count, float lr, float b1, float b2, float eps, float c1,
                            float c2, const uint8_t* __restrict__ is_weight, const int64_t* __restrict__ wb_index,
                            __nv_bfloat16* __restrict__ wb) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= count) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    w[i] = wi;
    if (is_weight[i]) wb[wb_index[i]] = __float2bfloat16_rn(wi);
}

__global__ void refresh_bf16(const float* __restrict__ w, int64_t count, const uint8_t* __restrict__ is_weight,
                             const int64_t* __restrict__ wb_index, __nv_bfloat16* __restrict__ wb) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < count && is_weight[i]) wb[wb_index[i]] = __float2bfloat16_rn(w[i]);
}

inline int blocks_for(int64_t n, int t) { return (int)((n + t - 1) / t); }

}  // namespace

struct bes_mlp {
    int device = 0;
    int n_in = 0, width = 0, depth = 0, n_out = 0, max_batch = 0, n_layers = 0;
    std::vector<int> fin, fout;
    std::vector<int64_t> w_off, b_off, wb_off; /* offsets in the parameter vector and in the BF16 weights */
    int64_t n_params = 0, n_wb = 0;
    float *master = nullptr, *grad = nullptr, *mom1 = nullptr, *mom2 = nullptr;
    __nv_bfloat16* wb = nullptr;
    uint8_t* is_weight = nullptr;
    int64_t* wb_index = nullptr;
    std::vector<__nv_bfloat16*> act; /* layer inputs, [n_layers] */
    std::vector<float*> pre;         /* pre-activations, [n_layers] */
    float *dbuf0 = nullptr, *dbuf1 = nullptr, *err = nullptr, *loss = nullptr;
    float *in_mean = nullptr, *in_std = nullptr, *out_mean = nullptr, *out_std = nullptr;
    float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    int64_t step = 0;
    std::string errmsg;
};

namespace {

bes_status mfail(bes_mlp* h, bes_status st, const char* msg, cudaError_t e = cudaSuccess) {
    if (h) h->errmsg = std::string(msg) + (e != cudaSuccess ? std::string(": ") + cudaGetErrorString(e) : "");
    return st;
}

#define MLP_TRY(h, call)                                         \
    do {                                                         \
        cudaError_t e_ = (call);                                 \
        if (e_ != cudaSuccess) return mfail((h), BES_ERR_CUDA, #call, e_); \
    } while (0)

void free_mlp(bes_mlp* h) {
    cudaSetDevice(h->device);
    void* ps[] = {h->master, h->grad, h->mom1, h->mom2, h->wb, h->is_weight, h->wb_index, h->dbuf0, h->dbuf1,
                  h->err, h->loss, h->in_mean, h->in_std, h->out_mean, h->out_std};
    for (void* p : ps)
        if (p) cudaFree(p);
    for (auto* p : h->act)
        if (p) cudaFree(p);
    for (auto* p : h->pre)
        if (p) cudaFree(p);
}

template <class TA, class TB, bool A_T, bool B_T>
cudaError_t gemm(int M, int N, int K, const TA* A, int lda, const TB* B, int ldb, float* C, int ldc,
                 cudaStream_t s) {
    dim3 grid((N + TILE - 1) / TILE, (M + TILE - 1) / TILE);
    gemm_kernel<TA, TB, A_T, B_T><<<grid, 256, 0, s>>>(M, N, K, A, lda, B, ldb, C, ldc);
    return cudaGetLastError();
}

/* forward through every layer; y (device, may be null) gets the de-standardised outputs */
bes_status forward(bes_mlp* h, const float* x, int batch, float* y, cudaStream_t s) {
    normalize_input<<<blocks_for((int64_t)batch * h->n_in, 256), 256, 0, s>>>(x, batch, h->n_in, h->in_mean,
                                                                              h->in_std, h->act[0]);
    MLP_TRY(h, cudaGetLastError());
    for (int l = 0; l < h->n_layers; l++) {
        const int I = h->fin[l], O = h->fout[l];
        MLP_TRY(h, (gemm<__nv_bfloat16, __nv_bfloat16, false, true>(batch, O, I, h->act[l], I, h->wb + h->wb_off[l],
                                                                     I, h->pre[l], O, s)));
        if (l + 1 < h->n_layers)
            bias_gelu<<<blocks_for((int64_t)batch * O, 256), 256, 0, s>>>(h->pre[l], h->master + h->b_off[l], batch, O,
                                                                        h->act[l + 1]);
        else
            bias_output<<<blocks_for((int64_t)batch * O, 256), 256, 0, s>>>(h->pre[l], h->master + h->b_off[l], batch,
                                                                           O, h->out_mean, h->out_std, y);
        MLP_TRY(h, cudaGetLastError());
    }
    return BES_OK;
}

}  // namespace

extern "C" {

bes_status bes_mlp_create(const bes_mlp_config* c, bes_mlp** out) {
    if (!c || !out || c->n_in < 1 || c->width < 1 || c->depth < 1 || c->n_out < 1 || c->max_batch < 1)
        return BES_ERR_ARGUMENT;
    *out = nullptr;
    bes_mlp* h = new bes_mlp();
    h->device = c->device;
    h->n_in = c->n_in;
    h->width = c->width;
    h->depth = c->depth;
    h->n_out = c->n_out;
    h->max_batch = c->max_batch;
    h->n_layers = c->depth + 1;
    for (int l = 0; l < h->n_layers; l++) {
        h->fin.push_back(l == 0 ? c->n_in : c->width);
        h->fout.push_back(l + 1 == h->n_layers ? c->n_out : c->width);
    }
    for (int l = 0; l < h->n_layers; l++) {
        h->w_off.push_back(h->n_params);
        h->n_params += (int64_t)h->fin[l] * h->fout[l];
        h->b_off.push_back(h->n_params);
        h->n_params += h->fout[l];
        h->wb_off.push_back(h->n_wb);
        h->n_wb += (int64_t)h->fin[l] * h->fout[l];
    }
    if (cudaSetDevice(h->device) != cudaSuccess) { delete h; return BES_ERR_CUDA; }
    /* host-side initialisation: uniform(-1, 1) * sqrt(6 / fan_in) (He-uniform), biases 0,
     * from a splitmix64 stream of the given seed */
    std::vector<float> w(h->n_params, 0.f);
    std::vector<uint8_t> isw(h->n_params, 0);
    std::vector<int64_t> wbi(h->n_params, 0);
    uint64_t st = c->seed * 0x9E3779B97F4A7C15ULL + 0x1234567ULL;
    auto next = [&]() {
        uint64_t z = (st += 0x9E3779B97F4A7C15ULL);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
        return z ^ (z >> 31);
    };
    for (int l = 0; l < h->n_layers; l++) {
        const float a = std::sqrt(6.f / (float)h->fin[l]);
        for (int64_t k = 0; k < (int64_t)h->fin[l] * h->fout[l]; k++) {
            const double u = (double)(next() >> 11) * (1.0 / 9007199254740992.0);
            w[h->w_off[l] + k] = (float)((2.0 * u - 1.0) * a);
            isw[h->w_off[l] + k] = 1;
            wbi[h->w_off[l] + k] = h->wb_off[l] + k;
        }
    }
    const size_t P = (size_t)h->n_params;
    cudaError_t e = cudaSuccess;
    auto mal = [&](void** p, size_t bytes) { if (e == cudaSuccess) e = cudaMalloc(p, bytes); };
    mal((void**)&h->master, P * 4);
    mal((void**)&h->grad, P * 4);
    mal((void**)&h->mom1, P * 4);
    mal((void**)&h->mom2, P * 4);
    mal((void**)&h->wb, (size_t)h->n_wb * 2);
    mal((void**)&h->is_weight, P);
    mal((void**)&h->wb_index, P * 8);
    const int64_t B = c->max_batch;
    h->act.assign(h->n_layers, nullptr);
    h->pre.assign(h->n_layers, nullptr);
    for (int l = 0; l < h->n_layers; l++) {
        mal((void**)&h->act[l], (size_t)B * h->fin[l] * 2);
        mal((void**)&h->pre[l], (size_t)B * h->fout[l] * 4);
    }
    const int wmax = std::max(std::max(c->width, c->n_in), c->n_out);
    mal((void**)&h->dbuf0, (size_t)B * wmax * 4);
    mal((void**)&h->dbuf1, (size_t)B * wmax * 4);
    mal((void**)&h->err, (size_t)B * c->n_out * 4);
    mal((void**)&h->loss, 4);
    mal((void**)&h->in_mean, (size_t)c->n_in * 4);
    mal((void**)&h->in_std, (size_t)c->n_in * 4);
    mal((void**)&h->out_mean, (size_t)c->n_out * 4);
    mal((void**)&h->out_std, (size_t)c->n_out * 4);
    if (e == cudaSuccess) e = cudaMemcpy(h->master, w.data(), P * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(h->is_weight, isw.data(), P, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(h->wb_index, wbi.data(), P * 8, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(h->mom1, 0, P * 4);
    if (e == cudaSuccess) e = cudaMemset(h->mom2, 0, P * 4);
    if (e == cudaSuccess) e = cudaMemset(h->grad, 0, P * 4);
    std::vector<float> zeros(std::max(c->n_in, c->n_out), 0.f), ones(std::max(c->n_in, c->n_out), 1.f);
    if (e == cudaSuccess) e = cudaMemcpy(h->in_mean, zeros.data(), c->n_in * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(h->in_std, ones.data(), c->n_in * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(h->out_mean, zeros.data(), c->n_out * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(h->out_std, ones.data(), c->n_out * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        refresh_bf16<<<blocks_for(h->n_params, 256), 256>>>(h->master, h->n_params, h->is_weight, h->wb_index, h->wb);
        e = cudaDeviceSynchronize();
    }
    if (e != cudaSuccess) {
        free_mlp(h);
        delete h;
        return e == cudaErrorMemoryAllocation ? BES_ERR_MEMORY : BES_ERR_CUDA;
    }
    *out = h;
    return BES_OK;
}

bes_status bes_mlp_destroy(bes_mlp* h) {
    if (!h) return BES_ERR_ARGUMENT;
    free_mlp(h);
    delete h;
    return BES_OK;
}

bes_status bes_mlp_parameter_count(bes_mlp* h, int64_t* count) {
    if (!h || !count) return BES_ERR_ARGUMENT;
    *count = h->n_params;
    return BES_OK;
}

bes_status bes_mlp_set_normalization(bes_mlp* h, const float* in_mean, const float* in_std, const float* out_mean,
                                     const float* out_std) {
    if (!h || !in_mean || !in_std || !out_mean || !out_std) return BES_ERR_ARGUMENT;
    MLP_TRY(h, cudaSetDevice(h->device));
    MLP_TRY(h, cudaMemcpy(h->in_mean, in_mean, h->n_in * 4, cudaMemcpyHostToDevice));
    MLP_TRY(h, cudaMemcpy(h->in_std, in_std, h->n_in * 4, cudaMemcpyHostToDevice));
    MLP_TRY(h, cudaMemcpy(h->out_mean, out_mean, h->n_out * 4, cudaMemcpyHostToDevice));
    MLP_TRY(h, cudaMemcpy(h->out_std, out_std, h->n_out * 4, cudaMemcpyHostToDevice));
    return BES_OK;
}

bes_status bes_mlp_get_parameters(bes_mlp* h, float* host, int64_t count) {
    if (!h || !host || count != h->n_params) return BES_ERR_ARGUMENT;
    MLP_TRY(h, cudaSetDevice(h->device));
    MLP_TRY(h, cudaMemcpy(host, h->master, count * 4, cudaMemcpyDeviceToHost));
    return BES_OK;
}

bes_status bes_mlp_set_parameters(bes_mlp* h, const float* host, int64_t count) {
    if (!h || !host || count != h->n_params) return BES_ERR_ARGUMENT;
    MLP_TRY(h, cudaSetDevice(h->device));
    MLP_TRY(h, cudaMemcpy(h->master, host, count * 4, cudaMemcpyHostToDevice));
    refresh_bf16<<<blocks_for(h->n_params, 256), 256>>>(h->master, h->n_params, h->is_weight, h->wb_index, h->wb);
    MLP_TRY(h, cudaDeviceSynchronize());
    return BES_OK;
}

bes_status bes_mlp_get_gradients(bes_mlp* h, float* host, int64_t count) {
    if (!h || !host || count != h->n_params) return BES_ERR_ARGUMENT;
    MLP_TRY(h, cudaSetDevice(h->device));
    MLP_TRY(h, cudaMemcpy(host, h->grad, count * 4, cudaMemcpyDeviceToHost));
    return BES_OK;
}

bes_status bes_mlp_forward(bes_mlp* h, const float* x, int32_t batch, float* y, void* stream) {
    if (!h || !x || !y || batch < 1 || batch > h->max_batch) return BES_ERR_ARGUMENT;
    MLP_TRY(h, cudaSetDevice(h->device));
    return forward(h, x, batch, y, (cudaStream_t)stream);
}

bes_status bes_mlp_backward(bes_mlp* h, const float* x, const float* target, int32_t batch, float* loss_host,
                            void* stream) {
    if (!h || !x || !target || batch < 1 || batch > h->max_batch) return BES_ERR_ARGUMENT;
    MLP_TRY(h, cudaSetDevice(h->device));
    cudaStream_t s = (cudaStream_t)stream;
    bes_status st = forward(h, x, batch, nullptr, s);
    if (st) return st;
    const int L = h->n_layers;
    const int O_last = h->fout[L - 1];
    float* dz = h->dbuf0;
    float* dx = h->dbuf1;
    mse_grad<<<blocks_for((int64_t)batch * O_last, 256), 256, 0, s>>>(h->pre[L - 1], target, batch, O_last,
                                                                      h->out_mean, h->out_std, dz, h->err);
    MLP_TRY(h, cudaGetLastError());
    for (int l = L - 1; l >= 0; l--) {
        const int I = h->fin[l], O = h->fout[l];
        /* dW = dZ^T X, db = column sums of dZ */
        MLP_TRY(h, (gemm<float, __nv_bfloat16, true, false>(O, I, batch, dz, O, h->act[l], I, h->grad + h->w_off[l], I, s)));
        column_sum<<<blocks_for(O, 8), 256, 0, s>>>(dz, batch, O, h->grad + h->b_off[l]);
        MLP_TRY(h, cudaGetLastError());
        if (l > 0) {
            /* dX = dZ W, then through the previous GELU */
            MLP_TRY(h, (gemm<float, __nv_bfloat16, false, false>(batch, I, O, dz, O, h->wb + h->wb_off[l], I, dx, I, s)));
            gelu_back<<<blocks_for((int64_t)batch * I, 256), 256, 0, s>>>(dx, h->pre[l - 1], (int64_t)batch * I);
            MLP_TRY(h, cudaGetLastError());
            float* t = dz;
            dz = dx;
            dx = t;
        }
    }
    if (loss_host) {
        sum_errors<<<1, 256, 0, s>>>(h->err, (int64_t)batch * O_last, h->loss);
        MLP_TRY(h, cudaGetLastError());
        MLP_TRY(h, cudaMemcpyAsync(loss_host, h->loss, 4, cudaMemcpyDeviceToHost, s));
        MLP_TRY(h, cudaStreamSynchronize(s));
    }
    return BES_OK;
}

bes_status bes_mlp_adam_step(bes_mlp* h, float lr, void* stream) {
    if (!h) return BES_ERR_ARGUMENT;
    MLP_TRY(h, cudaSetDevice(h->device));
    h->step++;
    const float c1 = 1.f - std::pow(h->b1, (float)h->step);
    const float c2 = 1.f - std::pow(h->b2, (float)h->step);
    adam_update<<<blocks_for(h->n_params, 256), 256, 0, (cudaStream_t)stream>>>(
        h->master, h->grad, h->mom1, h->mom2, h->n_params, lr, h->b1, h->b2, h->eps, c1, c2, h->is_weight,
        h->wb_index, h->wb);
    MLP_TRY(h, cudaGetLastError());
    return BES_OK;
}

const char* bes_mlp_last_error(const bes_mlp* h) { return h ? h->errmsg.c_str() : ""; }

}  // extern "C"
