/*
 * bes_peak.cu -- FP64 fused multiply-add throughput probe (the roofline
 * denominator of the FP64 solver kernel; no reference counterpart).
 *
 * Every thread advances 8 independent FMA chains, so the FP64 pipe, not
 * latency, bounds the loop; the grid covers every SM several times over.
 */
#include <cuda_runtime.h>

#include "../../include/bes.h"

namespace {

__global__ void __launch_bounds__(256) fma_loop(double* out, int iters, double b, double c) {
    double a0 = threadIdx.x * 1e-9, a1 = a0 + 1e-3, a2 = a0 + 2e-3, a3 = a0 + 3e-3;
    double a4 = a0 + 4e-3, a5 = a0 + 5e-3, a6 = a0 + 6e-3, a7 = a0 + 7e-3;
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int k = 0; k < 16; k++) {
            a0 = fma(a0, b, c); a1 = fma(a1, b, c); a2 = fma(a2, b, c); a3 = fma(a3, b, c);
            a4 = fma(a4, b, c); a5 = fma(a5, b, c); a6 = fma(a6, b, c); a7 = fma(a7, b, c);
        }
    }
    double s = ((a0 + a1) + (a2 + a3)) + ((a4 + a5) + (a6 + a7));
    if (s == 12345.678) out[blockIdx.x * blockDim.x + threadIdx.x] = s; /* keeps the loop alive */
}

}  // namespace

extern "C" bes_status bes_measure_fp64_peak(int32_t device, double* tflops) {
    if (!tflops) return BES_ERR_ARGUMENT;
    *tflops = 0.0;
    if (cudaSetDevice(device) != cudaSuccess) return BES_ERR_CUDA;
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return BES_ERR_CUDA;
    const int threads = 256, blocks = sms * 8, iters = 2048;
    double* out = nullptr;
    if (cudaMalloc(&out, sizeof(double) * (size_t)threads * blocks) != cudaSuccess) return BES_ERR_MEMORY;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    fma_loop<<<blocks, threads>>>(out, iters / 8, 0.999999, 1e-7); /* warm-up */
    float best = 1e30f;
    for (int rep = 0; rep < 5; rep++) {
        cudaEventRecord(e0);
        fma_loop<<<blocks, threads>>>(out, iters, 0.999999, 1e-7);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best) best = ms;
    }
    cudaError_t e = cudaGetLastError();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    if (e != cudaSuccess) return BES_ERR_CUDA;
    const double flops = 2.0 * 8 * 16 * (double)iters * threads * blocks;
    *tflops = flops / (best * 1e-3) / 1e12;
    return BES_OK;
}
