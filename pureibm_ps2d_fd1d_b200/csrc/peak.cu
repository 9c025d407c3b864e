// peak.cu -- FP64 arithmetic peak of the device (measurement only; no
// counterpart in the reference).  The FP64 flop fraction of the step is
// reported against this number, which no vendor figure replaces: a grid of
// 8 CTAs of 256 threads per SM runs chains of fused multiply-adds on eight
// independent accumulators per thread, timed with CUDA events.
#include <cuda_runtime.h>

#include "../../include/pibm.h"

namespace {

__global__ void __launch_bounds__(256) k_dfma_chain(double *out, int iters, double m, double c) {
    double a[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) a[k] = 1e-3 * (double)(threadIdx.x + k);
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < 8; ++k) a[k] = fma(a[k], m, c);
    }
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < 8; ++k) s += a[k];
    if (s == 12345.678) out[blockIdx.x * blockDim.x + threadIdx.x] = s;   // keeps the chains live
}

}  // namespace

extern "C" int pibm_fp64_peak(double *tflops, double *ms_out) {
    if (!tflops) return PIBM_ERR_ARG;
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return PIBM_ERR_CUDA;
    const int blocks = sms * 8, threads = 256, iters = 1 << 13;
    double *out = nullptr;
    if (cudaMalloc(&out, (size_t)blocks * threads * sizeof(double)) != cudaSuccess) return PIBM_ERR_NOMEM;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    k_dfma_chain<<<blocks, threads>>>(out, iters / 16, 1.0000001, 1e-9);   // warm-up
    float best = 1e30f;
    for (int rep = 0; rep < 5; ++rep) {
        cudaEventRecord(e0);
        k_dfma_chain<<<blocks, threads>>>(out, iters, 1.0000001, 1e-9);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best) best = ms;
    }
    const cudaError_t err = cudaGetLastError();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    if (err != cudaSuccess) return PIBM_ERR_CUDA;
    const double flops = 2.0 * 8.0 * (double)iters * (double)blocks * (double)threads;
    *tflops = flops / ((double)best * 1e-3) / 1e12;
    if (ms_out) *ms_out = best;
    return PIBM_OK;
}
