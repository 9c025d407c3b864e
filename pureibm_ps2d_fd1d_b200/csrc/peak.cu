// peak.cu -- FP64 arithmetic peak of the device (measurement only; no
// counterpart in the reference).  The FP64 flop fraction of the step is
// reported against this number, which no vendor figure replaces: a grid of
// 8 CTAs of 256 threads per SM runs chains of fused multiply-adds on eight
// independent accumulators per thread, timed with CUDA events.
#include <cuda_runtime.h>

#include "../../include/pibm.h"
#include "step_common.cuh"

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

// Bitwise comparison of qdiv(a, b, 1/b) with the division a / b.
__global__ void k_qdiv_check(const double *a, long long n, const double *b, int nb, unsigned long long *bad) {
    unsigned long long cnt = 0;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n * nb; t += (long long)gridDim.x * blockDim.x) {
        const double x = a[t % n], d = b[t / n];
        const double y = 1.0 / d;
        if (__double_as_longlong(pibm::qdiv(x, d, y)) != __double_as_longlong(x / d)) ++cnt;
    }
    if (cnt) atomicAdd(bad, cnt);
}

}  // namespace

extern "C" int pibm_qdiv_check(const double *a, long long n, const double *b, int nb, long long *mismatches) {
    if (!a || !b || !mismatches || n <= 0 || nb <= 0) return PIBM_ERR_ARG;
    double *da = nullptr, *db = nullptr;
    unsigned long long *dbad = nullptr;
    if (cudaMalloc(&da, (size_t)n * sizeof(double)) != cudaSuccess) return PIBM_ERR_NOMEM;
    if (cudaMalloc(&db, (size_t)nb * sizeof(double)) != cudaSuccess || cudaMalloc(&dbad, sizeof(*dbad)) != cudaSuccess) {
        cudaFree(da);
        cudaFree(db);
        return PIBM_ERR_NOMEM;
    }
    cudaMemcpy(da, a, (size_t)n * sizeof(double), cudaMemcpyHostToDevice);
    cudaMemcpy(db, b, (size_t)nb * sizeof(double), cudaMemcpyHostToDevice);
    cudaMemset(dbad, 0, sizeof(*dbad));
    k_qdiv_check<<<1184, 256>>>(da, n, db, nb, dbad);
    unsigned long long bad = 0;
    cudaMemcpy(&bad, dbad, sizeof(bad), cudaMemcpyDeviceToHost);
    const cudaError_t err = cudaGetLastError();
    cudaFree(da);
    cudaFree(db);
    cudaFree(dbad);
    if (err != cudaSuccess) return PIBM_ERR_CUDA;
    *mismatches = (long long)bad;
    return PIBM_OK;
}

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
