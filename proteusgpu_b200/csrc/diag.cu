// Diagnostics with no reference counterpart: the FP64 FMA rate of the device,
// the denominator of the FP64-pipe roofline of the KNN and clipping kernels.
#include <cuda_runtime.h>

#include "pgpu_ctx.h"

namespace {

constexpr int CHAINS = 8;  // independent FMA chains per thread hide the pipe latency

__global__ void k_fp64_fma(double* __restrict__ sink, int iters, double a, double b) {
    double x[CHAINS];
#pragma unroll
    for (int c = 0; c < CHAINS; c++) x[c] = (threadIdx.x + c) * 1e-7;
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int c = 0; c < CHAINS; c++) x[c] = fma(x[c], a, b);
    }
    double s = 0;
#pragma unroll
    for (int c = 0; c < CHAINS; c++) s += x[c];
    if (s == 1234.5678) sink[threadIdx.x] = s;  // never true; keeps the chains alive
}

}  // namespace

extern "C" int pgpu_fp64_peak(int device, float ms, double* tflops) {
    if (!tflops || ms <= 0) return PGPU_EINVAL;
    if (cudaSetDevice(device) != cudaSuccess) return PGPU_ECUDA;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return PGPU_ECUDA;
    double* sink = nullptr;
    if (cudaMalloc(&sink, 1024 * sizeof(double)) != cudaSuccess) return PGPU_ECUDA;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const int threads = 256, blocks = prop.multiProcessorCount * 8;
    int iters = 1 << 12;
    float t = 0;
    for (int rep = 0; rep < 12; rep++) {  // grow the loop until one launch lasts about `ms`
        cudaEventRecord(e0);
        k_fp64_fma<<<blocks, threads>>>(sink, iters, 0.999999, 1e-9);
        pgpu::count_launches(1);
        cudaEventRecord(e1);
        if (cudaEventSynchronize(e1) != cudaSuccess) break;
        cudaEventElapsedTime(&t, e0, e1);
        if (t >= ms) break;
        iters = (int)(iters * (t > 0.05f ? (ms / t) * 1.1f : 8.0f));
        if (iters > (1 << 28)) iters = 1 << 28;
    }
    const double flops = 2.0 * CHAINS * (double)iters * threads * blocks;
    *tflops = t > 0 ? flops / (t * 1e-3) / 1e12 : 0.0;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(sink);
    return cudaGetLastError() == cudaSuccess ? PGPU_OK : PGPU_ECUDA;
}
