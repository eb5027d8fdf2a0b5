// Diagnostics with no reference counterpart: the FP64 and FP32 FMA rates of the
// device, the denominators of the pipe rooflines of the KNN and clipping kernels.
#include <cuda_runtime.h>

#include "pgpu_ctx.h"

namespace {

constexpr int CHAINS = 8;  // independent FMA chains per thread hide the pipe latency

template <class T>
__global__ void k_fma(T* __restrict__ sink, int iters, T a, T b) {
    T x[CHAINS];
#pragma unroll
    for (int c = 0; c < CHAINS; c++) x[c] = (T)((threadIdx.x + c) * 1e-7);
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int c = 0; c < CHAINS; c++) x[c] = fma(x[c], a, b);
    }
    T s = 0;
#pragma unroll
    for (int c = 0; c < CHAINS; c++) s += x[c];
    if (s == (T)1234.5678) sink[threadIdx.x] = s;  // never true; keeps the chains alive
}

template <class T>
int fma_peak(int device, float ms, double* tflops) {
    if (!tflops || ms <= 0) return PGPU_EINVAL;
    if (cudaSetDevice(device) != cudaSuccess) return PGPU_ECUDA;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return PGPU_ECUDA;
    T* sink = nullptr;
    if (cudaMalloc(&sink, 1024 * sizeof(T)) != cudaSuccess) return PGPU_ECUDA;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const int threads = 256, blocks = prop.multiProcessorCount * 8;
    int iters = 1 << 12;
    float t = 0;
    for (int rep = 0; rep < 12; rep++) {  // grow the loop until one launch lasts about `ms`
        cudaEventRecord(e0);
        k_fma<T><<<blocks, threads>>>(sink, iters, (T)0.999999, (T)1e-9);
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

}  // namespace

extern "C" int pgpu_fp64_peak(int device, float ms, double* tflops) { return fma_peak<double>(device, ms, tflops); }

extern "C" int pgpu_fp32_peak(int device, float ms, double* tflops) { return fma_peak<float>(device, ms, tflops); }
