// Exclusive prefix sum of uint32 counts (reduce, scan the block sums, rescan).
// Used for ghost offsets, grid bin starts and the query list.  out[n] receives
// the total.  Deterministic: integer adds in a fixed tree.
#include "pgpu_ctx.h"

namespace pgpu {
namespace {

constexpr int SCAN_THREADS = 512;
constexpr int SCAN_ITEMS = 8;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;

__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += t;
    }
    return v;
}

// Block-wide exclusive scan of one value per thread; returns the exclusive
// prefix and writes the block total to *total.
__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t* total) {
    __shared__ uint32_t warp_sums[SCAN_THREADS / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint32_t inc = warp_incl_scan(v);
    if (lane == 31) warp_sums[wid] = inc;
    __syncthreads();
    if (wid == 0) {
        uint32_t w = lane < SCAN_THREADS / 32 ? warp_sums[lane] : 0;
        uint32_t wi = warp_incl_scan(w);
        if (lane < SCAN_THREADS / 32) warp_sums[lane] = wi - w;
        if (lane == 31) *total = wi;
    }
    __syncthreads();
    uint32_t r = inc - v + warp_sums[wid];
    __syncthreads();
    return r;
}

__global__ void k_block_sums(const uint32_t* __restrict__ in, int64_t n, uint32_t* __restrict__ sums) {
    const int64_t base = (int64_t)blockIdx.x * SCAN_TILE;
    uint32_t s = 0;
    for (int i = 0; i < SCAN_ITEMS; i++) {
        int64_t idx = base + (int64_t)i * SCAN_THREADS + threadIdx.x;
        if (idx < n) s += in[idx];
    }
    __shared__ uint32_t tot;
    block_excl_scan(s, &tot);
    if (threadIdx.x == 0) sums[blockIdx.x] = tot;
}

// Single block: exclusive scan of nb block sums in place; sums[nb] = total.
__global__ void k_scan_sums(uint32_t* sums, int64_t nb) {
    const int64_t per = (nb + SCAN_THREADS - 1) / SCAN_THREADS;
    const int64_t lo = threadIdx.x * per, hi = lo + per < nb ? lo + per : nb;
    uint32_t s = 0;
    for (int64_t i = lo; i < hi; i++) s += sums[i];
    __shared__ uint32_t tot;
    uint32_t run = block_excl_scan(s, &tot);
    for (int64_t i = lo; i < hi; i++) {
        uint32_t v = sums[i];
        sums[i] = run;
        run += v;
    }
    if (threadIdx.x == 0) sums[nb] = tot;
}

__global__ void k_rescan(const uint32_t* __restrict__ in, int64_t n, const uint32_t* __restrict__ sums,
                         uint32_t* __restrict__ out) {
    const int64_t base = (int64_t)blockIdx.x * SCAN_TILE + (int64_t)threadIdx.x * SCAN_ITEMS;
    uint32_t v[SCAN_ITEMS];
    uint32_t s = 0;
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; i++) {
        int64_t idx = base + i;
        v[i] = idx < n ? in[idx] : 0;
        s += v[i];
    }
    __shared__ uint32_t tot;
    uint32_t run = block_excl_scan(s, &tot) + sums[blockIdx.x];
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; i++) {
        int64_t idx = base + i;
        if (idx < n) out[idx] = run;
        run += v[i];
    }
    if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) out[n] = sums[gridDim.x];
}

}  // namespace

cudaError_t exclusive_scan_u32(const uint32_t* in, uint32_t* out, int64_t n, DevBuf& tmp, cudaStream_t s) {
    if (n <= 0) {
        return cudaMemsetAsync(out, 0, sizeof(uint32_t), s);
    }
    const int64_t nb = (n + SCAN_TILE - 1) / SCAN_TILE;
    cudaError_t e = cudaSuccess;
    uint32_t* sums = ensure<uint32_t>(tmp, nb + 1, &e);
    if (e != cudaSuccess) return e;
    k_block_sums<<<(unsigned)nb, SCAN_THREADS, 0, s>>>(in, n, sums);
    k_scan_sums<<<1, SCAN_THREADS, 0, s>>>(sums, nb);
    k_rescan<<<(unsigned)nb, SCAN_THREADS, 0, s>>>(in, n, sums, out);
    count_launches(3);
    return cudaGetLastError();
}

}  // namespace pgpu
