// Learned neighbour budget: a per-cell K proposal beside the reference's fixed
// _K_ (Config.sh; knn::solve, src/knn/knn.cpp:225-315, always returns K
// neighbours and the clip walks them until the security radius closes,
// src/voronoi/voronoi.cpp:129-147).
//
// Each hydro cell gets 8 features from the previous mesh and the new grid:
//   0 log2(1 + certified K of the previous step) / 8
//   1 log2(1 + points in the cell's grid bin) / 4
//   2 refinement level of that bin (dense bins are split into (2^L)^D sub-bins) / 4
//   3 relative volume change over the last step, (V - V_prev) / V, x 4 in [-4, 4]
//     (the cell's velocity divergence times dt)
//   4 log2(V * N) / 4, the cell's volume relative to the mean
//   5 1 if the previous proposal missed (the cell needed the fallback)
//   6 |centroid - generating point| / V^(1/D), clamped to 2
//   7 log2(1 + face count) / 5
// An MLP 8 -> 32 -> 32 -> 6 (GELU) classifies the cell's certified K into the
// classes {12,16,20,24,32,48} (2D) or {32,40,48,64,96,128} (3D); the proposal
// is the smallest class whose cumulative probability reaches the quantile.
// Every proposal is checked by the certificate: a cell that does not certify
// within its K is computed again at the plain budget, so the mesh is the plain
// method's mesh bit for bit.
//
// Training uses the K that the certificate records on plain-method steps
// (mean cross-entropy, Adam on FP32 master weights).  All products run on the
// tensor cores as BF16 x BF16 -> FP32 mma (m16n8k16), one warp per tile of 16
// cells: the forward pass, the input gradients (delta . W) and the weight
// gradients (delta^T . activations, with the 16 cells as the reduction
// dimension).  Per-warp partial gradients are reduced in a fixed order, so a
// training step is deterministic.
#include <cuda_bf16.h>
#include <math_constants.h>

#include <cmath>
#include <vector>

#include "pgpu_common.cuh"
#include "pgpu_ctx.h"

namespace pgpu {
namespace {

constexpr unsigned FULL = 0xffffffffu;
constexpr int KB_THREADS = 128;  // 4 warps per block

__constant__ int c_kclass[2][KB_CLASSES] = {{12, 16, 20, 24, 32, 48}, {32, 40, 48, 64, 96, 128}};

__device__ __forceinline__ uint32_t pack_bf2(float lo, float hi) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t*>(&v);
}
__device__ __forceinline__ uint32_t pack_u16(uint16_t lo, uint16_t hi) { return (uint32_t)lo | ((uint32_t)hi << 16); }
__device__ __forceinline__ uint32_t ld32(const uint16_t* p) { return *reinterpret_cast<const uint32_t*>(p); }
__device__ __forceinline__ void st32(uint16_t* p, uint32_t v) { *reinterpret_cast<uint32_t*>(p) = v; }

// D += A . B, A 16x16 (row), B 16x8 (col), BF16 in, FP32 accumulate.
__device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

__device__ __forceinline__ float gelu(float x) { return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float x) {
    return 0.5f * (1.0f + erff(x * 0.70710678118654752f)) + x * 0.39894228040143268f * expf(-0.5f * x * x);
}

// Weights staged in shared memory by every block: BF16 operands and FP32 biases.
struct __align__(16) MlpSmem {
    uint16_t wb[KB_NBF];
    float b1[KB_HIDDEN], b2[KB_HIDDEN], b3[8];
};

__device__ __forceinline__ void stage_weights(MlpSmem& S, const uint16_t* __restrict__ wbf, const float* __restrict__ w) {
    for (int i = threadIdx.x; i < KB_NBF / 2; i += blockDim.x)
        reinterpret_cast<uint32_t*>(S.wb)[i] = reinterpret_cast<const uint32_t*>(wbf)[i];
    for (int i = threadIdx.x; i < KB_HIDDEN; i += blockDim.x) {
        S.b1[i] = w[KB_B1 + i];
        S.b2[i] = w[KB_B2 + i];
    }
    if (threadIdx.x < 8) S.b3[threadIdx.x] = threadIdx.x < KB_CLASSES ? w[KB_B3 + threadIdx.x] : 0.0f;
    __syncthreads();
}

// Forward pass of one 16-cell tile held as the A fragment ax (features in
// columns 0-7, zero in 8-15).  Keeps the pre-activations for the backward pass.
struct Fwd {
    float z1[4][4], z2[4][4], lg[4];
    uint32_t h1[2][4], h2[2][4];  // BF16 activations as A fragments of the next layer
};

__device__ __forceinline__ void to_afrag(const float (&z)[4][4], uint32_t (&h)[2][4], bool act) {
#pragma unroll
    for (int s = 0; s < 2; s++) {
        float v[2][4];
#pragma unroll
        for (int t = 0; t < 2; t++)
#pragma unroll
            for (int r = 0; r < 4; r++) v[t][r] = act ? gelu(z[2 * s + t][r]) : z[2 * s + t][r];
        h[s][0] = pack_bf2(v[0][0], v[0][1]);
        h[s][1] = pack_bf2(v[0][2], v[0][3]);
        h[s][2] = pack_bf2(v[1][0], v[1][1]);
        h[s][3] = pack_bf2(v[1][2], v[1][3]);
    }
}

__device__ __forceinline__ void mlp_forward(const MlpSmem& S, const uint32_t (&ax)[4], Fwd& f, int g, int q) {
#pragma unroll
    for (int j = 0; j < 4; j++) {
        float d[4] = {S.b1[8 * j + 2 * q], S.b1[8 * j + 2 * q + 1], S.b1[8 * j + 2 * q], S.b1[8 * j + 2 * q + 1]};
        mma_bf16(d, ax, ld32(S.wb + KB_BW1 + (8 * j + g) * 8 + 2 * q), 0u);
#pragma unroll
        for (int r = 0; r < 4; r++) f.z1[j][r] = d[r];
    }
    to_afrag(f.z1, f.h1, true);
#pragma unroll
    for (int j = 0; j < 4; j++) {
        float d[4] = {S.b2[8 * j + 2 * q], S.b2[8 * j + 2 * q + 1], S.b2[8 * j + 2 * q], S.b2[8 * j + 2 * q + 1]};
#pragma unroll
        for (int s = 0; s < 2; s++)
            mma_bf16(d, f.h1[s], ld32(S.wb + KB_BW2 + (8 * j + g) * 32 + 16 * s + 2 * q),
                     ld32(S.wb + KB_BW2 + (8 * j + g) * 32 + 16 * s + 8 + 2 * q));
#pragma unroll
        for (int r = 0; r < 4; r++) f.z2[j][r] = d[r];
    }
    to_afrag(f.z2, f.h2, true);
    float d[4] = {S.b3[2 * q], S.b3[2 * q + 1], S.b3[2 * q], S.b3[2 * q + 1]};
#pragma unroll
    for (int s = 0; s < 2; s++)
        mma_bf16(d, f.h2[s], ld32(S.wb + KB_BW3 + g * 32 + 16 * s + 2 * q),
                 ld32(S.wb + KB_BW3 + g * 32 + 16 * s + 8 + 2 * q));
#pragma unroll
    for (int r = 0; r < 4; r++) f.lg[r] = d[r];
}

// Features of rows r0 = tile*16 + g and r0 + 8 as the A fragment.
__device__ __forceinline__ void load_x(const float* __restrict__ feat, int64_t ra, bool va, int64_t rb, bool vb, int q,
                                       uint32_t (&ax)[4], float2& xa, float2& xb) {
    xa = va ? *reinterpret_cast<const float2*>(feat + ra * KB_FEATURES + 2 * q) : make_float2(0.f, 0.f);
    xb = vb ? *reinterpret_cast<const float2*>(feat + rb * KB_FEATURES + 2 * q) : make_float2(0.f, 0.f);
    ax[0] = pack_bf2(xa.x, xa.y);
    ax[1] = pack_bf2(xb.x, xb.y);
    ax[2] = 0u;
    ax[3] = 0u;
}

__global__ void __launch_bounds__(KB_THREADS)
    k_mlp_infer(const float* __restrict__ feat, int64_t n, const uint16_t* __restrict__ wbf,
                const float* __restrict__ w, int dim_idx, int kcap, float quantile, uint16_t* __restrict__ kq,
                float* __restrict__ logits, unsigned long long* __restrict__ ksum) {
    __shared__ MlpSmem S;
    stage_weights(S, wbf, w);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, g = lane >> 2, q = lane & 3;
    const int64_t ntiles = (n + 15) / 16;
    unsigned long long my_k = 0;
    for (int64_t tile = (int64_t)blockIdx.x * 4 + warp; tile < ntiles; tile += (int64_t)gridDim.x * 4) {
        const int64_t ra = tile * 16 + g, rb = ra + 8;
        uint32_t ax[4];
        float2 xa, xb;
        load_x(feat, ra, ra < n, rb, rb < n, q, ax, xa, xb);
        Fwd f;
        mlp_forward(S, ax, f, g, q);
        // every lane of the quad gathers the 8 logits of rows g and g + 8
        float la[8], lb[8];
#pragma unroll
        for (int src = 0; src < 4; src++) {
            const int sl = (lane & ~3) | src;
            la[2 * src] = __shfl_sync(FULL, f.lg[0], sl);
            la[2 * src + 1] = __shfl_sync(FULL, f.lg[1], sl);
            lb[2 * src] = __shfl_sync(FULL, f.lg[2], sl);
            lb[2 * src + 1] = __shfl_sync(FULL, f.lg[3], sl);
        }
        const int64_t r = q == 0 ? ra : rb;
        if (q < 2 && r < n) {
            float l[KB_CLASSES];
#pragma unroll
            for (int c = 0; c < KB_CLASSES; c++) l[c] = q == 0 ? la[c] : lb[c];
            float m = l[0];
#pragma unroll
            for (int c = 1; c < KB_CLASSES; c++) m = fmaxf(m, l[c]);
            float e[KB_CLASSES], s = 0.0f;
#pragma unroll
            for (int c = 0; c < KB_CLASSES; c++) {
                e[c] = expf(l[c] - m);
                s += e[c];
            }
            // the first class whose cumulative probability reaches the quantile
            const float target = quantile * s;
            int cls = KB_CLASSES - 1;
            float acc = 0.0f;
            bool found = false;
#pragma unroll
            for (int c = 0; c < KB_CLASSES; c++) {
                acc += e[c];
                if (!found && acc >= target) {
                    cls = c;
                    found = true;
                }
            }
            const int K = min(c_kclass[dim_idx][cls], kcap);
            if (kq) kq[r] = (uint16_t)K;
            my_k += (unsigned long long)K;
            if (logits)
#pragma unroll
                for (int c = 0; c < KB_CLASSES; c++) logits[r * KB_CLASSES + c] = l[c];
        }
    }
    for (int o = 16; o > 0; o >>= 1) my_k += __shfl_xor_sync(FULL, my_k, o);
    if (ksum && lane == 0 && my_k) atomicAdd(ksum, my_k);
}

// Per-warp tiles for the backward pass (BF16, row = cell of the tile).
struct __align__(16) GradSmem {
    uint16_t x[16][8], h1[16][32], h2[16][32], d3[16][8], d2[16][32], d1[16][32];
};

// Mean cross-entropy gradient over nb rows.  Row i of the batch is feature row
// (off + i * stride) mod n (stride 0: row i).  Each warp writes one partial row
// of KB_PART floats: the gradient of its tiles and their loss.
__global__ void __launch_bounds__(KB_THREADS)
    k_mlp_grad(const float* __restrict__ feat, const int32_t* __restrict__ labels, int64_t n, int64_t nb, int64_t off,
               int64_t stride, const uint16_t* __restrict__ wbf, const float* __restrict__ w, float inv_b,
               float* __restrict__ part) {
    __shared__ MlpSmem S;
    __shared__ GradSmem G[4];
    stage_weights(S, wbf, w);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, g = lane >> 2, q = lane & 3;
    GradSmem& T = G[warp];
    float acc1[2][4] = {}, acc2[2][4][4] = {}, acc3[4][4] = {};
    float db1[4][2] = {}, db2[4][2] = {}, db3[2] = {};
    float loss = 0.0f;
    const int64_t ntiles = (nb + 15) / 16;
    for (int64_t tile = (int64_t)blockIdx.x * 4 + warp; tile < ntiles; tile += (int64_t)gridDim.x * 4) {
        const int64_t ia = tile * 16 + g, ib = ia + 8;
        const bool va = ia < nb, vb = ib < nb;
        const int64_t ra = stride ? (off + (ia % n) * stride) % n : ia;
        const int64_t rb = stride ? (off + (ib % n) * stride) % n : ib;
        uint32_t ax[4];
        float2 xa, xb;
        load_x(feat, ra, va, rb, vb, q, ax, xa, xb);
        const int ya = va ? labels[ra] : -1, yb = vb ? labels[rb] : -1;
        Fwd f;
        mlp_forward(S, ax, f, g, q);
        st32(&T.x[g][2 * q], ax[0]);
        st32(&T.x[g + 8][2 * q], ax[1]);
#pragma unroll
        for (int s = 0; s < 2; s++) {
            st32(&T.h1[g][16 * s + 2 * q], f.h1[s][0]);
            st32(&T.h1[g + 8][16 * s + 2 * q], f.h1[s][1]);
            st32(&T.h1[g][16 * s + 8 + 2 * q], f.h1[s][2]);
            st32(&T.h1[g + 8][16 * s + 8 + 2 * q], f.h1[s][3]);
            st32(&T.h2[g][16 * s + 2 * q], f.h2[s][0]);
            st32(&T.h2[g + 8][16 * s + 2 * q], f.h2[s][1]);
            st32(&T.h2[g][16 * s + 8 + 2 * q], f.h2[s][2]);
            st32(&T.h2[g + 8][16 * s + 8 + 2 * q], f.h2[s][3]);
        }
        // softmax over the 6 classes of each row (columns 6, 7 are padding)
        float d3[4];
#pragma unroll
        for (int half = 0; half < 2; half++) {
            const float l0 = f.lg[2 * half], l1 = f.lg[2 * half + 1];
            const bool c0ok = 2 * q < KB_CLASSES, c1ok = 2 * q + 1 < KB_CLASSES;
            float m = fmaxf(c0ok ? l0 : -CUDART_INF_F, c1ok ? l1 : -CUDART_INF_F);
            m = fmaxf(m, __shfl_xor_sync(FULL, m, 1));
            m = fmaxf(m, __shfl_xor_sync(FULL, m, 2));
            const float e0 = c0ok ? expf(l0 - m) : 0.0f, e1 = c1ok ? expf(l1 - m) : 0.0f;
            float s = e0 + e1;
            s += __shfl_xor_sync(FULL, s, 1);
            s += __shfl_xor_sync(FULL, s, 2);
            const int y = half ? yb : ya;
            const bool valid = half ? vb : va;
            const float scale = valid ? inv_b : 0.0f;
            d3[2 * half] = (e0 / s - (y == 2 * q ? 1.0f : 0.0f)) * scale;
            d3[2 * half + 1] = (e1 / s - (y == 2 * q + 1 ? 1.0f : 0.0f)) * scale;
            if (!c0ok) d3[2 * half] = 0.0f;
            if (!c1ok) d3[2 * half + 1] = 0.0f;
            if (valid && y == 2 * q) loss += -(l0 - m - logf(s));
            if (valid && y == 2 * q + 1) loss += -(l1 - m - logf(s));
        }
        db3[0] += d3[0] + d3[2];
        db3[1] += d3[1] + d3[3];
        const uint32_t d3a = pack_bf2(d3[0], d3[1]), d3b = pack_bf2(d3[2], d3[3]);
        st32(&T.d3[g][2 * q], d3a);
        st32(&T.d3[g + 8][2 * q], d3b);
        __syncwarp();
        // dW3 += d3^T . h2   (M = class, padded to 16; N = hidden; K = cells)
        {
            const uint32_t a[4] = {pack_u16(T.d3[2 * q][g], T.d3[2 * q + 1][g]), 0u,
                                   pack_u16(T.d3[8 + 2 * q][g], T.d3[9 + 2 * q][g]), 0u};
#pragma unroll
            for (int j = 0; j < 4; j++)
                mma_bf16(acc3[j], a, pack_u16(T.h2[2 * q][8 * j + g], T.h2[2 * q + 1][8 * j + g]),
                         pack_u16(T.h2[8 + 2 * q][8 * j + g], T.h2[9 + 2 * q][8 * j + g]));
        }
        // d2 = (d3 . W3) * gelu'(z2)
        float d2[4][4];
        {
            const uint32_t a[4] = {d3a, d3b, 0u, 0u};
#pragma unroll
            for (int j = 0; j < 4; j++) {
                float d[4] = {0.f, 0.f, 0.f, 0.f};
                mma_bf16(d, a, ld32(S.wb + KB_BW3T + (8 * j + g) * 8 + 2 * q), 0u);
#pragma unroll
                for (int r = 0; r < 4; r++) d2[j][r] = d[r] * gelu_grad(f.z2[j][r]);
                db2[j][0] += d2[j][0] + d2[j][2];
                db2[j][1] += d2[j][1] + d2[j][3];
                st32(&T.d2[g][8 * j + 2 * q], pack_bf2(d2[j][0], d2[j][1]));
                st32(&T.d2[g + 8][8 * j + 2 * q], pack_bf2(d2[j][2], d2[j][3]));
            }
        }
        __syncwarp();
        // dW2 += d2^T . h1
#pragma unroll
        for (int mt = 0; mt < 2; mt++) {
            const int o = 16 * mt + g;
            const uint32_t a[4] = {pack_u16(T.d2[2 * q][o], T.d2[2 * q + 1][o]),
                                   pack_u16(T.d2[2 * q][o + 8], T.d2[2 * q + 1][o + 8]),
                                   pack_u16(T.d2[8 + 2 * q][o], T.d2[9 + 2 * q][o]),
                                   pack_u16(T.d2[8 + 2 * q][o + 8], T.d2[9 + 2 * q][o + 8])};
#pragma unroll
            for (int j = 0; j < 4; j++)
                mma_bf16(acc2[mt][j], a, pack_u16(T.h1[2 * q][8 * j + g], T.h1[2 * q + 1][8 * j + g]),
                         pack_u16(T.h1[8 + 2 * q][8 * j + g], T.h1[9 + 2 * q][8 * j + g]));
        }
        // d1 = (d2 . W2) * gelu'(z1)
        {
            uint32_t a2[2][4];
            to_afrag(d2, a2, false);
#pragma unroll
            for (int j = 0; j < 4; j++) {
                float d[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
                for (int s = 0; s < 2; s++)
                    mma_bf16(d, a2[s], ld32(S.wb + KB_BW2T + (8 * j + g) * 32 + 16 * s + 2 * q),
                             ld32(S.wb + KB_BW2T + (8 * j + g) * 32 + 16 * s + 8 + 2 * q));
                float d1[4];
#pragma unroll
                for (int r = 0; r < 4; r++) d1[r] = d[r] * gelu_grad(f.z1[j][r]);
                db1[j][0] += d1[0] + d1[2];
                db1[j][1] += d1[1] + d1[3];
                st32(&T.d1[g][8 * j + 2 * q], pack_bf2(d1[0], d1[1]));
                st32(&T.d1[g + 8][8 * j + 2 * q], pack_bf2(d1[2], d1[3]));
            }
        }
        __syncwarp();
        // dW1 += d1^T . x
#pragma unroll
        for (int mt = 0; mt < 2; mt++) {
            const int o = 16 * mt + g;
            const uint32_t a[4] = {pack_u16(T.d1[2 * q][o], T.d1[2 * q + 1][o]),
                                   pack_u16(T.d1[2 * q][o + 8], T.d1[2 * q + 1][o + 8]),
                                   pack_u16(T.d1[8 + 2 * q][o], T.d1[9 + 2 * q][o]),
                                   pack_u16(T.d1[8 + 2 * q][o + 8], T.d1[9 + 2 * q][o + 8])};
            mma_bf16(acc1[mt], a, pack_u16(T.x[2 * q][g], T.x[2 * q + 1][g]),
                     pack_u16(T.x[8 + 2 * q][g], T.x[9 + 2 * q][g]));
        }
        __syncwarp();
    }
    // bias gradients: sum over the 8 row groups (lanes with the same q)
#pragma unroll
    for (int o = 4; o < 32; o <<= 1) {
#pragma unroll
        for (int j = 0; j < 4; j++)
#pragma unroll
            for (int r = 0; r < 2; r++) {
                db1[j][r] += __shfl_xor_sync(FULL, db1[j][r], o);
                db2[j][r] += __shfl_xor_sync(FULL, db2[j][r], o);
            }
        db3[0] += __shfl_xor_sync(FULL, db3[0], o);
        db3[1] += __shfl_xor_sync(FULL, db3[1], o);
    }
    for (int o = 16; o > 0; o >>= 1) loss += __shfl_xor_sync(FULL, loss, o);
    float* row = part + ((int64_t)blockIdx.x * 4 + warp) * KB_PART;
#pragma unroll
    for (int mt = 0; mt < 2; mt++)
#pragma unroll
        for (int r = 0; r < 4; r++) {
            const int o = 16 * mt + g + (r >= 2 ? 8 : 0);
            row[KB_W1 + o * 8 + 2 * q + (r & 1)] = acc1[mt][r];
#pragma unroll
            for (int j = 0; j < 4; j++) row[KB_W2 + o * 32 + 8 * j + 2 * q + (r & 1)] = acc2[mt][j][r];
        }
    if (g < KB_CLASSES)
#pragma unroll
        for (int j = 0; j < 4; j++)
#pragma unroll
            for (int r = 0; r < 2; r++) row[KB_W3 + g * 32 + 8 * j + 2 * q + r] = acc3[j][r];
    if (g == 0) {
#pragma unroll
        for (int j = 0; j < 4; j++)
#pragma unroll
            for (int r = 0; r < 2; r++) {
                row[KB_B1 + 8 * j + 2 * q + r] = db1[j][r];
                row[KB_B2 + 8 * j + 2 * q + r] = db2[j][r];
            }
#pragma unroll
        for (int r = 0; r < 2; r++)
            if (2 * q + r < KB_CLASSES) row[KB_B3 + 2 * q + r] = db3[r];
    }
    if (lane == 0) row[KB_NPARAM] = loss * inv_b;
}

__device__ __forceinline__ uint16_t bf16_bits(float x) { return __bfloat16_as_ushort(__float2bfloat16_rn(x)); }

// BF16 copies of master parameter p (W1, W2 and W2^T, W3 and W3^T).
__device__ __forceinline__ void write_bf16(int p, float v, uint16_t* __restrict__ wbf) {
    const uint16_t b = bf16_bits(v);
    if (p < KB_B1) {
        wbf[KB_BW1 + p] = b;
    } else if (p >= KB_W2 && p < KB_B2) {
        const int o = (p - KB_W2) / 32, i = (p - KB_W2) % 32;
        wbf[KB_BW2 + o * 32 + i] = b;
        wbf[KB_BW2T + i * 32 + o] = b;
    } else if (p >= KB_W3 && p < KB_B3) {
        const int c = (p - KB_W3) / 32, k = (p - KB_W3) % 32;
        wbf[KB_BW3 + c * 32 + k] = b;
        wbf[KB_BW3T + k * 8 + c] = b;
    }
}

// Sums the per-warp partials in a fixed order; optionally applies one Adam step.
__global__ void k_mlp_reduce(const float* __restrict__ part, int nparts, float* __restrict__ w, float* __restrict__ m,
                             float* __restrict__ v, float* __restrict__ gout, int update, float lr, float c1, float c2,
                             uint16_t* __restrict__ wbf) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p > KB_NPARAM) return;
    float s = 0.0f;
    for (int i = 0; i < nparts; i++) s += part[(int64_t)i * KB_PART + p];
    if (gout) gout[p] = s;
    if (p == KB_NPARAM || !update) return;
    const float mm = 0.9f * m[p] + 0.1f * s;
    const float vv = 0.999f * v[p] + 0.001f * s * s;
    m[p] = mm;
    v[p] = vv;
    const float wn = w[p] - lr * (mm / c1) / (sqrtf(vv / c2) + 1e-8f);
    w[p] = wn;
    write_bf16(p, wn, wbf);
}

__global__ void k_mlp_bf16_all(const float* __restrict__ w, uint16_t* __restrict__ wbf) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < KB_NPARAM) write_bf16(p, w[p], wbf);
}

// Features of each query slot's cell.  BY_ID: one thread per hydro cell in hydro-id
// order (every query is a hydro cell), so that the per-cell arrays indexed by id are read
// in order and only the sorted position, its query slot and the feature row are
// scattered; else one thread per query slot.  The values are the same either way.
template <int D, bool BY_ID>
__global__ void k_kb_features(const uint32_t* __restrict__ qs, const uint32_t* __restrict__ perm,
                              const uint32_t* __restrict__ inv, const uint32_t* __restrict__ qoff,
                              const typename PointOf<D>::type* __restrict__ spts, const uint32_t* __restrict__ bin_start,
                              const uint8_t* __restrict__ lvl, const InstPar* __restrict__ ip, const uint16_t* __restrict__ inst, int64_t nq,
                              int64_t n_hydro, const int* __restrict__ certk,
                              const double* __restrict__ vol, const uint32_t* __restrict__ fcnt,
                              const double* __restrict__ centroid, const double* __restrict__ pos,
                              float* __restrict__ hist_vol, uint8_t* __restrict__ miss, float* __restrict__ feat) {
    const int64_t u = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= (BY_ID ? n_hydro : nq)) return;
    uint32_t s, e;
    int64_t t;
    if (BY_ID) {
        e = (uint32_t)u;
        s = inv[e];
        t = qoff ? (int64_t)qoff[s] : (int64_t)s;
    } else {
        t = u;
        s = qs[t];
        e = perm[s];
    }
    float f[KB_FEATURES] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    if (e < (uint32_t)n_hydro) {
        const typename PointOf<D>::type p = spts[s];
        const InstPar& par = ip[inst[e]];
        const int G = par.G;
        const int bx = bin_coord(p.x, G), by = bin_coord(p.y, G), bz = D == 3 ? bin_coord(pz(p), G) : 0;
        const uint32_t own = par.slot0 + morton<D>(bx, by, bz);
        const uint32_t occ = bin_start[own + 1] - bin_start[own];
        const double V = vol[e];
        const float Vp = hist_vol[e];
        hist_vol[e] = (float)V;
        f[0] = log2f(1.0f + (float)certk[e]) * 0.125f;
        f[1] = log2f(1.0f + (float)occ) * 0.25f;
        f[2] = 0.25f * (float)lvl[own];
        f[3] = (Vp > 0.0f && V > 0.0) ? 4.0f * fminf(fmaxf((float)((V - (double)Vp) / V), -1.0f), 1.0f) : 0.0f;
        f[4] = V > 0.0 ? 0.25f * log2f((float)(V * (double)par.count)) : -2.0f;
        f[5] = miss[e] ? 1.0f : 0.0f;
        miss[e] = 0;
        if (V > 0.0) {
            double d2 = 0.0;
#pragma unroll
            for (int a = 0; a < D; a++) {
                const double dd = centroid[3 * (int64_t)e + a] - pos[(int64_t)e * D + a];
                d2 += dd * dd;
            }
            const double R = D == 2 ? sqrt(V) : cbrt(V);
            f[6] = fminf((float)(sqrt(d2) / R), 2.0f);
        }
        f[7] = log2f(1.0f + (float)fcnt[e]) * 0.2f;
    }
    float4* out = reinterpret_cast<float4*>(feat + t * KB_FEATURES);
    out[0] = make_float4(f[0], f[1], f[2], f[3]);
    out[1] = make_float4(f[4], f[5], f[6], f[7]);
}

// Class of each query slot's certified K: the smallest class K >= certk
// (uncertified cells, certk 0, and certk above every class: the last class).
__global__ void k_kb_labels(const uint32_t* __restrict__ qs, const uint32_t* __restrict__ perm,
                            const int* __restrict__ certk, int64_t nq, int dim_idx, int32_t* __restrict__ labels) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nq) return;
    const int ck = certk[perm[qs[t]]];
    int cls = KB_CLASSES - 1;
    if (ck > 0)
        for (int c = KB_CLASSES - 1; c >= 0; c--)
            if (c_kclass[dim_idx][c] >= ck) cls = c;
    labels[t] = cls;
}

__global__ void k_kb_mark(const uint32_t* __restrict__ sorted_pos, const uint32_t* __restrict__ perm, int64_t n,
                          uint8_t* __restrict__ miss) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) miss[perm[sorted_pos[i]]] = 1;
}

inline unsigned nblk(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

uint64_t splitmix(uint64_t& s) {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

}  // namespace

int kb_class_k(int dim, int cls) {
    static const int k[2][KB_CLASSES] = {{12, 16, 20, 24, 32, 48}, {32, 40, 48, 64, 96, 128}};
    return k[dim == 3 ? 1 : 0][cls];
}

// Xavier-uniform weights from the seed, zero biases and Adam moments.
cudaError_t kb_init_weights(pgpu_ctx* c) {
    KBudget& kb = c->kb;
    cudaError_t e = cudaSuccess;
    float* w = ensure<float>(kb.w, KB_NPARAM + 2, &e);
    float* m = ensure<float>(kb.adam_m, KB_NPARAM + 2, &e);
    float* v = ensure<float>(kb.adam_v, KB_NPARAM + 2, &e);
    uint16_t* wb = ensure<uint16_t>(kb.wbf, KB_NBF, &e);
    if (e) return e;
    std::vector<float> h(KB_NPARAM, 0.0f);
    uint64_t s = kb.seed;
    auto fill = [&](int at, int fan_out, int fan_in) {
        const double a = std::sqrt(6.0 / (double)(fan_in + fan_out));
        for (int i = 0; i < fan_out * fan_in; i++) {
            const double u = (double)(splitmix(s) >> 11) * (1.0 / 9007199254740992.0);
            h[at + i] = (float)((2.0 * u - 1.0) * a);
        }
    };
    fill(KB_W1, KB_HIDDEN, KB_FEATURES);
    fill(KB_W2, KB_HIDDEN, KB_HIDDEN);
    fill(KB_W3, KB_CLASSES, KB_HIDDEN);
    if ((e = cudaMemcpyAsync(w, h.data(), KB_NPARAM * sizeof(float), cudaMemcpyHostToDevice, c->stream))) return e;
    if ((e = cudaMemsetAsync(m, 0, KB_NPARAM * sizeof(float), c->stream))) return e;
    if ((e = cudaMemsetAsync(v, 0, KB_NPARAM * sizeof(float), c->stream))) return e;
    if ((e = cudaMemsetAsync(wb, 0, KB_NBF * sizeof(uint16_t), c->stream))) return e;
    k_mlp_bf16_all<<<nblk(KB_NPARAM, 256), 256, 0, c->stream>>>(w, wb);
    count_launches(1);
    kb.adam_t = 0;
    return cudaGetLastError();
}

cudaError_t kb_sync_bf16(pgpu_ctx* c) {
    k_mlp_bf16_all<<<nblk(KB_NPARAM, 256), 256, 0, c->stream>>>((const float*)c->kb.w.p, (uint16_t*)c->kb.wbf.p);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t kb_features(pgpu_ctx* c) {
    KBudget& kb = c->kb;
    cudaError_t e = cudaSuccess;
    const int64_t nq = c->n_query, nh = c->n_hydro;
    float* feat = ensure<float>(kb.feat, (size_t)nq * KB_FEATURES + 8, &e);
    const size_t hv_before = kb.hist_vol.bytes;
    float* hv = ensure<float>(kb.hist_vol, nh + 1, &e);
    const size_t ms_before = kb.miss.bytes;
    uint8_t* ms = ensure<uint8_t>(kb.miss, nh + 1, &e);
    if (e) return e;
    // first use (or growth, which does not keep contents): no history yet
    if (kb.hist_vol.bytes != hv_before && (e = cudaMemsetAsync(hv, 0, (nh + 1) * sizeof(float), c->stream))) return e;
    if (kb.miss.bytes != ms_before && (e = cudaMemsetAsync(ms, 0, nh + 1, c->stream))) return e;
    if (nq == 0) return cudaSuccess;
    // every query a hydro cell: walk the cells in id order (query slot = the sorted position
    // when every point is a query, else its rank among the hydro points)
    const bool by_id = nq == nh;
    const uint32_t* qoff = (c->all_cells || c->n_ext == nh) ? nullptr : (const uint32_t*)c->qoff.p;
    const unsigned blocks = nblk(by_id ? nh : nq, 256);
#define PGPU_KBF(DD, PT, BI)                                                                                  \
    k_kb_features<DD, BI><<<blocks, 256, 0, c->stream>>>(                                                     \
        (const uint32_t*)c->qs.p, (const uint32_t*)c->perm.p, (const uint32_t*)c->inv.p, qoff,               \
        (const PT*)c->spts.p, (const uint32_t*)c->bin_start.p, (const uint8_t*)c->bin_lvl.p,                 \
        (const InstPar*)c->inst.d_par.p, (const uint16_t*)c->inst.d_inst_e.p, nq, nh, (const int*)c->certk.p, \
        (const double*)c->vol.p, (const uint32_t*)c->fcnt.p, (const double*)c->centroid.p,                  \
        (const double*)c->pos.p, hv, ms, feat)
    if (c->prm.dim == 2) {
        if (by_id) PGPU_KBF(2, double2, true); else PGPU_KBF(2, double2, false);
    } else {
        if (by_id) PGPU_KBF(3, double4, true); else PGPU_KBF(3, double4, false);
    }
#undef PGPU_KBF
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t kb_infer(pgpu_ctx* c, const float* feat, int64_t n, uint16_t* kq, float* logits) {
    KBudget& kb = c->kb;
    cudaError_t e = cudaSuccess;
    unsigned long long* ks = ensure<unsigned long long>(kb.ksum, 1, &e);
    if (e) return e;
    if ((e = cudaMemsetAsync(ks, 0, sizeof(unsigned long long), c->stream))) return e;
    if (n <= 0) return cudaSuccess;
    const int64_t tiles = (n + 15) / 16;
    int blocks = (int)std::min<int64_t>((tiles + 3) / 4, 148 * 16);
    k_mlp_infer<<<blocks, KB_THREADS, 0, c->stream>>>(feat, n, (const uint16_t*)kb.wbf.p, (const float*)kb.w.p,
                                                      c->prm.dim == 3 ? 1 : 0, c->prm.k, kb.quantile, kq, logits, ks);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t kb_grad(pgpu_ctx* c, const float* feat, const int32_t* labels, int64_t n, const uint32_t* /*sample*/,
                    int64_t nb, bool update) {
    KBudget& kb = c->kb;
    cudaError_t e = cudaSuccess;
    const int nparts = KB_GRAD_BLOCKS * KB_GRAD_WARPS;
    float* part = ensure<float>(kb.part, (size_t)nparts * KB_PART, &e);
    float* gout = ensure<float>(kb.tmp_out, KB_PART, &e);
    if (e) return e;
    if (nb <= 0 || n <= 0) return cudaSuccess;
    int64_t off = 0, stride = 0;
    if (nb < n || update) {
        // a pseudo-random subset: rows off + i * stride (mod n), stride a prime not dividing n
        uint64_t s = kb.seed ^ (0x632BE59BD9B4E019ull * (uint64_t)(kb.adam_t + 1));
        off = (int64_t)(splitmix(s) % (uint64_t)n);
        const int64_t primes[3] = {1000003, 999983, 999979};
        stride = primes[0];
        for (int i = 0; i < 3; i++)
            if (n % primes[i] != 0) {
                stride = primes[i] % n;
                break;
            }
        if (stride == 0) stride = 1;
    }
    k_mlp_grad<<<KB_GRAD_BLOCKS, KB_THREADS, 0, c->stream>>>(feat, labels, n, nb, off, stride,
                                                           (const uint16_t*)kb.wbf.p, (const float*)kb.w.p,
                                                           1.0f / (float)nb, part);
    float c1 = 1.0f, c2 = 1.0f;
    if (update) {
        kb.adam_t++;
        c1 = 1.0f - std::pow(0.9f, (float)kb.adam_t);
        c2 = 1.0f - std::pow(0.999f, (float)kb.adam_t);
    }
    k_mlp_reduce<<<nblk(KB_NPARAM + 1, 256), 256, 0, c->stream>>>(part, nparts, (float*)kb.w.p,
                                                                  (float*)kb.adam_m.p, (float*)kb.adam_v.p, gout,
                                                                  update ? 1 : 0, kb.lr, c1, c2, (uint16_t*)kb.wbf.p);
    count_launches(2);
    return cudaGetLastError();
}

cudaError_t kb_train_step(pgpu_ctx* c) {
    KBudget& kb = c->kb;
    cudaError_t e = cudaSuccess;
    const int64_t nq = c->n_query;
    int32_t* lab = ensure<int32_t>(kb.labels, nq + 1, &e);
    if (e) return e;
    if (nq == 0) return cudaSuccess;
    k_kb_labels<<<nblk(nq, 256), 256, 0, c->stream>>>((const uint32_t*)c->qs.p, (const uint32_t*)c->perm.p,
                                                      (const int*)c->certk.p, nq, c->prm.dim == 3 ? 1 : 0, lab);
    count_launches(1);
    const int64_t nb = std::min<int64_t>(kb.batch, nq);
    for (int it = 0; it < kb.iters; it++)
        if ((e = kb_grad(c, (const float*)kb.feat.p, lab, nq, nullptr, nb, true))) return e;
    float loss = 0.0f;
    if ((e = cudaMemcpyAsync(&loss, (float*)kb.tmp_out.p + KB_NPARAM, sizeof(float), cudaMemcpyDeviceToHost,
                             c->stream)))
        return e;
    if ((e = cudaStreamSynchronize(c->stream))) return e;
    kb.last_loss = loss;
    return cudaSuccess;
}

cudaError_t kb_mark_miss(pgpu_ctx* c, const uint32_t* sorted_pos, int64_t n) {
    if (n <= 0) return cudaSuccess;
    k_kb_mark<<<nblk(n, 256), 256, 0, c->stream>>>(sorted_pos, (const uint32_t*)c->perm.p, n, (uint8_t*)c->kb.miss.p);
    count_launches(1);
    return cudaGetLastError();
}

}  // namespace pgpu
