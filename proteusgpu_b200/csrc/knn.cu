// Exact K nearest neighbours on the Morton-ordered grid (replaces
// knn::solve / cpu_knearest, src/knn/knn.cpp:225-315).
//
// One warp per query point.  Bins are visited in Chebyshev rings around the
// query's bin (as the reference's ring-sorted offset table does), each ring's
// bins expanded 32 at a time into a flat candidate range by a warp prefix sum,
// so that every lane evaluates one candidate per iteration whatever the bin
// occupancy.  A bin is skipped once the list is full and its box lies farther
// than the current K-th neighbour; the search stops when the K-th neighbour is
// closer than everything outside the rings visited so far.
//
// The K best are kept ascending in R registers per lane (element r*32 + lane).
// Candidates that beat the current K-th best are queued in shared memory;
// a full queue is bitonic-sorted across the warp with shuffles and merged row
// by row (bitonic merge of the row with the reversed queue).  Keys are
// (squared distance, extended id), so ties break by index.
//
// The squared distance is the reference's dist2_point (src/knn/knn.h:64-75),
// dx*dx + dy*dy (+ dz*dz) with dx = query - candidate, compiled without FMA:
// the values, and therefore the order, equal the reference's.
#include <math_constants.h>

#include "pgpu_common.cuh"
#include "pgpu_ctx.h"

namespace pgpu {
namespace {

constexpr int KNN_WARPS = 4;
constexpr unsigned FULL = 0xffffffffu;

__device__ __forceinline__ bool key_less(double ad, uint32_t ai, double bd, uint32_t bi) {
    return ad < bd || (ad == bd && ai < bi);
}

__device__ __forceinline__ uint32_t warp_incl_scan_u32(uint32_t v, int lane) {
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t t = __shfl_up_sync(FULL, v, o);
        if (lane >= o) v += t;
    }
    return v;
}

// Ascending bitonic sort of one (d, id) key per lane across the warp.
__device__ __forceinline__ void bitonic_sort32(double& d, uint32_t& id, int lane) {
#pragma unroll
    for (int k = 2; k <= 32; k <<= 1) {
#pragma unroll
        for (int j = k >> 1; j > 0; j >>= 1) {
            double od = __shfl_xor_sync(FULL, d, j);
            uint32_t oi = __shfl_xor_sync(FULL, id, j);
            bool up = (lane & k) == 0;
            bool lower = (lane & j) == 0;
            bool take = (lower == up) ? key_less(od, oi, d, id) : key_less(d, id, od, oi);
            if (take) {
                d = od;
                id = oi;
            }
        }
    }
}

// Ascending sort of a bitonic sequence held one key per lane.
__device__ __forceinline__ void bitonic_merge32(double& d, uint32_t& id, int lane) {
#pragma unroll
    for (int j = 16; j > 0; j >>= 1) {
        double od = __shfl_xor_sync(FULL, d, j);
        uint32_t oi = __shfl_xor_sync(FULL, id, j);
        bool lower = (lane & j) == 0;
        bool take = lower ? key_less(od, oi, d, id) : key_less(d, id, od, oi);
        if (take) {
            d = od;
            id = oi;
        }
    }
}

// Merges qn queued keys into the ascending rows (rd, ri), keeping the 32R smallest.
template <int R>
__device__ __forceinline__ void merge_queue(double (&rd)[R], uint32_t (&ri)[R], const double* qd,
                                            const uint32_t* qi, int qn, int lane) {
    double d = lane < qn ? qd[lane] : CUDART_INF;
    uint32_t id = lane < qn ? qi[lane] : NO_NEIGHBOR;
    bitonic_sort32(d, id, lane);
#pragma unroll
    for (int r = 0; r < R; r++) {
        double qmin = __shfl_sync(FULL, d, 0);
        uint32_t qmini = __shfl_sync(FULL, id, 0);
        double rmax = __shfl_sync(FULL, rd[r], 31);
        uint32_t rmaxi = __shfl_sync(FULL, ri[r], 31);
        if (!key_less(qmin, qmini, rmax, rmaxi)) continue;  // the queue lies entirely above this row
        double od = __shfl_sync(FULL, d, 31 - lane);
        uint32_t oi = __shfl_sync(FULL, id, 31 - lane);
        bool rl = key_less(rd[r], ri[r], od, oi);
        double lod = rl ? rd[r] : od, hid = rl ? od : rd[r];
        uint32_t loi = rl ? ri[r] : oi, hii = rl ? oi : ri[r];
        bitonic_merge32(lod, loi, lane);
        bitonic_merge32(hid, hii, lane);
        rd[r] = lod;
        ri[r] = loi;
        d = hid;
        id = hii;
    }
}

template <int R>
__device__ __forceinline__ void kth_key(const double (&rd)[R], const uint32_t (&ri)[R], int rk, int lk, double& td,
                                        uint32_t& ti) {
    double d = rd[0];
    uint32_t i = ri[0];
#pragma unroll
    for (int r = 1; r < R; r++)
        if (r == rk) {
            d = rd[r];
            i = ri[r];
        }
    td = __shfl_sync(FULL, d, lk);
    ti = __shfl_sync(FULL, i, lk);
}

template <int D, int R>
__global__ void __launch_bounds__(KNN_WARPS * 32)
    k_knn(const typename PointOf<D>::type* __restrict__ spts, const uint32_t* __restrict__ perm,
          const uint32_t* __restrict__ bin_start, int G, const uint32_t* __restrict__ qs, int64_t nq, int K,
          uint32_t* __restrict__ out, unsigned long long* __restrict__ cand_counter) {
    __shared__ double sq_d[KNN_WARPS][32];
    __shared__ uint32_t sq_i[KNN_WARPS][32];
    __shared__ uint32_t sb_start[KNN_WARPS][32];
    __shared__ uint32_t sb_excl[KNN_WARPS][32];
    using PT = typename PointOf<D>::type;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int64_t t = (int64_t)blockIdx.x * KNN_WARPS + w;
    if (t >= nq) return;  // warp-uniform
    const uint32_t s = qs[t];
    const PT p = spts[s];
    const uint32_t qid = perm[s];
    const double pc[3] = {p.x, p.y, pz(p)};
    const int bc[3] = {bin_coord(p.x, G), bin_coord(p.y, G), D == 3 ? bin_coord(pz(p), G) : 0};
    const double h = 1.0 / (double)G;

    double rd[R];
    uint32_t ri[R];
#pragma unroll
    for (int r = 0; r < R; r++) rd[r] = CUDART_INF, ri[r] = NO_NEIGHBOR;
    const int rk = (K - 1) >> 5, lk = (K - 1) & 31;
    double thr_d = CUDART_INF;
    uint32_t thr_i = NO_NEIGHBOR;
    int qn = 0;
    unsigned long long ncand = 0;

    for (int r = 0;; r++) {
        if (r >= 1) {
            // Every point not yet visited lies outside the cube of rings <= r-1.
            double lb = CUDART_INF;
            bool all = true;
#pragma unroll
            for (int a = 0; a < D; a++) {
                int lo = bc[a] - (r - 1), hi = bc[a] + (r - 1);
                if (lo > 0) {
                    all = false;
                    lb = fmin(lb, pc[a] - (double)lo * h);
                }
                if (hi < G - 1) {
                    all = false;
                    lb = fmin(lb, (double)(hi + 1) * h - pc[a]);
                }
            }
            if (all) break;
            if (thr_i != NO_NEIGHBOR && lb > 0.0 && thr_d < lb * lb * (1.0 - 1e-12)) break;
            if (r > G) break;
        }
        const int w1 = 2 * r + 1;
        const int ncube = D == 2 ? w1 * w1 : w1 * w1 * w1;
        for (int c0 = 0; c0 < ncube; c0 += 32) {
            const int ci = c0 + lane;
            uint32_t bstart = 0, bcnt = 0;
            if (ci < ncube) {
                int dx = ci % w1 - r;
                int rest = ci / w1;
                int dy = rest % w1 - r;
                int dz = D == 3 ? rest / w1 - r : 0;
                int cheb = max(abs(dx), max(abs(dy), abs(dz)));
                int x = bc[0] + dx, y = bc[1] + dy, z = bc[2] + dz;
                bool ok = cheb == r && x >= 0 && x < G && y >= 0 && y < G && (D == 2 || (z >= 0 && z < G));
                if (ok && thr_i != NO_NEIGHBOR) {
                    const int bx[3] = {x, y, z};
                    double bd2 = 0.0;
#pragma unroll
                    for (int a = 0; a < D; a++) {
                        double lo = (double)bx[a] * h, hi = (double)(bx[a] + 1) * h;
                        double dd = pc[a] < lo ? lo - pc[a] : (pc[a] > hi ? pc[a] - hi : 0.0);
                        bd2 += dd * dd;
                    }
                    if (bd2 * (1.0 - 1e-12) > thr_d) ok = false;
                }
                if (ok) {
                    uint32_t key = morton<D>(x, y, z);
                    bstart = bin_start[key];
                    bcnt = bin_start[key + 1] - bstart;
                }
            }
            const uint32_t incl = warp_incl_scan_u32(bcnt, lane);
            const uint32_t total = __shfl_sync(FULL, incl, 31);
            if (total == 0) continue;
            sb_start[w][lane] = bstart;
            sb_excl[w][lane] = incl - bcnt;
            __syncwarp();
            ncand += total;
            for (uint32_t k0 = 0; k0 < total; k0 += 32) {
                const uint32_t tt = k0 + lane;
                bool valid = tt < total;
                double d2 = CUDART_INF;
                uint32_t eid = NO_NEIGHBOR;
                if (valid) {
                    int j = 0;
#pragma unroll
                    for (int step = 16; step > 0; step >>= 1)
                        if (j + step < 32 && sb_excl[w][j + step] <= tt) j += step;
                    const uint32_t sidx = sb_start[w][j] + (tt - sb_excl[w][j]);
                    eid = perm[sidx];
                    if (eid == qid) {
                        valid = false;
                    } else {
                        const PT c = spts[sidx];
                        double ddx = p.x - c.x;
                        double ddy = p.y - c.y;
                        if (D == 2) {
                            d2 = ddx * ddx + ddy * ddy;
                        } else {
                            double ddz = pz(p) - pz(c);
                            d2 = ddx * ddx + ddy * ddy + ddz * ddz;
                        }
                    }
                }
                bool surv = valid && key_less(d2, eid, thr_d, thr_i);
                unsigned bal = __ballot_sync(FULL, surv);
                if (bal == 0) continue;
                if (qn + __popc(bal) > 32) {
                    __syncwarp();
                    merge_queue<R>(rd, ri, sq_d[w], sq_i[w], qn, lane);
                    qn = 0;
                    kth_key<R>(rd, ri, rk, lk, thr_d, thr_i);
                    surv = surv && key_less(d2, eid, thr_d, thr_i);
                    bal = __ballot_sync(FULL, surv);
                }
                if (surv) {
                    int pos = qn + __popc(bal & ((1u << lane) - 1u));
                    sq_d[w][pos] = d2;
                    sq_i[w][pos] = eid;
                }
                qn += __popc(bal);
                __syncwarp();
            }
            __syncwarp();
        }
        if (qn > 0) {
            __syncwarp();
            merge_queue<R>(rd, ri, sq_d[w], sq_i[w], qn, lane);
            qn = 0;
            kth_key<R>(rd, ri, rk, lk, thr_d, thr_i);
        }
    }
#pragma unroll
    for (int r = 0; r < R; r++) {
        int idx = r * 32 + lane;
        if (idx < K) out[t * K + idx] = ri[r];
    }
    if (cand_counter && lane == 0) atomicAdd(cand_counter, ncand);
}

template <int D>
cudaError_t knn_dispatch(pgpu_ctx* c, const uint32_t* qs, int64_t nq, int K, uint32_t* out,
                         unsigned long long* cc) {
    if (nq <= 0) return cudaSuccess;
    const unsigned blocks = (unsigned)((nq + KNN_WARPS - 1) / KNN_WARPS);
    using PT = typename PointOf<D>::type;
    const PT* sp = (const PT*)c->spts.p;
    const uint32_t* perm = (const uint32_t*)c->perm.p;
    const uint32_t* bs = (const uint32_t*)c->bin_start.p;
    const int G = c->grid_G;
#define PGPU_KNN_CASE(RR) k_knn<D, RR><<<blocks, KNN_WARPS * 32, 0, c->stream>>>(sp, perm, bs, G, qs, nq, K, out, cc)
    if (K <= 32)
        PGPU_KNN_CASE(1);
    else if (K <= 64)
        PGPU_KNN_CASE(2);
    else if (K <= 96)
        PGPU_KNN_CASE(3);
    else if (K <= 128)
        PGPU_KNN_CASE(4);
    else if (K <= 192)
        PGPU_KNN_CASE(6);
    else
        PGPU_KNN_CASE(8);
#undef PGPU_KNN_CASE
    count_launches(1);
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_knn_list(pgpu_ctx* c, const uint32_t* qs, int64_t nq, int K, uint32_t* out) {
    DevScalars* sc = (DevScalars*)c->scalars.p;
    unsigned long long* cc = &sc->knn_cand;
    return c->prm.dim == 2 ? knn_dispatch<2>(c, qs, nq, K, out, cc) : knn_dispatch<3>(c, qs, nq, K, out, cc);
}

cudaError_t launch_knn(pgpu_ctx* c) {
    cudaError_t e = cudaSuccess;
    const int K = c->prm.k;
    uint32_t* out = ensure<uint32_t>(c->knn, (size_t)c->n_query * K + 1, &e);
    if (e) return e;
    DevScalars* sc = (DevScalars*)c->scalars.p;
    if ((e = cudaMemsetAsync(&sc->knn_cand, 0, sizeof(unsigned long long), c->stream))) return e;
    return launch_knn_list(c, (const uint32_t*)c->qs.p, c->n_query, K, out);
}

}  // namespace pgpu
