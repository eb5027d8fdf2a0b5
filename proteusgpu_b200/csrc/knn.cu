// Exact K nearest neighbours on the Morton-ordered grid (replaces
// knn::solve / cpu_knearest, src/knn/knn.cpp:225-315).
//
// One warp per query point.  Neighbour bins are visited in the order of a
// host-built offset table sorted by the lower bound of the distance from any
// point of the query's bin to the offset bin, h^2 * sum_a max(|d_a| - 1, 0)^2
// (the reference's ring table, knn.cpp:39-89, orders by Chebyshev ring with the
// bound (ring - 1)^2 h^2; this order is tighter).  Thirty-two table entries are
// taken per step, one per lane; a bin whose box lies farther than the current
// K-th neighbour is skipped, and the search ends as soon as the table's bound
// passes the K-th neighbour.  The chunk's bins are expanded into one flat
// candidate range by a warp prefix sum so that every lane evaluates one
// candidate per step whatever the bin occupancy.  Beyond the table (sparse
// regions) the search continues ring by ring.
//
// The K best are kept ascending in shared memory, ceil(K/32) rows of 32 per
// warp.  Candidates that beat the current K-th best queue in shared memory; a
// full queue is bitonic-sorted across the warp with shuffles and merged row by
// row (bitonic merge of the row with the reversed queue), in a loop that is not
// unrolled so the kernel's code stays small.  Keys order by (squared distance,
// extended id): ties break by index.  The search runs on packed 64-bit keys (the
// distance rounded up to FP32 above the id); a query whose list a tie of rounded
// distances could change is searched again with exact keys (k_knn_exact), so the
// lists are the exact ones.
//
// The squared distance is the reference's dist2_point (src/knn/knn.h:64-75),
// dx*dx + dy*dy (+ dz*dz) with dx = query - candidate, without FMA, so the
// values and therefore the order equal the reference's.
#include <math_constants.h>

#include <algorithm>
#include <vector>

#include "pgpu_common.cuh"
#include "pgpu_ctx.h"

namespace pgpu {
namespace {

constexpr int MAX_ROWS = MAX_K / 32;
constexpr unsigned FULL = 0xffffffffu;
constexpr int TABLE_R3 = 8;   // offsets with |d|_inf <= 8 in 3D (17^3 entries)
constexpr int TABLE_R2 = 24;  // and |d|_inf <= 24 in 2D (49^2 entries)
#ifndef KNN_FLUSH_MIN
#define KNN_FLUSH_MIN 24  // queued survivors that trigger a merge at a table-chunk boundary
#endif

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

// Keys of the K-best rows.  Exact: (squared distance, extended id), compared
// lexicographically.  Packed: one 64-bit integer, the squared distance rounded up to
// FP32 in the high word and the id in the low word, so that an exchange takes two
// shuffles and one integer compare instead of three shuffles and a pair compare.
// Rounding up is monotone, so the packed order equals the exact one except between
// keys whose rounded distances are equal; the packed search flags every such tie
// that could change its list (see knn_query) and the query is searched again with
// exact keys.  A packed K-th key's rounded distance bounds the exact one from
// above, so box pruning against it keeps every box the exact search keeps.
template <bool PK>
struct KeyOps;

template <>
struct KeyOps<false> {
    struct K {
        double d;
        uint32_t i;
    };
    static __device__ __forceinline__ K none() { return {CUDART_INF, NO_NEIGHBOR}; }
    static __device__ __forceinline__ K make(double d, uint32_t i) { return {d, i}; }
    static __device__ __forceinline__ bool lt(const K& a, const K& b) { return key_less(a.d, a.i, b.d, b.i); }
    static __device__ __forceinline__ K shfl_xor(const K& a, int j) {
        return {__shfl_xor_sync(FULL, a.d, j), __shfl_xor_sync(FULL, a.i, j)};
    }
    static __device__ __forceinline__ K shfl(const K& a, int src) {
        return {__shfl_sync(FULL, a.d, src), __shfl_sync(FULL, a.i, src)};
    }
    static __device__ __forceinline__ uint32_t id(const K& a) { return a.i; }
    static __device__ __forceinline__ bool held(const K& a) { return a.i != NO_NEIGHBOR; }
    static __device__ __forceinline__ double bound(const K& a) { return a.d; }
    static __device__ __forceinline__ bool tie(const K&, const K&) { return false; }
};

template <>
struct KeyOps<true> {
    using K = unsigned long long;
    static __device__ __forceinline__ K none() { return ~0ull; }
    static __device__ __forceinline__ K make(double d, uint32_t i) {
        return ((K)__float_as_uint(__double2float_ru(d)) << 32) | i;
    }
    static __device__ __forceinline__ bool lt(K a, K b) { return a < b; }
    static __device__ __forceinline__ K shfl_xor(K a, int j) { return __shfl_xor_sync(FULL, a, j); }
    static __device__ __forceinline__ K shfl(K a, int src) { return __shfl_sync(FULL, a, src); }
    static __device__ __forceinline__ uint32_t id(K a) { return (uint32_t)a; }
    static __device__ __forceinline__ bool held(K a) { return a != ~0ull; }
    static __device__ __forceinline__ double bound(K a) { return (double)__uint_as_float((uint32_t)(a >> 32)); }
    static __device__ __forceinline__ bool tie(K a, K b) { return (a >> 32) == (b >> 32); }
};

// One warp's shared memory: the K best (rows of 32), the survivor queue and the
// chunk's bin table.
template <bool PK>
struct WarpKnn;

template <>
struct WarpKnn<false> {
    using K = KeyOps<false>::K;
    double row_d[MAX_ROWS * 32];
    uint32_t row_i[MAX_ROWS * 32];
    double q_d[32];
    uint32_t q_i[32];
    uint32_t b_start[32];
    uint32_t b_excl[32];
    __device__ __forceinline__ K row(int x) const { return {row_d[x], row_i[x]}; }
    __device__ __forceinline__ void set_row(int x, const K& k) {
        row_d[x] = k.d;
        row_i[x] = k.i;
    }
    __device__ __forceinline__ K q(int x) const { return {q_d[x], q_i[x]}; }
    __device__ __forceinline__ void set_q(int x, const K& k) {
        q_d[x] = k.d;
        q_i[x] = k.i;
    }
};

template <>
struct WarpKnn<true> {
    using K = KeyOps<true>::K;
    K row_k[MAX_ROWS * 32];
    K q_k[32];
    uint32_t b_start[32];
    uint32_t b_excl[32];
    __device__ __forceinline__ K row(int x) const { return row_k[x]; }
    __device__ __forceinline__ void set_row(int x, K k) { row_k[x] = k; }
    __device__ __forceinline__ K q(int x) const { return q_k[x]; }
    __device__ __forceinline__ void set_q(int x, K k) { q_k[x] = k; }
};

// Ascending bitonic sort of one key per lane across the warp.
template <bool PK, int KMAX = 32>
__device__ __forceinline__ void bitonic_sort32(typename KeyOps<PK>::K& a, int lane) {
    using O = KeyOps<PK>;
#pragma unroll
    for (int k = 2; k <= KMAX; k <<= 1) {
#pragma unroll
        for (int j = k >> 1; j > 0; j >>= 1) {
            const typename O::K o = O::shfl_xor(a, j);
            const bool up = (lane & k) == 0;
            const bool lower = (lane & j) == 0;
            // packed keys are distinct but for the empty key, so "a < o" is "not o < a" up to
            // swapping two equal keys: one integer compare per stage
            const bool take = PK ? (O::lt(o, a) == (lower == up)) : ((lower == up) ? O::lt(o, a) : O::lt(a, o));
            if (take) a = o;
        }
    }
}

// Ascending sort of a bitonic sequence held one key per lane.
template <bool PK>
__device__ __forceinline__ void bitonic_merge32(typename KeyOps<PK>::K& a, int lane) {
    using O = KeyOps<PK>;
#pragma unroll
    for (int j = 16; j > 0; j >>= 1) {
        const typename O::K o = O::shfl_xor(a, j);
        const bool lower = (lane & j) == 0;
        const bool take = PK ? (O::lt(o, a) == lower) : (lower ? O::lt(o, a) : O::lt(a, o));
        if (take) a = o;
    }
}

// Merges qn queued keys into the warp's ascending rows, keeping the 32 * nrows
// smallest.  Packed keys: returns whether an evicted key's rounded distance equals
// the last held key's (a tie across the rows' end).
template <bool PK>
__device__ __noinline__ bool merge_queue(WarpKnn<PK>& S, int qn, int nrows, int lane) {
    using O = KeyOps<PK>;
    using K = typename O::K;
    K a = lane < qn ? S.q(lane) : O::none();
    // at most 16 queued keys: lanes 16-31 hold the empty key, so the first four levels leave
    // lanes 0-15 ascending and the sequence sorted (the last level would change nothing)
    if (qn <= 16)
        bitonic_sort32<PK, 16>(a, lane);
    else
        bitonic_sort32<PK>(a, lane);
#pragma unroll 1
    for (int r = 0; r < nrows; r++) {
        const K qmin = O::shfl(a, 0);
        const K rmax = S.row(r * 32 + 31);
        if (!O::lt(qmin, rmax)) continue;  // the queue lies entirely above this row
        const K o = O::shfl(a, 31 - lane);
        const K c = S.row(r * 32 + lane);
        const bool rl = O::lt(c, o);
        K lo = rl ? c : o, hi = rl ? o : c;
        bitonic_merge32<PK>(lo, lane);
        bitonic_merge32<PK>(hi, lane);
        __syncwarp();
        S.set_row(r * 32 + lane, lo);
        __syncwarp();
        a = hi;
    }
    if constexpr (PK) {
        const K m = O::shfl(a, 0);
        return O::held(m) && O::tie(m, S.row(nrows * 32 - 1));
    }
    return false;
}

// Processes one set of up to 32 bins (bstart, bcnt per lane) against the query.
// thr is the K-th held key (none until K are held); tie collects the packed
// search's rejected keys whose rounded distance equals thr's.
template <int D, bool PK>
__device__ __forceinline__ void scan_bins(const typename PointOf<D>::type* __restrict__ spts,
                                          const uint32_t* __restrict__ perm, uint32_t bstart, uint32_t bcnt,
                                          const typename PointOf<D>::type& p, uint32_t qid, WarpKnn<PK>& S,
                                          int lane, int nrows, int K, int& qn, typename KeyOps<PK>::K& thr,
                                          unsigned long long& ncand, bool& tie) {
    using PT = typename PointOf<D>::type;
    using O = KeyOps<PK>;
    const uint32_t incl = warp_incl_scan_u32(bcnt, lane);
    const uint32_t total = __shfl_sync(FULL, incl, 31);
    if (total == 0) return;
    __syncwarp();
    S.b_start[lane] = bstart;
    S.b_excl[lane] = incl - bcnt;
    __syncwarp();
    ncand += total;
    for (uint32_t k0 = 0; k0 < total; k0 += 32) {
        const uint32_t tt = k0 + lane;
        bool valid = tt < total;
        typename O::K key = O::none();
        if (valid) {
            // after the steps 16 .. 2s, j is a multiple of 2s and at most 32 - 2s, so j + s <= 31
            int j = 0;
#pragma unroll
            for (int step = 16; step > 0; step >>= 1)
                if (S.b_excl[j + step] <= tt) j += step;
            const uint32_t sidx = S.b_start[j] + (tt - S.b_excl[j]);
            const uint32_t eid = perm[sidx];
            if (eid == qid) {
                valid = false;
            } else {
                const PT c = spts[sidx];
                double ddx = p.x - c.x;
                double ddy = p.y - c.y;
                double d2;
                if (D == 2) {
                    d2 = ddx * ddx + ddy * ddy;
                } else {
                    double ddz = pz(p) - pz(c);
                    d2 = ddx * ddx + ddy * ddy + ddz * ddz;
                }
                if (PK && d2 != d2) valid = false;  // NaN: the exact compare drops it too
                key = O::make(d2, eid);
            }
        }
        bool surv = valid && O::lt(key, thr);
        if (PK) tie |= valid && !surv && O::tie(key, thr);
        unsigned bal = __ballot_sync(FULL, surv);
        if (bal == 0) continue;
        if (qn + __popc(bal) > 32) {
            __syncwarp();
            tie |= merge_queue<PK>(S, qn, nrows, lane);
            qn = 0;
            __syncwarp();
            thr = S.row(K - 1);
            surv = surv && O::lt(key, thr);
            if (PK) tie |= valid && !surv && O::tie(key, thr);
            bal = __ballot_sync(FULL, surv);
        }
        if (surv) S.set_q(qn + __popc(bal & ((1u << lane) - 1u)), key);
        qn += __popc(bal);
        __syncwarp();
    }
}

template <bool PK>
__device__ __forceinline__ void flush_queue(WarpKnn<PK>& S, int lane, int nrows, int K, int& qn,
                                            typename KeyOps<PK>::K& thr, bool& tie) {
    if (qn == 0) return;
    __syncwarp();
    tie |= merge_queue<PK>(S, qn, nrows, lane);
    qn = 0;
    __syncwarp();
    thr = S.row(K - 1);
}

// Squared distance from p to the box of bin (x, y, z).
template <int D>
__device__ __forceinline__ double box_d2(const double* pc, int x, int y, int z, double h) {
    const int bx[3] = {x, y, z};
    double bd2 = 0.0;
#pragma unroll
    for (int a = 0; a < D; a++) {
        double lo = (double)bx[a] * h, hi = (double)(bx[a] + 1) * h;
        double dd = pc[a] < lo ? lo - pc[a] : (pc[a] > hi ? pc[a] - hi : 0.0);
        bd2 += dd * dd;
    }
    return bd2;
}

// Sorted-point range of the level-Lq box (x, y, z) for a query whose own box is
// qb.  In a bin refined at least as finely the box is an aligned block of
// Morton-consecutive sub-bins.  In a coarser bin the box lies inside one larger
// sub-bin S, which is scanned whole, once: from the box of S nearest the query
// (the query's box clamped into S), whose box distance is S's own.
template <int D>
__device__ __forceinline__ bool box_range(const SubGrid& g, uint32_t slot0, int Lq, int x, int y, int z,
                                          const int (&qb)[3], uint32_t& start, uint32_t& cnt) {
    const int cx = x >> Lq, cy = y >> Lq, cz = z >> Lq;
    const uint32_t m = slot0 + morton<D>(cx, cy, cz);
    const int Lb = g.lvl[m];
    const uint32_t base = g.sub_off[m];
    uint32_t a, b;
    if (Lb >= Lq) {
        const int sh = Lb - Lq;
        const uint32_t first = morton<D>(x - (cx << Lq), y - (cy << Lq), z - (cz << Lq)) << (D * sh);
        a = base + first;
        b = a + (1u << (D * sh));
    } else {
        const int sh = Lq - Lb;
        const int sx = x >> sh, sy = y >> sh, sz = z >> sh;
        const int bxs[3] = {x, y, z}, sxs[3] = {sx, sy, sz};
#pragma unroll
        for (int k = 0; k < D; k++) {
            const int lo = sxs[k] << sh, hi = lo + (1 << sh) - 1;
            const int nearest = qb[k] < lo ? lo : (qb[k] > hi ? hi : qb[k]);
            if (bxs[k] != nearest) return false;
        }
        a = base + morton<D>(sx - (cx << Lb), sy - (cy << Lb), sz - (cz << Lb));
        b = a + 1;
    }
    start = g.sub_start[a];
    cnt = g.sub_start[b] - start;
    return true;
}

// One query's search by one warp (query t, budget K): the K nearest ext ids of the
// query point, ascending, written to out[t * stride ...].  Packed keys: returns
// true (and writes nothing) when a tie of rounded distances could make the list
// differ from the exact one -- two equal rounded distances side by side among the
// first K + 1 held keys, or a rejected or evicted key whose rounded distance equals
// the K-th's at the time -- so that the query is searched again with exact keys.
template <int D, bool PK>
__device__ __forceinline__ bool knn_query(const typename PointOf<D>::type* __restrict__ spts,
                                          const uint32_t* __restrict__ perm, const SubGrid& grid,
                                          const int2* __restrict__ table, int table_n, int table_r,
                                          const uint32_t* __restrict__ qs, int64_t t, int K, int stride,
                                          uint32_t* __restrict__ out, WarpKnn<PK>& S, int lane,
                                          unsigned long long& ncand) {
    using PT = typename PointOf<D>::type;
    using O = KeyOps<PK>;
    const int nrows = (K + 31) >> 5;
    for (int r = 0; r < nrows; r++) S.set_row(r * 32 + lane, O::none());
    __syncwarp();
    const uint32_t s = qs[t];
    const PT p = spts[s];
    const uint32_t qid = perm[s];
    if (!(isfinite(p.x) && isfinite(p.y) && isfinite(pz(p)))) {  // no neighbours for a point without a position
        for (int idx = lane; idx < K; idx += 32) out[t * stride + idx] = NO_NEIGHBOR;
        return false;
    }
    const double pc[3] = {p.x, p.y, pz(p)};
    // the query searches its own instance's grid at its own bin's level: boxes of side 1 / (G << Lq)
    const InstPar& ipq = grid.ip[grid.inst[qid]];
    const int G0 = ipq.G;
    const uint32_t slot0 = ipq.slot0;
    const int Lq =
        grid.lvl[slot0 + morton<D>(bin_coord(p.x, G0), bin_coord(p.y, G0), D == 3 ? bin_coord(pz(p), G0) : 0)];
    const int G = G0 << Lq;
    const int bc[3] = {sub_coord(p.x, G0, Lq), sub_coord(p.y, G0, Lq), D == 3 ? sub_coord(pz(p), G0, Lq) : 0};
    const double h = 1.0 / (double)G;
    typename O::K thr = O::none();
    int qn = 0;
    bool tie = false;

    // 1. offsets in order of their lower bound
    for (int c0 = 0; c0 < table_n; c0 += 32) {
        const int2 first = table[c0];
        // every remaining table bin is farther than the K-th neighbour; bins beyond the
        // table (which may be nearer than the table's last entries) are left to the
        // ring search, whose first test ends it at once when they are all too far
        if (O::held(thr) && (double)first.y * h * h * (1.0 - 1e-12) > O::bound(thr)) break;
        const int ci = c0 + lane;
        uint32_t bstart = 0, bcnt = 0;
        if (ci < table_n) {
            const int2 ent = table[ci];
            const int dx = (int)(signed char)(ent.x & 255), dy = (int)(signed char)((ent.x >> 8) & 255),
                      dz = (int)(signed char)((ent.x >> 16) & 255);
            const int x = bc[0] + dx, y = bc[1] + dy, z = bc[2] + dz;
            bool ok = x >= 0 && x < G && y >= 0 && y < G && (D == 2 || (z >= 0 && z < G));
            if (ok && O::held(thr) && box_d2<D>(pc, x, y, z, h) * (1.0 - 1e-12) > O::bound(thr)) ok = false;
            if (ok && !box_range<D>(grid, slot0, Lq, x, y, z, bc, bstart, bcnt)) bcnt = 0;
        }
        scan_bins<D, PK>(spts, perm, bstart, bcnt, p, qid, S, lane, nrows, K, qn, thr, ncand, tie);
        // the bound is tested at chunk boundaries: merge what is queued once it is worth a
        // merge (a staler bound only prunes less; the rows fill up first)
        if (qn >= KNN_FLUSH_MIN || !O::held(thr)) flush_queue<PK>(S, lane, nrows, K, qn, thr, tie);
    }
    flush_queue<PK>(S, lane, nrows, K, qn, thr, tie);

    // 2. beyond the table: Chebyshev rings table_r + 1, table_r + 2, ... (sparse regions)
    for (int r = table_r + 1;; r++) {
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
        if (all || r > G + 1) break;
        if (O::held(thr) && lb > 0.0 && O::bound(thr) < lb * lb * (1.0 - 1e-12)) break;
        const int w1 = 2 * r + 1;
        const int ncube = D == 2 ? w1 * w1 : w1 * w1 * w1;
        for (int c0 = 0; c0 < ncube; c0 += 32) {
            const int ci = c0 + lane;
            uint32_t bstart = 0, bcnt = 0;
            if (ci < ncube) {
                const int dx = ci % w1 - r;
                const int rest = ci / w1;
                const int dy = rest % w1 - r;
                const int dz = D == 3 ? rest / w1 - r : 0;
                const int cheb = max(abs(dx), max(abs(dy), abs(dz)));
                const int x = bc[0] + dx, y = bc[1] + dy, z = bc[2] + dz;
                bool ok = cheb == r && x >= 0 && x < G && y >= 0 && y < G && (D == 2 || (z >= 0 && z < G));
                if (ok && O::held(thr) && box_d2<D>(pc, x, y, z, h) * (1.0 - 1e-12) > O::bound(thr)) ok = false;
                if (ok && !box_range<D>(grid, slot0, Lq, x, y, z, bc, bstart, bcnt)) bcnt = 0;
            }
            scan_bins<D, PK>(spts, perm, bstart, bcnt, p, qid, S, lane, nrows, K, qn, thr, ncand, tie);
        }
        flush_queue<PK>(S, lane, nrows, K, qn, thr, tie);
    }
    __syncwarp();
    if (PK) {
        // equal rounded distances side by side among the first K + 1 held keys
        for (int idx = lane; idx < K; idx += 32)
            if (idx + 1 < nrows * 32) {
                const typename O::K a = S.row(idx);
                if (O::held(a) && O::tie(a, S.row(idx + 1))) tie = true;
            }
        tie = __any_sync(FULL, tie);
        if (tie) return true;
    }
    for (int idx = lane; idx < K; idx += 32) out[t * stride + idx] = O::id(S.row(idx));
    return false;
}

// 40 warps per SM: at most 48 registers a thread, a few spilled (the search is latency
// bound on its warp-collective chains; more resident warps hide more of them: 122.0 ->
// 118.4 ms at 16.8M clustered points against 32 warps).  Packed keys; a query with a tie
// is listed in redo for k_knn_exact.
template <int D, int KW>
__global__ void __launch_bounds__(KW * 32, KW == 1 ? 32 : 40 / KW)
    k_knn(const typename PointOf<D>::type* __restrict__ spts, const uint32_t* __restrict__ perm, SubGrid grid,
          const int2* __restrict__ table, int table_n, int table_r, const uint32_t* __restrict__ qs, int64_t nq,
          int K, const uint16_t* __restrict__ kq, int stride, uint32_t* __restrict__ out,
          unsigned long long* __restrict__ cand_counter, int skip_upto, uint32_t* __restrict__ redo,
          unsigned* __restrict__ redo_n) {
    __shared__ WarpKnn<true> S_all[KW];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int64_t t = (int64_t)blockIdx.x * KW + w;
    if (t >= nq) return;  // warp-uniform
    if (kq) K = kq[t];
    if (K <= skip_upto) return;  // done by k_knn_t
    unsigned long long ncand = 0;
    const bool tie = knn_query<D, true>(spts, perm, grid, table, table_n, table_r, qs, t, K, stride, out, S_all[w],
                                        lane, ncand);
    if (lane == 0) {
        if (tie) redo[atomicAdd(redo_n, 1u)] = (uint32_t)t;
        if (cand_counter) atomicAdd(cand_counter, ncand);
    }
}

// The queries k_knn listed in redo, searched again with exact keys; warps stride
// over the list, whose length the device holds.
template <int D, int KW>
__global__ void __launch_bounds__(KW * 32, 32 / KW)
    k_knn_exact(const typename PointOf<D>::type* __restrict__ spts, const uint32_t* __restrict__ perm,
                SubGrid grid, const int2* __restrict__ table, int table_n, int table_r,
                const uint32_t* __restrict__ qs, int Kall, const uint16_t* __restrict__ kq, int stride,
                uint32_t* __restrict__ out, unsigned long long* __restrict__ cand_counter,
                const uint32_t* __restrict__ redo, const unsigned* __restrict__ redo_n,
                unsigned* __restrict__ redo_total) {
    __shared__ WarpKnn<false> S_all[KW];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int64_t n = *redo_n;
    if (blockIdx.x == 0 && threadIdx.x == 0 && n) atomicAdd(redo_total, (unsigned)n);
    unsigned long long ncand = 0;
    for (int64_t i = (int64_t)blockIdx.x * KW + w; i < n; i += (int64_t)gridDim.x * KW) {  // warp-uniform
        const int64_t t = redo[i];
        const int K = kq ? (int)kq[t] : Kall;
        knn_query<D, false>(spts, perm, grid, table, table_n, table_r, qs, t, K, stride, out, S_all[w], lane,
                            ncand);
    }
    if (cand_counter && lane == 0 && ncand) atomicAdd(cand_counter, ncand);
}

// Thread-per-query variant for small K (<= KT): the same bins in the same order,
// pruned against the running K-th key, the K best kept sorted in the thread's own
// list by insertion.  Pruning only drops boxes that cannot hold a key below the
// final K-th, so the list equals the warp kernel's.  Queries with a larger K return
// at once here and are done by k_knn, which skips the ones done here.
// The lists live in shared memory, entry i of thread t at [i * KNN_T_THREADS + t]
// (conflict-free; per-thread local arrays of this size spill out of L1).  Keys are
// packed like k_knn's, with the same tie rule for a list of exactly K: a rejected key
// whose rounded distance equals the K-th's, a key pushed out whose rounded distance
// equals the new K-th's, or two equal rounded distances side by side in the list send
// the query to redo for k_knn_exact.
constexpr int KNN_T_THREADS = 64;

// Dynamic shared memory: kcap * KNN_T_THREADS packed keys, kcap = min(Kall, KT).
template <int D>
__global__ void __launch_bounds__(KNN_T_THREADS)
    k_knn_t(const typename PointOf<D>::type* __restrict__ spts, const uint32_t* __restrict__ perm, SubGrid grid,
            const int2* __restrict__ table, int table_n, int table_r, const uint32_t* __restrict__ qs, int64_t nq,
            int Kall, int KT, const uint16_t* __restrict__ kq, int stride, uint32_t* __restrict__ out,
            unsigned long long* __restrict__ cand_counter, uint32_t* __restrict__ redo,
            unsigned* __restrict__ redo_n) {
    using PT = typename PointOf<D>::type;
    using O = KeyOps<true>;
    using Key = O::K;
    extern __shared__ __align__(16) unsigned char knn_t_smem[];
    const int kcap = min(Kall, KT);
    Key* kk = (Key*)knn_t_smem + threadIdx.x;
    constexpr int S = KNN_T_THREADS;
    const int64_t t = (int64_t)blockIdx.x * KNN_T_THREADS + threadIdx.x;
    unsigned long long ncand = 0;
    if (t < nq) {
        const int K = kq ? (int)kq[t] : Kall;
        if (K <= kcap) {  // the rest: k_knn
            int cnt = 0;
            Key thr = O::none();  // the K-th key once K are held
            bool tie = false;
            const uint32_t s = qs[t];
            const PT p = spts[s];
            const uint32_t qid = perm[s];
            if (isfinite(p.x) && isfinite(p.y) && isfinite(pz(p))) {
                const double pc[3] = {p.x, p.y, pz(p)};
                const InstPar& ipq = grid.ip[grid.inst[qid]];
                const int G0 = ipq.G;
                const uint32_t slot0 = ipq.slot0;
                const int Lq = grid.lvl[slot0 + morton<D>(bin_coord(p.x, G0), bin_coord(p.y, G0),
                                                          D == 3 ? bin_coord(pz(p), G0) : 0)];
                const int G = G0 << Lq;
                const int bc[3] = {sub_coord(p.x, G0, Lq), sub_coord(p.y, G0, Lq),
                                   D == 3 ? sub_coord(pz(p), G0, Lq) : 0};
                const double h = 1.0 / (double)G;
                auto scan_range = [&](uint32_t bstart, uint32_t bcnt) {
                    ncand += bcnt;
                    for (uint32_t q = bstart; q < bstart + bcnt; q++) {
                        const uint32_t eid = perm[q];
                        if (eid == qid) continue;
                        const PT c = spts[q];
                        const double ddx = p.x - c.x, ddy = p.y - c.y;
                        double d2;
                        if (D == 2) {
                            d2 = ddx * ddx + ddy * ddy;
                        } else {
                            const double ddz = pz(p) - pz(c);
                            d2 = ddx * ddx + ddy * ddy + ddz * ddz;
                        }
                        if (d2 != d2) continue;  // NaN: the exact compare drops it too
                        const Key key = O::make(d2, eid);
                        if (!(key < thr)) {
                            if (O::held(thr) && O::tie(key, thr)) tie = true;
                            continue;
                        }
                        const Key out_key = cnt == K ? kk[(K - 1) * S] : O::none();
                        int i = cnt < K ? cnt : K - 1;
                        while (i > 0) {
                            const Key o = kk[(i - 1) * S];
                            if (!(key < o)) break;
                            kk[i * S] = o;
                            i--;
                        }
                        kk[i * S] = key;
                        if (cnt < K) cnt++;
                        if (cnt == K) {
                            thr = kk[(K - 1) * S];
                            if (O::held(out_key) && O::tie(out_key, thr)) tie = true;
                        }
                    }
                };
                // 1. offsets in order of their lower bound
                for (int ci = 0; ci < table_n; ci++) {
                    const int2 ent = table[ci];
                    if (O::held(thr) && (double)ent.y * h * h * (1.0 - 1e-12) > O::bound(thr)) break;
                    const int dx = (int)(signed char)(ent.x & 255), dy = (int)(signed char)((ent.x >> 8) & 255),
                              dz = (int)(signed char)((ent.x >> 16) & 255);
                    const int x = bc[0] + dx, y = bc[1] + dy, z = bc[2] + dz;
                    if (!(x >= 0 && x < G && y >= 0 && y < G && (D == 2 || (z >= 0 && z < G)))) continue;
                    if (O::held(thr) && box_d2<D>(pc, x, y, z, h) * (1.0 - 1e-12) > O::bound(thr)) continue;
                    uint32_t bstart, bcnt;
                    if (box_range<D>(grid, slot0, Lq, x, y, z, bc, bstart, bcnt)) scan_range(bstart, bcnt);
                }
                // 2. beyond the table: Chebyshev rings
                for (int r = table_r + 1;; r++) {
                    double lb = CUDART_INF;
                    bool all = true;
                    for (int a = 0; a < D; a++) {
                        const int lo = bc[a] - (r - 1), hi = bc[a] + (r - 1);
                        if (lo > 0) {
                            all = false;
                            lb = fmin(lb, pc[a] - (double)lo * h);
                        }
                        if (hi < G - 1) {
                            all = false;
                            lb = fmin(lb, (double)(hi + 1) * h - pc[a]);
                        }
                    }
                    if (all || r > G + 1) break;
                    if (O::held(thr) && lb > 0.0 && O::bound(thr) < lb * lb * (1.0 - 1e-12)) break;
                    const int w1 = 2 * r + 1;
                    const int ncube = D == 2 ? w1 * w1 : w1 * w1 * w1;
                    for (int ci = 0; ci < ncube; ci++) {
                        const int dx = ci % w1 - r, rest = ci / w1;
                        const int dy = rest % w1 - r, dz = D == 3 ? rest / w1 - r : 0;
                        if (max(abs(dx), max(abs(dy), abs(dz))) != r) continue;
                        const int x = bc[0] + dx, y = bc[1] + dy, z = bc[2] + dz;
                        if (!(x >= 0 && x < G && y >= 0 && y < G && (D == 2 || (z >= 0 && z < G)))) continue;
                        if (O::held(thr) && box_d2<D>(pc, x, y, z, h) * (1.0 - 1e-12) > O::bound(thr)) continue;
                        uint32_t bstart, bcnt;
                        if (box_range<D>(grid, slot0, Lq, x, y, z, bc, bstart, bcnt)) scan_range(bstart, bcnt);
                    }
                }
            }
            for (int i = 0; i + 1 < cnt; i++)
                if (O::tie(kk[i * S], kk[(i + 1) * S])) tie = true;
            if (tie)
                redo[atomicAdd(redo_n, 1u)] = (uint32_t)t;
            else
                for (int i = 0; i < K; i++) out[t * stride + i] = i < cnt ? O::id(kk[i * S]) : NO_NEIGHBOR;
        }
    }
    if (cand_counter) {
        for (int o = 16; o > 0; o >>= 1) ncand += __shfl_xor_sync(FULL, ncand, o);
        if ((threadIdx.x & 31) == 0 && ncand) atomicAdd(cand_counter, ncand);
    }
}

}  // namespace

// Offset table: every (dx, dy, dz) with |d|_inf <= R, sorted by the lower bound
// sum_a max(|d_a| - 1, 0)^2 (bin units), then by Chebyshev ring, then by index.
cudaError_t build_knn_table(pgpu_ctx* c) {
    const int D = c->prm.dim;
    const int R = D == 2 ? TABLE_R2 : TABLE_R3;
    struct E {
        int lb, ring, order, packed;
    };
    std::vector<E> es;
    int order = 0;
    for (int dz = (D == 3 ? -R : 0); dz <= (D == 3 ? R : 0); dz++)
        for (int dy = -R; dy <= R; dy++)
            for (int dx = -R; dx <= R; dx++) {
                auto g = [](int d) { return std::max(std::abs(d) - 1, 0); };
                E e;
                e.lb = g(dx) * g(dx) + g(dy) * g(dy) + g(dz) * g(dz);
                e.ring = std::max(std::abs(dx), std::max(std::abs(dy), std::abs(dz)));
                e.order = order++;
                e.packed = (dx & 255) | ((dy & 255) << 8) | ((dz & 255) << 16);
                es.push_back(e);
            }
    std::sort(es.begin(), es.end(), [](const E& a, const E& b) {
        if (a.lb != b.lb) return a.lb < b.lb;
        if (a.ring != b.ring) return a.ring < b.ring;
        return a.order < b.order;
    });
    std::vector<int2> host(es.size());
    for (size_t i = 0; i < es.size(); i++) host[i] = make_int2(es[i].packed, es[i].lb);
    cudaError_t e = cudaSuccess;
    int2* d = ensure<int2>(c->knn_table, host.size(), &e);
    if (e) return e;
    if ((e = cudaMemcpyAsync(d, host.data(), host.size() * sizeof(int2), cudaMemcpyHostToDevice, c->stream))) return e;
    c->knn_table_n = (int)host.size();
    c->knn_table_r = R;
    return cudaStreamSynchronize(c->stream);
}

cudaError_t launch_knn_list(pgpu_ctx* c, const uint32_t* qs, int64_t nq, int K, uint32_t* out, const uint16_t* kq,
                            int stride) {
    if (nq <= 0) return cudaSuccess;
    cudaError_t e = cudaSuccess;
    if (c->knn_table_n == 0 && (e = build_knn_table(c))) return e;
    DevScalars* sc = (DevScalars*)c->scalars.p;
    const int KW = c->tune.knn_warps;  // warps (queries) per block: autotuned, 1, 2, 4 or 8
    const int KT = c->tune.knn_thread;  // queries with K <= KT: one thread each (0 = none)
    const bool all_small = KT > 0 && K <= KT;  // K bounds every per-query kq
    const unsigned blocks = (unsigned)((nq + KW - 1) / KW);
    const uint32_t* perm = (const uint32_t*)c->perm.p;
    const SubGrid grid = {(const InstPar*)c->inst.d_par.p, (const uint16_t*)c->inst.d_inst_e.p,
                          (const uint8_t*)c->bin_lvl.p, (const uint32_t*)c->sub_off.p,
                          (const uint32_t*)c->sub_start.p};
    const int2* tab = (const int2*)c->knn_table.p;
    // queries whose packed-key search met a tie, for the exact-key search at the end
    uint32_t* redo = ensure<uint32_t>(c->knn_redo, (size_t)nq, &e);
    if (e) return e;
    if ((e = cudaMemsetAsync(&sc->knn_redo, 0, sizeof(unsigned), c->stream))) return e;
    int launches = 0;
    if (KT > 0) {
        const unsigned tblocks = (unsigned)((nq + KNN_T_THREADS - 1) / KNN_T_THREADS);
        const size_t smem = (size_t)std::min(K, KT) * KNN_T_THREADS * sizeof(unsigned long long);
#define PGPU_KNN_T(DD, PT)                                                                                    \
    k_knn_t<DD><<<tblocks, KNN_T_THREADS, smem, c->stream>>>((const PT*)c->spts.p, perm, grid, tab,            \
                                                              c->knn_table_n, c->knn_table_r, qs, nq, K, KT, kq, \
                                                              stride, out, &sc->knn_cand, redo, &sc->knn_redo)
        if (c->prm.dim == 2) PGPU_KNN_T(2, double2); else PGPU_KNN_T(3, double4);
#undef PGPU_KNN_T
        launches++;
    }
    if (!all_small) {
        const int skip = KT > 0 ? std::min(K, KT) : 0;  // the queries k_knn_t did
#define PGPU_KNN(DD, PT, WW)                                                                                 \
    k_knn<DD, WW><<<blocks, WW * 32, 0, c->stream>>>((const PT*)c->spts.p, perm, grid, tab, c->knn_table_n,     \
                                                      c->knn_table_r, qs, nq, K, kq, stride, out, &sc->knn_cand, \
                                                      skip, redo, &sc->knn_redo)
        // one query per block (at most 32 blocks, so 32 warps, per SM) frees each warp's slot as
        // soon as its own query is done; two or more allow 40 warps per SM: the autotuner picks
        if (c->prm.dim == 2) {
            if (KW == 1) PGPU_KNN(2, double2, 1); else if (KW == 2) PGPU_KNN(2, double2, 2); else if (KW == 8) PGPU_KNN(2, double2, 8); else PGPU_KNN(2, double2, 4);
        } else {
            if (KW == 1) PGPU_KNN(3, double4, 1); else if (KW == 2) PGPU_KNN(3, double4, 2); else if (KW == 8) PGPU_KNN(3, double4, 8); else PGPU_KNN(3, double4, 4);
        }
#undef PGPU_KNN
        launches++;
    }
    // the tied queries again with exact keys: a fixed grid whose warps stride over the
    // device-held list (no read-back of its length)
    const unsigned xblocks = (unsigned)std::min<int64_t>(blocks, 148 * 4);
#define PGPU_KNNX(DD, PT, WW)                                                                                   \
    k_knn_exact<DD, WW><<<xblocks, WW * 32, 0, c->stream>>>((const PT*)c->spts.p, perm, grid, tab,               \
                                                             c->knn_table_n, c->knn_table_r, qs, K, kq, stride,  \
                                                             out, &sc->knn_cand, redo, &sc->knn_redo,            \
                                                             &sc->knn_redo_total)
    if (c->prm.dim == 2) {
        if (KW == 2) PGPU_KNNX(2, double2, 2); else if (KW == 8) PGPU_KNNX(2, double2, 8); else PGPU_KNNX(2, double2, 4);
    } else {
        if (KW == 2) PGPU_KNNX(3, double4, 2); else if (KW == 8) PGPU_KNNX(3, double4, 8); else PGPU_KNNX(3, double4, 4);
    }
#undef PGPU_KNNX
    count_launches(launches + 1);
    return cudaGetLastError();
}

cudaError_t launch_knn(pgpu_ctx* c) {
    cudaError_t e = cudaSuccess;
    const int K = c->use_kq ? c->knn_stride : c->prm.k;
    if (!c->use_kq) c->knn_stride = K;
    uint32_t* out = ensure<uint32_t>(c->knn, (size_t)c->n_query * K + 1, &e);
    if (e) return e;
    DevScalars* sc = (DevScalars*)c->scalars.p;
    if ((e = cudaMemsetAsync(&sc->knn_cand, 0, sizeof(unsigned long long), c->stream))) return e;
    if ((e = cudaMemsetAsync(&sc->knn_redo_total, 0, sizeof(unsigned), c->stream))) return e;
    return launch_knn_list(c, (const uint32_t*)c->qs.p, c->n_query, K, out,
                           c->use_kq ? (const uint16_t*)c->kq.p : nullptr, K);
}

}  // namespace pgpu
