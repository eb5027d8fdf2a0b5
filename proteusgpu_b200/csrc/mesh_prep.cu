// Mesh inputs on the device: ghost layer + unit-box scaling, Morton-ordered
// grid sort, and the list of cells to compute.
//
// Ghosts restate src/voronoi/periodic_mesh.cpp:63-126: for every hydro point,
// the 8 (2D) or 26 (3D) boundary regions are tested in the reference's order,
// which numbers the ghosts (ghost ids appear as face neighbours).  A count
// pass, a prefix sum and a write pass place each point's ghosts after all hydro
// points, exactly where the reference's serial append puts them.
//
// The grid sort replaces knn::sort_points_into_grid (src/knn/knn.cpp:119-154):
// points are binned on a uniform grid whose bins are numbered in Morton order,
// so that spatially close bins are close in memory; a histogram, a prefix sum
// and a scatter produce the sorted points and the sorted -> extended-id map.
#include "pgpu_common.cuh"
#include "pgpu_ctx.h"

namespace pgpu {
namespace {

// Shift vectors of the ghost regions in the order of periodic_mesh.cpp:71-79
// (2D) and :83-110 (3D); a +1 shift selects the open interval (0, buff) on that
// axis, -1 selects (1 - buff, 1), 0 selects (0, 1).
__constant__ int8_t c_reg2[8][2] = {{1, 0}, {0, -1}, {-1, 0}, {0, 1}, {1, 1}, {1, -1}, {-1, -1}, {-1, 1}};
__constant__ int8_t c_reg3[26][3] = {
    {0, 0, 1},  {1, 0, 0},   {0, -1, 0},  {-1, 0, 0}, {0, 1, 0},  {0, 0, -1}, {0, 1, 1},   {1, 0, 1},   {0, -1, 1},
    {-1, 0, 1}, {1, 1, 0},   {1, -1, 0},  {-1, -1, 0}, {-1, 1, 0}, {1, 0, -1}, {0, -1, -1}, {-1, 0, -1}, {0, 1, -1},
    {1, 1, 1},  {1, -1, 1},  {-1, -1, 1}, {-1, 1, 1}, {1, 1, -1}, {1, -1, -1}, {-1, -1, -1}, {-1, 1, -1}};

template <int D>
__device__ __forceinline__ int shift_of(int r, int a) {
    return D == 2 ? c_reg2[r][a] : c_reg3[r][a];
}

template <int D>
__device__ __forceinline__ bool in_region(const double* p, int r, double buff) {
#pragma unroll
    for (int a = 0; a < D; a++) {
        int s = shift_of<D>(r, a);
        double lo = s > 0 ? 0. : (s < 0 ? 1. - buff : 0.);
        double hi = s > 0 ? 0. + buff : 1.;
        if (!(p[a] > lo && p[a] < hi)) return false;
    }
    return true;
}

template <int D>
__global__ void k_ghost_count(const double* __restrict__ pos, int64_t n, const uint16_t* __restrict__ inst,
                              const InstPar* __restrict__ ip, uint32_t* __restrict__ cnt) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double buff = ip[inst[i]].buff;
    double p[D];
#pragma unroll
    for (int a = 0; a < D; a++) p[a] = pos[i * D + a];
    constexpr int NR = D == 2 ? 8 : 26;
    uint32_t c = 0;
    for (int r = 0; r < NR; r++) c += in_region<D>(p, r, buff) ? 1u : 0u;
    cnt[i] = c;
}

template <int D>
__global__ void k_ghost_write(const double* __restrict__ pos, int64_t n, const uint16_t* __restrict__ inst,
                              const InstPar* __restrict__ ip, int no_ghosts, const uint32_t* __restrict__ goff,
                              typename PointOf<D>::type* __restrict__ ext, uint32_t* __restrict__ gsrc,
                              uint32_t* __restrict__ gcode, uint16_t* __restrict__ inst_e) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint16_t b = inst[i];
    const InstPar par = ip[b];
    const double buff = par.buff, scale = par.scale_in;
    const int mirror = par.mirror;
    double p[D];
#pragma unroll
    for (int a = 0; a < D; a++) p[a] = pos[i * D + a];
    inst_e[i] = b;
    if (no_ghosts) {  // compute_mesh: points are used as given
        ext[i] = make_pt<D>(p[0], p[1], D == 3 ? p[D - 1] : 0.0);
        return;
    }
    // scale into [0,1]^D: scale * (x - 0.5) + 0.5 (periodic_mesh.cpp:119-126)
    double q[3] = {0, 0, 0};
#pragma unroll
    for (int a = 0; a < D; a++) q[a] = scale * (p[a] - 0.5) + 0.5;
    ext[i] = make_pt<D>(q[0], q[1], q[2]);
    constexpr int NR = D == 2 ? 8 : 26;
    uint32_t k = goff[i];
    for (int r = 0; r < NR; r++) {
        if (!in_region<D>(p, r, buff)) continue;
        double g[3] = {0, 0, 0};
        uint32_t code = 0, mul = 1;
#pragma unroll
        for (int a = 0; a < D; a++) {
            int s = shift_of<D>(r, a);
            if (!mirror)
                g[a] = p[a] + (double)s;  // add_ghost (periodic_mesh.cpp:28-33)
            else
                g[a] = s > 0 ? -p[a] : (s < 0 ? 2.0 - p[a] : p[a]);
            code += (s == 0 ? 0u : (s > 0 ? 1u : 2u)) * mul;
            mul *= 3;
        }
#pragma unroll
        for (int a = 0; a < D; a++) g[a] = scale * (g[a] - 0.5) + 0.5;
        ext[n + k] = make_pt<D>(g[0], g[1], g[2]);
        inst_e[n + k] = b;
        gsrc[k] = (uint32_t)i;
        gcode[k] = code;
        k++;
    }
}

template <int D>
__global__ void k_bin_count(const typename PointOf<D>::type* __restrict__ ext, int64_t n,
                            const uint16_t* __restrict__ inst_e, const InstPar* __restrict__ ip,
                            uint32_t* __restrict__ key, uint32_t* __restrict__ cnt) {
    int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    typename PointOf<D>::type p = ext[e];
    const InstPar& par = ip[inst_e[e]];
    const int G = par.G;
    uint32_t k = par.slot0 + morton<D>(bin_coord(p.x, G), bin_coord(p.y, G), D == 3 ? bin_coord(pz(p), G) : 0);
    key[e] = k;
    atomicAdd(&cnt[k], 1u);
}

// Refinement level of each coarse bin: dense bins (clustered inputs) are split
// into (2^L)^D sub-bins so that the search works at the local point spacing.
template <int D>
__global__ void k_bin_levels(const uint32_t* __restrict__ cnt, int64_t M, uint8_t* __restrict__ lvl,
                             uint32_t* __restrict__ size) {
    const int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= M) return;
    const uint32_t c = cnt[m];
    int L = 0;
    if (c > SUB_SPLIT)
        while (L < SUB_LMAX && (uint64_t)c > (uint64_t)SUB_FILL << (D * L)) L++;
    lvl[m] = (uint8_t)L;
    size[m] = 1u << (D * L);
}

// Sub-bin slot of every point (overwrites its coarse key) and the slot counts.
template <int D>
__global__ void k_sub_count(const typename PointOf<D>::type* __restrict__ ext, int64_t n,
                            const uint16_t* __restrict__ inst_e, const InstPar* __restrict__ ip,
                            const uint8_t* __restrict__ lvl, const uint32_t* __restrict__ sub_off,
                            uint32_t* __restrict__ key, uint32_t* __restrict__ sub_cnt) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    const typename PointOf<D>::type p = ext[e];
    const int G = ip[inst_e[e]].G;
    const uint32_t b = key[e];
    const int L = lvl[b];
    uint32_t slot = sub_off[b];
    if (L > 0) {
        const int lx = sub_coord(p.x, G, L) - (bin_coord(p.x, G) << L);
        const int ly = sub_coord(p.y, G, L) - (bin_coord(p.y, G) << L);
        const int lz = D == 3 ? sub_coord(pz(p), G, L) - (bin_coord(pz(p), G) << L) : 0;
        slot += morton<D>(lx, ly, lz);
    }
    key[e] = slot;
    atomicAdd(&sub_cnt[slot], 1u);
}

// Points of each sub-bin in ascending extended id (the scatter's atomics leave
// them in arbitrary order), so that every walk over a sub-bin is deterministic.
// Sub-bins of more points than this are sorted by a block each (k_sub_sort_big);
// the smaller ones, nearly all, by one thread.
constexpr uint32_t SUBSORT_THREAD_MAX = 64;
constexpr uint32_t SUBSORT_SMEM_KEYS = 8192;  // larger ones sort their keys in global scratch

template <int D>
__global__ void k_sub_sort(const uint32_t* __restrict__ sub_start, int64_t T,
                           typename PointOf<D>::type* __restrict__ spts, uint32_t* __restrict__ perm,
                           uint32_t* __restrict__ inv, uint32_t* __restrict__ big, unsigned int* __restrict__ n_big) {
    const int64_t slot = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (slot >= T) return;
    const uint32_t a = sub_start[slot], b = sub_start[slot + 1];
    if (b - a < 2) return;
    if (b - a > SUBSORT_THREAD_MAX) {  // gas piled beyond the deepest refinement level
        big[atomicAdd(n_big, 1u)] = (uint32_t)slot;
        return;
    }
    for (uint32_t i = a + 1; i < b; i++) {
        const uint32_t id = perm[i];
        const typename PointOf<D>::type pt = spts[i];
        uint32_t j = i;
        while (j > a && perm[j - 1] > id) {
            perm[j] = perm[j - 1];
            spts[j] = spts[j - 1];
            j--;
        }
        perm[j] = id;
        spts[j] = pt;
    }
    for (uint32_t i = a; i < b; i++) inv[perm[i]] = i;
}

// Ascending sort of n keys by one block: the bitonic network in the form whose
// compare-exchanges all put the smaller key first (a mirrored stage, then
// half-cleaners, per merge size), on n rounded up to a power of two with the
// missing keys taken as +inf -- they never move, so they need no storage.
__device__ void block_sort_u64(unsigned long long* k, uint32_t n) {
    uint32_t P = 1;
    while (P < n) P <<= 1;
    for (uint32_t size = 2; size <= P; size <<= 1) {
        for (uint32_t t = threadIdx.x; t < P / 2; t += blockDim.x) {
            const uint32_t half = size / 2, blk = t / half, off = t % half;
            const uint32_t lo = blk * size + off, hi = blk * size + size - 1 - off;
            if (hi < n && k[hi] < k[lo]) {
                const unsigned long long x = k[lo];
                k[lo] = k[hi];
                k[hi] = x;
            }
        }
        __syncthreads();
        for (uint32_t j = size / 4; j > 0; j >>= 1) {
            for (uint32_t t = threadIdx.x; t < P / 2; t += blockDim.x) {
                const uint32_t lo = (t / j) * 2 * j + t % j, hi = lo + j;
                if (hi < n && k[hi] < k[lo]) {
                    const unsigned long long x = k[lo];
                    k[lo] = k[hi];
                    k[hi] = x;
                }
            }
            __syncthreads();
        }
    }
}

// The large sub-bins listed by k_sub_sort, a block each: keys (id, position in the
// sub-bin) sorted in shared memory (or, beyond SUBSORT_SMEM_KEYS, in the scratch at
// the sub-bin's own range), then ids and points put in that order through a copy.
template <int D>
__global__ void __launch_bounds__(256)
    k_sub_sort_big(const uint32_t* __restrict__ sub_start, const uint32_t* __restrict__ big,
                   const unsigned int* __restrict__ n_big, typename PointOf<D>::type* __restrict__ spts,
                   uint32_t* __restrict__ perm, uint32_t* __restrict__ inv, unsigned long long* __restrict__ keys,
                   typename PointOf<D>::type* __restrict__ tmp) {
    extern __shared__ unsigned long long sk[];
    const unsigned nb = *n_big;
    for (unsigned i = blockIdx.x; i < nb; i += gridDim.x) {
        const uint32_t slot = big[i];
        const uint32_t a = sub_start[slot], m = sub_start[slot + 1] - a;
        unsigned long long* k = m <= SUBSORT_SMEM_KEYS ? sk : keys + a;
        for (uint32_t j = threadIdx.x; j < m; j += blockDim.x) {
            k[j] = ((unsigned long long)perm[a + j] << 32) | j;
            tmp[a + j] = spts[a + j];
        }
        __syncthreads();
        block_sort_u64(k, m);
        for (uint32_t j = threadIdx.x; j < m; j += blockDim.x) {
            const unsigned long long key = k[j];
            const uint32_t id = (uint32_t)(key >> 32);
            perm[a + j] = id;
            spts[a + j] = tmp[a + (uint32_t)(key & 0xffffffffull)];
            inv[id] = a + j;
        }
        __syncthreads();
    }
}

// Point range of each coarse bin from the sub-bin starts.
__global__ void k_bin_from_sub(const uint32_t* __restrict__ sub_off, const uint32_t* __restrict__ sub_start,
                               int64_t M, uint32_t* __restrict__ bin_start) {
    const int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (m <= M) bin_start[m] = sub_start[sub_off[m]];
}

template <int D>
__global__ void k_bin_scatter(const typename PointOf<D>::type* __restrict__ ext, int64_t n,
                              const uint32_t* __restrict__ key, const uint32_t* __restrict__ start,
                              uint32_t* __restrict__ fill, typename PointOf<D>::type* __restrict__ spts,
                              uint32_t* __restrict__ perm, uint32_t* __restrict__ inv) {
    int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    uint32_t k = key[e];
    uint32_t s = start[k] + atomicAdd(&fill[k], 1u);
    spts[s] = ext[e];
    perm[s] = (uint32_t)e;
    inv[e] = s;
}

__global__ void k_query_flags(const uint32_t* __restrict__ perm, int64_t n_ext, int64_t n_hydro,
                              uint32_t* __restrict__ flag) {
    int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n_ext) return;
    flag[s] = perm[s] < (uint32_t)n_hydro ? 1u : 0u;
}

__global__ void k_query_compact(const uint32_t* __restrict__ flag, const uint32_t* __restrict__ off, int64_t n_ext,
                                uint32_t* __restrict__ qs) {
    int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n_ext) return;
    if (flag[s]) qs[off[s]] = (uint32_t)s;
}

__global__ void k_iota(uint32_t* __restrict__ q, int64_t n) {
    int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s < n) q[s] = (uint32_t)s;
}

inline unsigned nblk(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

__global__ void k_fill_inst(uint16_t* __restrict__ inst, const int64_t* __restrict__ hydro0, int nb, int64_t n) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int lo = 0, hi = nb - 1;  // last instance whose first hydro id is <= i
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (hydro0[mid] <= i) lo = mid; else hi = mid - 1;
    }
    inst[i] = (uint16_t)lo;
}

__global__ void k_gather_u32(const uint32_t* __restrict__ src, const int64_t* __restrict__ idx, int n,
                             uint32_t* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = src[idx[i]];
}

}  // namespace

static cudaError_t upload_par(pgpu_ctx* c) {
    Instances& I = c->inst;
    cudaError_t e = cudaSuccess;
    InstPar* d = ensure<InstPar>(I.d_par, I.n, &e);
    if (e) return e;
    return cudaMemcpyAsync(d, I.par.data(), I.n * sizeof(InstPar), cudaMemcpyHostToDevice, c->stream);
}

static cudaError_t setup_instances(pgpu_ctx* c, int nb, const int64_t* counts, const double* buff,
                                   const double* gamma, const int* mirror) {
    Instances& I = c->inst;
    I.n = nb;
    I.count.assign(counts, counts + nb);
    I.hydro0.assign(nb + 1, 0);
    for (int b = 0; b < nb; b++) I.hydro0[b + 1] = I.hydro0[b] + counts[b];
    I.par.assign(nb, InstPar{});
    for (int b = 0; b < nb; b++) {
        InstPar& q = I.par[b];
        q.buff = buff[b];
        q.scale_in = 1. / (1. + (2 * buff[b]));
        q.scale_out = 1. + (2 * buff[b]);
        q.gamma = gamma[b];
        q.mirror = mirror[b];
        q.count = (uint32_t)counts[b];
    }
    const int64_t n = I.hydro0[nb];
    cudaError_t e = cudaSuccess;
    uint16_t* ih = ensure<uint16_t>(I.d_inst_h, n + 1, &e);
    ensure<unsigned long long>(I.d_dt, nb + 1, &e);
    if (e) return e;
    if (nb == 1) {
        if ((e = cudaMemsetAsync(ih, 0, (n + 1) * sizeof(uint16_t), c->stream))) return e;
    } else if (n > 0) {
        int64_t* h0 = ensure<int64_t>(I.d_gather, nb + 1, &e);
        if (e) return e;
        if ((e = cudaMemcpyAsync(h0, I.hydro0.data(), (nb + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, c->stream)))
            return e;
        k_fill_inst<<<nblk(n, 256), 256, 0, c->stream>>>(ih, h0, nb, n);
        count_launches(1);
        if ((e = cudaStreamSynchronize(c->stream))) return e;  // d_gather is reused below
    }
    return upload_par(c);
}

cudaError_t set_single_instance(pgpu_ctx* c, int64_t n) {
    const int mir = c->prm.boundary == PGPU_REFLECTIVE;
    return setup_instances(c, 1, &n, &c->prm.buff, &c->prm.gamma, &mir);
}

cudaError_t set_instances(pgpu_ctx* c, int nb, const int64_t* counts, const double* buff, const double* gamma,
                          const int* boundary) {
    std::vector<int> mir(nb);
    for (int b = 0; b < nb; b++) mir[b] = boundary[b] == PGPU_REFLECTIVE;
    return setup_instances(c, nb, counts, buff, gamma, mir.data());
}

cudaError_t launch_ghosts(pgpu_ctx* c, const double* pos_dev, int64_t n, bool no_ghosts) {
    const int D = c->prm.dim;
    cudaError_t e = cudaSuccess;
    Instances& I = c->inst;
    if (I.hydro0.empty() || I.hydro0[I.n] != n) return cudaErrorInvalidValue;  // instances not set for n points
    const InstPar* ip = (const InstPar*)I.d_par.p;
    const uint16_t* ih = (const uint16_t*)I.d_inst_h.p;
    int64_t ng = 0;
    std::vector<int64_t> ext_count(I.count);
    if (!no_ghosts) {
        uint32_t* cnt = ensure<uint32_t>(c->gcnt, n + 1, &e);
        uint32_t* off = ensure<uint32_t>(c->goff, n + 1, &e);
        if (e) return e;
        if (n > 0) {
            if (D == 2)
                k_ghost_count<2><<<nblk(n, 256), 256, 0, c->stream>>>(pos_dev, n, ih, ip, cnt);
            else
                k_ghost_count<3><<<nblk(n, 256), 256, 0, c->stream>>>(pos_dev, n, ih, ip, cnt);
        }
        if (n > 0) count_launches(1);
        if ((e = exclusive_scan_u32(cnt, off, n, c->scan_tmp, c->stream))) return e;
        // ghost offsets at every instance's first point (the last entry is the total)
        std::vector<uint32_t> at(I.n + 1, 0);
        if (I.n == 1) {
            if ((e = cudaMemcpyAsync(&at[1], off + n, sizeof(uint32_t), cudaMemcpyDeviceToHost, c->stream))) return e;
        } else {
            int64_t* idx = ensure<int64_t>(I.d_gather, 2 * (I.n + 1) + 2, &e);
            if (e) return e;
            uint32_t* outv = (uint32_t*)(idx + I.n + 1);
            if ((e = cudaMemcpyAsync(idx, I.hydro0.data(), (I.n + 1) * sizeof(int64_t), cudaMemcpyHostToDevice,
                                     c->stream)))
                return e;
            k_gather_u32<<<nblk(I.n + 1, 256), 256, 0, c->stream>>>(off, idx, I.n + 1, outv);
            count_launches(1);
            if ((e = cudaMemcpyAsync(at.data(), outv, (I.n + 1) * sizeof(uint32_t), cudaMemcpyDeviceToHost,
                                     c->stream)))
                return e;
        }
        if ((e = cudaStreamSynchronize(c->stream))) return e;
        ng = at[I.n];
        for (int b = 0; b < I.n; b++) ext_count[b] += (int64_t)at[b + 1] - (int64_t)at[b];
    }
    c->n_hydro = n;
    c->n_ext = n + ng;
    I.ext_count = ext_count;
    const size_t pt_bytes = D == 2 ? 16 : 32;
    if ((e = ensure_bytes(c->ext, (size_t)(c->n_ext + 1) * pt_bytes))) return e;
    ensure<uint32_t>(c->ghost_src, ng + 1, &e);
    ensure<uint32_t>(c->ghost_code, ng + 1, &e);
    uint16_t* ie = ensure<uint16_t>(I.d_inst_e, c->n_ext + 1, &e);
    if (e) return e;
    if (n > 0) {
        const uint32_t* off = (const uint32_t*)c->goff.p;
        if (D == 2)
            k_ghost_write<2><<<nblk(n, 256), 256, 0, c->stream>>>(pos_dev, n, ih, ip, no_ghosts, off,
                                                                  (double2*)c->ext.p, (uint32_t*)c->ghost_src.p,
                                                                  (uint32_t*)c->ghost_code.p, ie);
        else
            k_ghost_write<3><<<nblk(n, 256), 256, 0, c->stream>>>(pos_dev, n, ih, ip, no_ghosts, off,
                                                                  (double4*)c->ext.p, (uint32_t*)c->ghost_src.p,
                                                                  (uint32_t*)c->ghost_code.p, ie);
    }
    if (n > 0) count_launches(1);
    if (no_ghosts)
        for (auto& q : I.par) q.scale_out = 1.0;  // compute_mesh: no unit-box scaling
    c->unit_scale = I.par[0].scale_out;
    return cudaGetLastError();
}

// Grid resolution: about ppb points per coarse bin (autotuned; 2 by default).
static int grid_resolution(int64_t n, int D, double ppb) {
    double g = D == 2 ? sqrt((double)n / ppb) : cbrt((double)n / ppb);
    int G = (int)(g + 0.5);
    if (G < 1) G = 1;
    const int gmax = D == 2 ? 32768 : 1024;
    return G > gmax ? gmax : G;
}

// Two-level counting sort: coarse Morton bins, each split into Morton-ordered
// sub-bins when dense, so that every coarse bin and every aligned block of its
// sub-bins is one contiguous range of the sorted points.
cudaError_t launch_grid_sort(pgpu_ctx* c) {
    const int D = c->prm.dim;
    const int64_t n = c->n_ext;
    cudaError_t e = cudaSuccess;
    // one grid per instance, sized by its own point count; their Morton slots follow each other
    Instances& I = c->inst;
    int64_t M = 0;
    for (int b = 0; b < I.n; b++) {
        const int Gb = grid_resolution(I.ext_count[b], D, c->tune.ppb);
        int64_t P = 1;
        while (P < Gb) P <<= 1;
        I.par[b].G = Gb;
        I.par[b].slot0 = (uint32_t)M;
        M += D == 2 ? P * P : P * P * P;
    }
    if (M >= (1ll << 32)) return cudaErrorInvalidValue;
    if ((e = upload_par(c))) return e;
    const InstPar* ip = (const InstPar*)I.d_par.p;
    const uint16_t* ie = (const uint16_t*)I.d_inst_e.p;
    c->grid_G = I.par[0].G;
    c->morton_slots = M;
    uint32_t* cnt = ensure<uint32_t>(c->bin_cnt, M + 1, &e);
    uint32_t* start = ensure<uint32_t>(c->bin_start, M + 1, &e);
    uint32_t* key = ensure<uint32_t>(c->bin_key, n + 1, &e);
    uint8_t* lvl = ensure<uint8_t>(c->bin_lvl, M + 1, &e);
    uint32_t* soff = ensure<uint32_t>(c->sub_off, M + 1, &e);
    const size_t pt_bytes = D == 2 ? 16 : 32;
    if (e || (e = ensure_bytes(c->spts, (size_t)(n + 1) * pt_bytes))) return e;
    uint32_t* perm = ensure<uint32_t>(c->perm, n + 1, &e);
    uint32_t* inv = ensure<uint32_t>(c->inv, n + 1, &e);
    if (e) return e;
    if ((e = cudaMemsetAsync(cnt, 0, (M + 1) * sizeof(uint32_t), c->stream))) return e;
    if (n > 0) {
        if (D == 2)
            k_bin_count<2><<<nblk(n, 256), 256, 0, c->stream>>>((const double2*)c->ext.p, n, ie, ip, key, cnt);
        else
            k_bin_count<3><<<nblk(n, 256), 256, 0, c->stream>>>((const double4*)c->ext.p, n, ie, ip, key, cnt);
        count_launches(1);
    }
    // levels, sub-table offsets (one slot per coarse bin at level 0)
    if (D == 2)
        k_bin_levels<2><<<nblk(M, 256), 256, 0, c->stream>>>(cnt, M, lvl, start);
    else
        k_bin_levels<3><<<nblk(M, 256), 256, 0, c->stream>>>(cnt, M, lvl, start);
    count_launches(1);
    if ((e = exclusive_scan_u32(start, soff, M, c->scan_tmp, c->stream))) return e;
    uint32_t T = 0;
    if ((e = cudaMemcpyAsync(&T, soff + M, sizeof(T), cudaMemcpyDeviceToHost, c->stream))) return e;
    if ((e = cudaStreamSynchronize(c->stream))) return e;
    c->sub_slots = T;
    uint32_t* scnt = ensure<uint32_t>(c->sub_cnt, (size_t)T + 1, &e);
    uint32_t* sstart = ensure<uint32_t>(c->sub_start, (size_t)T + 1, &e);
    if (e) return e;
    if ((e = cudaMemsetAsync(scnt, 0, ((size_t)T + 1) * sizeof(uint32_t), c->stream))) return e;
    if (n > 0) {
        if (D == 2)
            k_sub_count<2><<<nblk(n, 256), 256, 0, c->stream>>>((const double2*)c->ext.p, n, ie, ip, lvl, soff, key,
                                                                scnt);
        else
            k_sub_count<3><<<nblk(n, 256), 256, 0, c->stream>>>((const double4*)c->ext.p, n, ie, ip, lvl, soff, key,
                                                                scnt);
        count_launches(1);
    }
    if ((e = exclusive_scan_u32(scnt, sstart, T, c->scan_tmp, c->stream))) return e;
    k_bin_from_sub<<<nblk(M + 1, 256), 256, 0, c->stream>>>(soff, sstart, M, start);
    count_launches(1);
    if ((e = cudaMemsetAsync(scnt, 0, ((size_t)T + 1) * sizeof(uint32_t), c->stream))) return e;
    if (n > 0) {
        if (D == 2)
            k_bin_scatter<2><<<nblk(n, 256), 256, 0, c->stream>>>((const double2*)c->ext.p, n, key, sstart, scnt,
                                                                  (double2*)c->spts.p, perm, inv);
        else
            k_bin_scatter<3><<<nblk(n, 256), 256, 0, c->stream>>>((const double4*)c->ext.p, n, key, sstart, scnt,
                                                                  (double4*)c->spts.p, perm, inv);
        DevScalars* sc = (DevScalars*)c->scalars.p;
        uint32_t* big = ensure<uint32_t>(c->sort_big, (size_t)T + 1, &e);
        if (e) return e;
        if ((e = cudaMemsetAsync(&sc->sort_big, 0, sizeof(unsigned int), c->stream))) return e;
        if (D == 2)
            k_sub_sort<2><<<nblk(T, 256), 256, 0, c->stream>>>(sstart, T, (double2*)c->spts.p, perm, inv, big,
                                                               &sc->sort_big);
        else
            k_sub_sort<3><<<nblk(T, 256), 256, 0, c->stream>>>(sstart, T, (double4*)c->spts.p, perm, inv, big,
                                                               &sc->sort_big);
        count_launches(2);
        unsigned int nbig = 0;
        if ((e = cudaMemcpyAsync(&nbig, &sc->sort_big, sizeof(nbig), cudaMemcpyDeviceToHost, c->stream))) return e;
        if ((e = cudaStreamSynchronize(c->stream))) return e;
        if (nbig > 0) {
            const size_t psz = D == 2 ? sizeof(double2) : sizeof(double4);
            unsigned long long* keys = ensure<unsigned long long>(c->sort_keys, (size_t)n + 1, &e);
            void* tmp = ensure<unsigned char>(c->sort_pts, ((size_t)n + 1) * psz, &e);
            if (e) return e;
            const unsigned grid = nbig < 296u ? nbig : 296u;
            const size_t smem = SUBSORT_SMEM_KEYS * sizeof(unsigned long long);
            if (D == 2) {
                if ((e = cudaFuncSetAttribute(k_sub_sort_big<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)))
                    return e;
                k_sub_sort_big<2><<<grid, 256, smem, c->stream>>>(sstart, big, &sc->sort_big, (double2*)c->spts.p,
                                                                  perm, inv, keys, (double2*)tmp);
            } else {
                if ((e = cudaFuncSetAttribute(k_sub_sort_big<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)))
                    return e;
                k_sub_sort_big<3><<<grid, 256, smem, c->stream>>>(sstart, big, &sc->sort_big, (double4*)c->spts.p,
                                                                  perm, inv, keys, (double4*)tmp);
            }
            count_launches(1);
        }
    }
    return cudaGetLastError();
}

cudaError_t launch_query_list(pgpu_ctx* c, bool all_cells) {
    cudaError_t e = cudaSuccess;
    const int64_t n = c->n_ext;
    uint32_t* qs = ensure<uint32_t>(c->qs, n + 1, &e);
    if (e) return e;
    c->all_cells = all_cells;
    if (all_cells || c->n_hydro == n) {
        c->n_query = n;
        if (n > 0) {
            k_iota<<<nblk(n, 256), 256, 0, c->stream>>>(qs, n);
            count_launches(1);
        }
        return cudaGetLastError();
    }
    uint32_t* flag = ensure<uint32_t>(c->qflag, n + 1, &e);
    uint32_t* off = ensure<uint32_t>(c->qoff, n + 1, &e);
    if (e) return e;
    k_query_flags<<<nblk(n, 256), 256, 0, c->stream>>>((const uint32_t*)c->perm.p, n, c->n_hydro, flag);
    if ((e = exclusive_scan_u32(flag, off, n, c->scan_tmp, c->stream))) return e;
    k_query_compact<<<nblk(n, 256), 256, 0, c->stream>>>(flag, off, n, qs);
    count_launches(2);
    c->n_query = c->n_hydro;
    return cudaGetLastError();
}

}  // namespace pgpu
