// Device -> reference layout conversions, run only when a caller asks for host
// copies (the drop-in entry points and the tests).
//
// k_gather_faces replaces voronoi::unpermute_vmesh (src/voronoi/voronoi.cpp:212-333):
// the extraction writes each cell's faces contiguously at a reserved slot; this
// rebuilds the reference's CSR layout (cells in input order, face_ptr = prefix
// sum of face_counts).  Neighbour ids are already input ids.
#include "pgpu_common.cuh"
#include "pgpu_ctx.h"

namespace pgpu {
namespace {

inline unsigned nblk(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

__global__ void k_gather_faces(const uint32_t* __restrict__ fptr, const uint32_t* __restrict__ fcnt,
                               const uint32_t* __restrict__ new_ptr, const int32_t* __restrict__ f_nb,
                               const double4* __restrict__ f_geo, int64_t n, int32_t* __restrict__ nb_out,
                               double* __restrict__ nrm_out, double* __restrict__ area_out) {
    // one warp per cell
    const int64_t e = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (e >= n) return;
    const uint32_t src = fptr[e], cnt = fcnt[e], dst = new_ptr[e];
    for (uint32_t q = lane; q < cnt; q += 32) {
        const double4 g = f_geo[src + q];
        nb_out[dst + q] = f_nb[src + q];
        nrm_out[3 * (size_t)(dst + q)] = g.x;
        nrm_out[3 * (size_t)(dst + q) + 1] = g.y;
        nrm_out[3 * (size_t)(dst + q) + 2] = g.z;
        area_out[dst + q] = g.w;
    }
}

// VMesh seeds: the unit-box point scaled back, (s - 0.5) * scale + 0.5
// (periodic_mesh.cpp:146-166); 3 doubles per cell, z = 0 in 2D.  As in the
// reference, only extracted cells carry their seed (cell.cpp:418-420); the
// others hold the scaled-back zero.
template <int D>
__global__ void k_seeds(const typename PointOf<D>::type* __restrict__ ext, const int* __restrict__ status,
                        int64_t n, const InstPar* __restrict__ ip, const uint16_t* __restrict__ inst, int no_scale,
                        double* __restrict__ out) {
    int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    const double scale = ip[inst[e]].scale_out;
    const typename PointOf<D>::type p = ext[e];
    const bool ok = status[e] == ST_SUCCESS;
    double c[3] = {ok ? p.x : 0.0, ok ? p.y : 0.0, ok ? pz(p) : 0.0};
    for (int a = 0; a < 3; a++) out[3 * e + a] = (a < D && !no_scale) ? (c[a] - 0.5) * scale + 0.5 : c[a];
}

__global__ void k_knn_rows(const uint32_t* __restrict__ knn, const uint32_t* __restrict__ qs,
                           const uint32_t* __restrict__ perm, int64_t nq, int K, uint32_t* __restrict__ out) {
    const int64_t t = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (t >= nq) return;
    const uint32_t q = perm[qs[t]];
    for (int j = lane; j < K; j += 32) out[(size_t)q * K + j] = knn[(size_t)t * K + j];
}

template <int D>
__global__ void k_unpack_points(const typename PointOf<D>::type* __restrict__ p, int64_t n, double* __restrict__ out) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    out[i * D] = p[i].x;
    out[i * D + 1] = p[i].y;
    if (D == 3) out[i * D + 2] = pz(p[i]);
}

// One thread per sampled query slot t: its extended id, the neighbour row the
// main clip used (kq[t] ids, or K) padded to W ids, and the cell's outputs.
__global__ void k_sample_cells(const uint32_t* __restrict__ slots, int64_t n, int64_t n_query,
                               const uint32_t* __restrict__ qs, const uint32_t* __restrict__ perm,
                               const uint32_t* __restrict__ knn, int stride, int K, int W,
                               const uint16_t* __restrict__ kq,
                               const int* __restrict__ status, const int* __restrict__ certk,
                               const double* __restrict__ vol, const double* __restrict__ cen,
                               const uint32_t* __restrict__ fcnt, uint32_t* __restrict__ ext_out,
                               uint16_t* __restrict__ len_out, uint32_t* __restrict__ rows_out,
                               int32_t* __restrict__ st_out, int32_t* __restrict__ ck_out,
                               double* __restrict__ vol_out, double* __restrict__ cen_out,
                               uint32_t* __restrict__ fc_out) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t t = slots[i];
    if ((int64_t)t >= n_query) {  // rejected on the host; kept as a guard
        ext_out[i] = NO_NEIGHBOR;
        fc_out[i] = 0;
        return;
    }
    const uint32_t e = perm[qs[t]];
    const int len = kq ? min((int)kq[t], K) : K;
    ext_out[i] = e;
    len_out[i] = (uint16_t)len;
    for (int j = 0; j < W; j++) rows_out[(size_t)i * W + j] = j < len ? knn[(size_t)t * stride + j] : NO_NEIGHBOR;
    st_out[i] = status[e];
    ck_out[i] = certk[e];
    vol_out[i] = vol[e];
    for (int a = 0; a < 3; a++) cen_out[3 * i + a] = cen[3 * (size_t)e + a];
    fc_out[i] = status[e] == ST_SUCCESS ? fcnt[e] : 0u;
}

// One warp per sampled cell: its faces, in stored order, at dst_ptr[i].
__global__ void k_sample_faces(const uint32_t* __restrict__ ext_ids, const uint32_t* __restrict__ fc,
                               const uint64_t* __restrict__ dst_ptr, int64_t n, const uint32_t* __restrict__ fptr,
                               const int32_t* __restrict__ f_nb, const double4* __restrict__ f_geo,
                               int32_t* __restrict__ nb_out, double* __restrict__ nrm_out,
                               double* __restrict__ area_out) {
    const int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (i >= n) return;
    const uint32_t cnt = fc[i];
    if (cnt == 0) return;
    const uint32_t src = fptr[ext_ids[i]];
    const uint64_t dst = dst_ptr[i];
    for (uint32_t q = lane; q < cnt; q += 32) {
        const double4 g = f_geo[src + q];
        nb_out[dst + q] = f_nb[src + q];
        nrm_out[3 * (dst + q)] = g.x;
        nrm_out[3 * (dst + q) + 1] = g.y;
        nrm_out[3 * (dst + q) + 2] = g.z;
        area_out[dst + q] = g.w;
    }
}

}  // namespace

cudaError_t launch_sample_cells(pgpu_ctx* c, const uint32_t* slots, int64_t n, uint32_t* ext_out, uint16_t* len_out,
                                uint32_t* rows_out, int32_t* st_out, int32_t* ck_out, double* vol_out,
                                double* cen_out, uint32_t* fc_out) {
    if (n <= 0) return cudaSuccess;
    k_sample_cells<<<nblk(n, 128), 128, 0, c->stream>>>(
        slots, n, c->n_query, (const uint32_t*)c->qs.p, (const uint32_t*)c->perm.p, (const uint32_t*)c->knn.p,
        c->knn_stride, c->use_kq ? c->knn_stride : c->prm.k, c->prm.k,
        c->use_kq ? (const uint16_t*)c->kq.p : nullptr,
        (const int*)c->status.p, (const int*)c->certk.p, (const double*)c->vol.p, (const double*)c->centroid.p,
        (const uint32_t*)c->fcnt.p, ext_out, len_out, rows_out, st_out, ck_out, vol_out, cen_out, fc_out);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_sample_faces(pgpu_ctx* c, const uint32_t* ext_ids, const uint32_t* fc, const uint64_t* dst_ptr,
                                int64_t n, int32_t* nb_out, double* nrm_out, double* area_out) {
    if (n <= 0) return cudaSuccess;
    k_sample_faces<<<nblk(n * 32, 256), 256, 0, c->stream>>>(ext_ids, fc, dst_ptr, n, (const uint32_t*)c->fptr.p,
                                                            (const int32_t*)c->f_nb.p, (const double4*)c->f_geo.p,
                                                            nb_out, nrm_out, area_out);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_mesh_compact(pgpu_ctx* c, uint32_t* new_ptr, int32_t* nb_out, double* nrm_out, double* area_out) {
    const int64_t n = c->n_ext;
    cudaError_t e = exclusive_scan_u32((const uint32_t*)c->fcnt.p, new_ptr, n, c->scan_tmp, c->stream);
    if (e) return e;
    if (n > 0)
        k_gather_faces<<<nblk(n * 32, 256), 256, 0, c->stream>>>(
            (const uint32_t*)c->fptr.p, (const uint32_t*)c->fcnt.p, new_ptr, (const int32_t*)c->f_nb.p,
            (const double4*)c->f_geo.p, n, nb_out, nrm_out, area_out);
    if (n > 0) count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_seeds(pgpu_ctx* c, double* out, bool no_scale) {
    const int64_t n = c->n_ext;
    if (n <= 0) return cudaSuccess;
    if (c->prm.dim == 2)
        k_seeds<2><<<nblk(n, 256), 256, 0, c->stream>>>((const double2*)c->ext.p, (const int*)c->status.p, n,
                                                        (const InstPar*)c->inst.d_par.p,
                                                        (const uint16_t*)c->inst.d_inst_e.p, no_scale, out);
    else
        k_seeds<3><<<nblk(n, 256), 256, 0, c->stream>>>((const double4*)c->ext.p, (const int*)c->status.p, n,
                                                        (const InstPar*)c->inst.d_par.p,
                                                        (const uint16_t*)c->inst.d_inst_e.p, no_scale, out);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_knn_rows(pgpu_ctx* c, uint32_t* out) {
    const int64_t nq = c->n_query;
    if (nq <= 0) return cudaSuccess;
    k_knn_rows<<<nblk(nq * 32, 256), 256, 0, c->stream>>>((const uint32_t*)c->knn.p, (const uint32_t*)c->qs.p,
                                                           (const uint32_t*)c->perm.p, nq, c->prm.k, out);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_unpack_points(pgpu_ctx* c, const void* pts, int64_t n, double* out) {
    if (n <= 0) return cudaSuccess;
    if (c->prm.dim == 2)
        k_unpack_points<2><<<nblk(n, 256), 256, 0, c->stream>>>((const double2*)pts, n, out);
    else
        k_unpack_points<3><<<nblk(n, 256), 256, 0, c->stream>>>((const double4*)pts, n, out);
    count_launches(1);
    return cudaGetLastError();
}

}  // namespace pgpu
