// Voronoi cells by half-space clipping with the security-radius certificate,
// fused with the extraction of faces, areas, volumes and centroids
// (replaces cpu_compute_cell + ConvexCell + extract_cell_to_vmesh,
// src/voronoi/voronoi.cpp:115-155, src/voronoi/cell.cpp:42-669; the method is
// Ray, Sokolov, Lefebvre, Levy, "Meshless Voronoi on the GPU", ACM TOG 2018).
//
// One warp per cell.  The cell lives in shared memory in dual form: planes
// (a, b, c, d) and vertices as plane triples (pairs in 2D), consistently
// oriented.  Per clipping plane:
//   1. every lane tests its vertices against the plane with the reference's
//      determinant predicate and error bound (cell.cpp:175-221);
//   2. the cavity boundary is the set of edges of removed vertices whose twin
//      belongs to a kept vertex (3D: one key match over the removed vertices'
//      edges, or a 64x64 edge bit matrix for large cavities; 2D: the two lines
//      used once), checked to be a single cycle; one new vertex (plane, x, y)
//      per boundary edge x -> y, which is the vertex the reference's boundary
//      walk (cell.cpp:224-364) creates for that edge;
//   3. kept vertices are compacted in order and new ones appended, each with
//      its squared distance to the seed cached for the certificate
//      (cell.cpp:369-384), whose maximum is a warp reduction.
// Predicates, vertex coordinates and plane equations use the reference's
// expansions without FMA, so every decision, and the mesh topology, equal the
// reference's.  Vertex order inside a cell differs, which changes face-area
// and volume rounding only (3D); 2D edge lengths are bit-identical.
//
// Extraction: faces are the planes with >= D vertices, in plane order (box
// planes first, then neighbours in clipping order).  Each lane builds one
// face polygon by following the triangle orientation around its plane, and
// sums the fan area and the divergence-theorem volume as cell.cpp:582-631
// does.  A cell's faces are written contiguously at a slot reserved with one
// atomic add; placement varies run to run, contents do not.
#include <math_constants.h>

#include <type_traits>

#include "pgpu_common.cuh"
#include "pgpu_ctx.h"

namespace pgpu {
namespace {

constexpr int CLIP_WARPS = 4;
constexpr unsigned FULL = 0xffffffffu;
constexpr int FACE_MAX_V = 32;  // vertices per face polygon handled by one lane

struct WarpCell {
    double4 hp[MAX_P];
    int vid[MAX_P];
    uint32_t tri[MAX_T];
    union {
        struct {
            double vd2[MAX_T];
            double fvol[MAX_P];      // per-face volume contribution (3D) for an ordered sum
            double fcen[MAX_P][3];   // per-face centroid moment (3D)
        };
        struct {                     // k_clip32 while clipping
            float4 V32[MAX_T];       // homogeneous vertex coordinates (rx, ry, rz, rw)
            float2 P32[MAX_T];       // bounds of their rounding: (largest permanent of the x, y, z
                                     // cofactors' minors, permanent of the w cofactor's)
            float D32[MAX_T];        // squared distance of the vertex to the seed
        };
    };
    union {
        struct {
            unsigned long long emask[MAX_P];
            unsigned char nxt[MAX_P];
            float4 hp32[MAX_P];   // FP32 local-frame planes (k_clip32)
            uint32_t stage[MAX_P];  // new vertices of the current cut, in their final order
            double stage_d2[MAX_P]; // and their squared distances to the seed (FP64 clip)
        } b;
        double vpos[MAX_T][3];
    } u;
};

// k_clip32's cell in 3D: the FP32 clipping arrays and the FP64 extraction arrays share
// memory (clipping is over when extraction begins): 6.9 KB a warp instead of 7.9 KB,
// for 32 resident warps per SM.
struct WarpCell32 {
    int vid[MAX_P];
    uint32_t tri[MAX_T];
    union {
        struct {  // FP32 clipping
            float4 hp32[MAX_P];
            float4 V32[MAX_T];
            float2 P32[MAX_T];
            float D32[MAX_T];
            unsigned long long emask[MAX_P];
            uint32_t stage[MAX_P];
            uint32_t rl[MAX_T];
            unsigned char nxt[MAX_P];
            float4 sb_eq[32];  // the current batch of neighbour planes (local frame)
            float sb_d2[32];   // their squared distances to the seed
            uint32_t sb_z[32]; // their ext ids
        } c;
        struct {  // FP64 extraction
            double4 hp[MAX_P];
            double vpos[MAX_T][3];
            double fvol[MAX_P];
            double fcen[MAX_P][3];
        } x;
    };
};

// Member access shared by the kernels' two cell layouts.
__device__ __forceinline__ double4* hp_of(WarpCell& W) { return W.hp; }
__device__ __forceinline__ double4* hp_of(WarpCell32& W) { return W.x.hp; }
__device__ __forceinline__ double (*vpos_of(WarpCell& W))[3] { return W.u.vpos; }
__device__ __forceinline__ double (*vpos_of(WarpCell32& W))[3] { return W.x.vpos; }
__device__ __forceinline__ uint32_t* rl_of(WarpCell& W) { return reinterpret_cast<uint32_t*>(W.u.b.stage_d2); }
__device__ __forceinline__ uint32_t* rl_of(WarpCell32& W) { return W.c.rl; }
__device__ __forceinline__ uint32_t* stage_of(WarpCell& W) { return W.u.b.stage; }
__device__ __forceinline__ uint32_t* stage_of(WarpCell32& W) { return W.c.stage; }
__device__ __forceinline__ unsigned long long* emask_of(WarpCell& W) { return W.u.b.emask; }
__device__ __forceinline__ unsigned long long* emask_of(WarpCell32& W) { return W.c.emask; }
__device__ __forceinline__ unsigned char* nxt_of(WarpCell& W) { return W.u.b.nxt; }
__device__ __forceinline__ unsigned char* nxt_of(WarpCell32& W) { return W.c.nxt; }
__device__ __forceinline__ double* fvol_of(WarpCell& W) { return W.fvol; }
__device__ __forceinline__ double* fvol_of(WarpCell32& W) { return W.x.fvol; }
__device__ __forceinline__ double (*fcen_of(WarpCell& W))[3] { return W.fcen; }
__device__ __forceinline__ double (*fcen_of(WarpCell32& W))[3] { return W.x.fcen; }
__device__ __forceinline__ float4* hp32_of(WarpCell& W) { return W.u.b.hp32; }
__device__ __forceinline__ float4* hp32_of(WarpCell32& W) { return W.c.hp32; }
__device__ __forceinline__ float4* V32_of(WarpCell& W) { return W.V32; }
__device__ __forceinline__ float4* V32_of(WarpCell32& W) { return W.c.V32; }
__device__ __forceinline__ float2* P32_of(WarpCell& W) { return W.P32; }
__device__ __forceinline__ float2* P32_of(WarpCell32& W) { return W.c.P32; }
__device__ __forceinline__ float* D32_of(WarpCell& W) { return W.D32; }
__device__ __forceinline__ float* D32_of(WarpCell32& W) { return W.c.D32; }
__device__ __forceinline__ const float* D32_of(const WarpCell& W) { return W.D32; }
__device__ __forceinline__ const float* D32_of(const WarpCell32& W) { return W.c.D32; }

__device__ __forceinline__ uint32_t tri_a(uint32_t t) { return t & 255u; }
__device__ __forceinline__ uint32_t tri_b(uint32_t t) { return (t >> 8) & 255u; }
__device__ __forceinline__ uint32_t tri_c(uint32_t t) { return (t >> 16) & 255u; }
__device__ __forceinline__ uint32_t pack3(uint32_t a, uint32_t b, uint32_t c) { return a | (b << 8) | (c << 16); }

// compute_vertex_point with the perspective divide (cell.cpp:388-411)
template <int D>
__device__ __forceinline__ void vertex_pos(const double4* hp, uint32_t t, double& x, double& y, double& z) {
    const double4 p1 = hp[tri_a(t)], p2 = hp[tri_b(t)];
    if (D == 2) {
        double rx = -det2(p1.w, p1.y, p2.w, p2.y);
        double ry = -det2(p1.x, p1.w, p2.x, p2.w);
        double rw = det2(p1.x, p1.y, p2.x, p2.y);
        x = rx / rw;
        y = ry / rw;
        z = 0.0;
    } else {
        const double4 p3 = hp[tri_c(t)];
        double rx = -det3(p1.w, p1.y, p1.z, p2.w, p2.y, p2.z, p3.w, p3.y, p3.z);
        double ry = -det3(p1.x, p1.w, p1.z, p2.x, p2.w, p2.z, p3.x, p3.w, p3.z);
        double rz = -det3(p1.x, p1.y, p1.w, p2.x, p2.y, p2.w, p3.x, p3.y, p3.w);
        double rw = det3(p1.x, p1.y, p1.z, p2.x, p2.y, p2.z, p3.x, p3.y, p3.z);
        x = rx / rw;
        y = ry / rw;
        z = rz / rw;
    }
}

// squared distance to the seed as is_security_radius_reached computes it
__device__ __forceinline__ double seed_d2(double x, double y, double z, double sx, double sy, double sz) {
    double dx = x - sx, dy = y - sy, dz = z - sz;
    return dx * dx + dy * dy + dz * dz;
}

__device__ __forceinline__ double fmax3(double a, double b, double c) {
    double m = a > b ? a : b;
    return m > c ? m : c;
}

// vert_is_in_conflict (cell.cpp:175-221): returns det > 0, sets *near when |det| < eps.
// In robust mode a near-zero determinant keeps the vertex (not cut) instead.
template <int D>
__device__ __forceinline__ bool in_conflict(const double4* hp, uint32_t t, const double4& e, bool* near,
                                            bool robust) {
    const double4 p1 = hp[tri_a(t)], p2 = hp[tri_b(t)];
    double det, eps;
    if (D == 2) {
        det = det3(p1.x, p2.x, e.x, p1.y, p2.y, e.y, p1.w, p2.w, e.w);
        double maxx = fmax3(fabs(p1.x), fabs(p2.x), fabs(e.x));
        double maxy = fmax3(fabs(p1.y), fabs(p2.y), fabs(e.y));
        double maxw = fmax3(fabs(p1.w), fabs(p2.w), fabs(e.w));
        double max_max = fmax3(maxx, maxy, maxw);
        eps = 1e-14 * maxx * maxy * maxw;
        eps *= max_max;
    } else {
        const double4 p3 = hp[tri_c(t)];
        det = det4(p1.x, p2.x, p3.x, e.x, p1.y, p2.y, p3.y, e.y, p1.z, p2.z, p3.z, e.z, p1.w, p2.w, p3.w, e.w);
        double maxx = fmax3(fmax3(fabs(p1.x), fabs(p2.x), fabs(p3.x)), fabs(e.x), 0.0);
        double maxy = fmax3(fmax3(fabs(p1.y), fabs(p2.y), fabs(p3.y)), fabs(e.y), 0.0);
        double maxz = fmax3(fmax3(fabs(p1.z), fabs(p2.z), fabs(p3.z)), fabs(e.z), 0.0);
        eps = 1e-14 * maxx * maxy * maxz;
        double max_max = fmax3(maxx, maxy, maxz);
        eps *= (max_max * max_max);
    }
    if (fabs(det) < eps) {
        if (robust) return false;
        *near = true;
    }
    return det > 0.0;
}

// Maximum that propagates NaN: a vertex with w = 0 (three planes sharing a line,
// which mirror-symmetric point sets produce) has no position, and a cell holding
// one must not pass the certificate.  The reference's running std::max
// (cell.cpp:377) keeps or drops such a NaN depending on vertex order.
__device__ __forceinline__ double nan_max(double a, double b) { return (a != a || b != b) ? (a + b) : fmax(a, b); }

__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = nan_max(v, __shfl_xor_sync(FULL, v, o));
    return v;
}

__device__ __forceinline__ double max_vd2(const WarpCell& W, int n, int lane, const uint32_t* keep_mask) {
    double m = 0.0;
#pragma unroll
    for (int j = 0; j < 3; j++) {
        int i = lane + 32 * j;
        if (i < n && (keep_mask == nullptr || ((keep_mask[j] >> lane) & 1u))) m = nan_max(m, W.vd2[i]);
    }
    return warp_max(m);
}

struct ClipParams {
    const uint32_t* qs;
    const uint32_t* slots;  // optional: work item t is query slot slots[t] (lists of qs/knn reused)
    const uint32_t* perm;
    const void* spts;
    const void* ext;
    const uint32_t* knn;
    const uint16_t* kq;     // optional: neighbour budget of query slot t (<= K, the list stride)
    const uint32_t* ghost_src;
    const uint32_t* ghost_code;
    int64_t nq;
    int64_t n_hydro;
    int K;
    int robust;
    unsigned int* uncertified;  // hydro cells ending with SECURITY_RADIUS_NOT_REACHED
    unsigned int* reclip;       // cells the FP32 kernel hands to the FP64 kernel
    const InstPar* ip;      // per instance: unit box -> physical scale (scale_out)
    const uint16_t* inst;   // instance of each extended id
    double* vol;
    uint32_t* fptr;
    uint32_t* fcnt;
    int* status;
    int* certk;
    double* centroid;  // 3 per cell
    int32_t* f_nb;
    uint32_t* f_own;
    double4* f_geo;
    unsigned long long* face_counter;
    unsigned long long* walk_stats;  // grid walk: points clipped, boxes visited
    unsigned int* overflow;
    unsigned long long face_cap;
    int walk_prefix;  // grid walk: list neighbours clipped before the walk (same in every form)
    int walk_certk;   // grid walk: certified K reported for walked cells
};

// Cell outputs of a cell that was not extracted (the reference leaves volume 0
// and no faces, voronoi.cpp:150-152).
__device__ __forceinline__ void store_failed(const ClipParams& P, int lane, uint32_t e, int status) {
    if (lane == 0) {
        if (status == ST_SECURITY_RADIUS_NOT_REACHED && (int64_t)e < P.n_hydro) atomicAdd(P.uncertified, 1u);
        P.vol[e] = 0.0;
        P.fptr[e] = 0;
        P.fcnt[e] = 0;
        P.status[e] = status;
        P.certk[e] = 0;
        P.centroid[3 * (size_t)e] = P.centroid[3 * (size_t)e + 1] = P.centroid[3 * (size_t)e + 2] = 0.0;
    }
}

// Extraction (cell.cpp:416-669) of a certified cell held in W with FP64 planes:
// vertices, faces in plane order, areas, volume, centroid; faces written at a
// reserved slot, cell outputs at extended id e.
template <int D, class Cell>
__device__ __forceinline__ void compute_vpos(Cell& W, int lane, int nb_t) {
    __syncwarp();
    double (*vp)[3] = vpos_of(W);
#pragma unroll
    for (int j = 0; j < 3; j++) {
        int i = lane + 32 * j;
        if (i < nb_t) vertex_pos<D>(hp_of(W), W.tri[i], vp[i][0], vp[i][1], vp[i][2]);
    }
    __syncwarp();
}

template <int D, class Cell>
__device__ __forceinline__ void extract_and_store(Cell& W, const ClipParams& P, int w, int lane, int nb_v, int nb_t,
                                                  uint32_t e, int certk, double sx, double sy, double sz,
                                                  bool vpos_ready = false, double ox = 0.0, double oy = 0.0,
                                                  double oz = 0.0) {
    // (ox, oy, oz): origin of the frame the cell was clipped in, added to the centroid
    if (!vpos_ready) compute_vpos<D>(W, lane, nb_t);
    double (*vp)[3] = vpos_of(W);

    double cell_vol = 0.0, cen[3] = {0.0, 0.0, 0.0};
    if constexpr (D == 2) {
        // compute_cell_area_2d (cell.cpp:475-498): vertices ordered by angle about their mean
        double cx = 0, cy = 0;
        for (int i = 0; i < nb_t; i++) cx += vp[i][0], cy += vp[i][1];
        cx /= nb_t;
        cy /= nb_t;
        // rank of each vertex by angle; lane-parallel, then lane 0 sums in order
        __shared__ unsigned char order_s[CLIP_WARPS][MAX_T];
#pragma unroll
        for (int j = 0; j < 3; j++) {
            int i = lane + 32 * j;
            if (i < nb_t) W.vd2[i] = atan2(vp[i][1] - cy, vp[i][0] - cx);
        }
        __syncwarp();
#pragma unroll
        for (int j = 0; j < 3; j++) {
            int i = lane + 32 * j;
            if (i < nb_t) {
                const double ai = W.vd2[i];
                int rank = 0;
                for (int q = 0; q < nb_t; q++) {
                    const double aq = W.vd2[q];
                    rank += (aq < ai || (aq == ai && q < i)) ? 1 : 0;
                }
                order_s[w][rank] = (unsigned char)i;
            }
        }
        __syncwarp();
        if (lane == 0) {
            double a = 0, mx = 0, my = 0, sa = 0;
            for (int i = 0; i < nb_t; i++) {
                int j = (i + 1) % nb_t;
                const double* pp = vp[order_s[w][i]];
                const double* qq = vp[order_s[w][j]];
                a += pp[0] * qq[1];
                a -= qq[0] * pp[1];
                double cr = (pp[0] - cx) * (qq[1] - cy) - (qq[0] - cx) * (pp[1] - cy);
                mx += (pp[0] + qq[0] - 2 * cx) * cr;
                my += (pp[1] + qq[1] - 2 * cy) * cr;
                sa += cr;
            }
            cell_vol = fabs(a) / 2.0;
            cen[0] = cx + mx / (3.0 * sa);
            cen[1] = cy + my / (3.0 * sa);
        }
    }

    // faces: lane handles planes p = lane and p = lane + 32
    bool valid[2] = {false, false};
    double area[2] = {0.0, 0.0};
    double* fvol = fvol_of(W);
    double (*fcen)[3] = fcen_of(W);
#pragma unroll
    for (int pass = 0; pass < 2; pass++) {
        const int p = lane + 32 * pass;
        if (p >= nb_v) continue;
        if (D == 2) {
            int cnt = 0, v0 = -1, v1 = -1;
            for (int i = 0; i < nb_t; i++) {
                uint32_t tv = W.tri[i];
                if ((int)tri_a(tv) == p || (int)tri_b(tv) == p) {
                    if (cnt == 0) v0 = i; else if (cnt == 1) v1 = i;
                    cnt++;
                }
            }
            if (cnt >= 2) {
                double ddx = vp[v1][0] - vp[v0][0];
                double ddy = vp[v1][1] - vp[v0][1];
                area[pass] = sqrt(ddx * ddx + ddy * ddy);
                valid[pass] = true;
            }
        } else {
            unsigned char fa[FACE_MAX_V], fb[FACE_MAX_V], fi[FACE_MAX_V];
            int cnt = 0;
            bool over = false;
            for (int i = 0; i < nb_t; i++) {
                uint32_t tv = W.tri[i];
                uint32_t a = tri_a(tv), b = tri_b(tv), c = tri_c(tv);
                uint32_t x, y;
                if ((int)a == p) x = b, y = c;
                else if ((int)b == p) x = c, y = a;
                else if ((int)c == p) x = a, y = b;
                else continue;
                if (cnt < FACE_MAX_V) {
                    fa[cnt] = (unsigned char)x;
                    fb[cnt] = (unsigned char)y;
                    fi[cnt] = (unsigned char)i;
                } else {
                    over = true;
                }
                cnt++;
            }
            double fv = 0.0, fc0 = 0.0, fc1 = 0.0, fc2 = 0.0;
            if (cnt >= 3 && !over) {
                // Walk the polygon: after vertex (p, a, b) comes (p, b, c).  Fan
                // triangles (v0, v_{i-1}, v_i) give the area and, with the seed,
                // the signed volume and first moment (cell.cpp:611-627).
                const double* v0 = vp[fi[0]];
                const double a0 = v0[0] - sx, a1 = v0[1] - sy, a2 = v0[2] - sz;
                int curv = 0;
                double meas = 0.0;
                bool ok = true;
                for (int st = 1; st < cnt; st++) {
                    int nx = -1;
                    for (int q = 1; q < cnt; q++)
                        if (fa[q] == fb[curv]) {
                            nx = q;
                            break;
                        }
                    if (nx < 0) {
                        ok = false;
                        break;
                    }
                    if (st >= 2) {
                        const double* vi = vp[fi[curv]];
                        const double* vj = vp[fi[nx]];
                        double e1x = vi[0] - v0[0], e1y = vi[1] - v0[1], e1z = vi[2] - v0[2];
                        double e2x = vj[0] - v0[0], e2y = vj[1] - v0[1], e2z = vj[2] - v0[2];
                        double crx = e1y * e2z - e1z * e2y;
                        double cry = e1z * e2x - e1x * e2z;
                        double crz = e1x * e2y - e1y * e2x;
                        meas += 0.5 * sqrt(crx * crx + cry * cry + crz * crz);
                        double b0 = vi[0] - sx, b1 = vi[1] - sy, b2 = vi[2] - sz;
                        double c0 = vj[0] - sx, c1 = vj[1] - sy, c2 = vj[2] - sz;
                        double x0 = b1 * c2 - b2 * c1;
                        double x1 = b2 * c0 - b0 * c2;
                        double x2 = b0 * c1 - b1 * c0;
                        double tv = (a0 * x0 + a1 * x1 + a2 * x2) / 6.0;
                        fv += tv;
                        fc0 += tv * (a0 + b0 + c0) * 0.25;
                        fc1 += tv * (a1 + b1 + c1) * 0.25;
                        fc2 += tv * (a2 + b2 + c2) * 0.25;
                    }
                    curv = nx;
                }
                if (ok && fb[curv] != fa[0]) ok = false;  // the walk must close on v0
                if (ok) {
                    valid[pass] = true;
                    area[pass] = meas;
                }
            }
            fvol[p] = valid[pass] ? fv : 0.0;
            fcen[p][0] = valid[pass] ? fc0 : 0.0;
            fcen[p][1] = valid[pass] ? fc1 : 0.0;
            fcen[p][2] = valid[pass] ? fc2 : 0.0;
        }
    }
    const uint32_t vb0 = __ballot_sync(FULL, valid[0]);
    const uint32_t vb1 = __ballot_sync(FULL, valid[1]);
    const int nf = __popc(vb0) + __popc(vb1);
    __syncwarp();
    if (D == 3 && lane == 0) {
        for (int p = 0; p < nb_v; p++) {  // plane order, as the reference accumulates
            cell_vol += fvol[p];
            cen[0] += fcen[p][0];
            cen[1] += fcen[p][1];
            cen[2] += fcen[p][2];
        }
        const double sv = cell_vol;
        cell_vol = fabs(sv);
        cen[0] = sx + cen[0] / sv;
        cen[1] = sy + cen[1] / sv;
        cen[2] = sz + cen[2] / sv;
    }
    // unit box -> physical: the cell's instance's 1 + 2 buff
    const double uscale = P.ip[P.inst[e]].scale_out;
    const double vscale = D == 2 ? uscale * uscale : uscale * uscale * uscale;
    const double ascale = D == 2 ? uscale : uscale * uscale;
    unsigned long long base = 0;
    if (lane == 0) base = atomicAdd(P.face_counter, (unsigned long long)nf);
    base = __shfl_sync(FULL, base, 0);
    const bool fits = base + (unsigned long long)nf <= P.face_cap;
    if (!fits) {
        if (lane == 0) atomicOr(P.overflow, 1u);
    } else {
#pragma unroll
        for (int pass = 0; pass < 2; pass++) {
            if (!valid[pass]) continue;
            const int p = lane + 32 * pass;
            const uint32_t vb = pass == 0 ? vb0 : vb1;
            const int idx = (pass == 0 ? 0 : __popc(vb0)) + __popc(vb & ((1u << lane) - 1u));
            const size_t f = base + idx;
            const double4 pe = hp_of(W)[p];
            const double nlen = sqrt(pe.x * pe.x + pe.y * pe.y + pe.z * pe.z);  // compute_face_normal
            const int nbr = W.vid[p];
            P.f_nb[f] = nbr;
            uint32_t own = BOX_FACE;
            if (nbr >= 0) {
                if ((int64_t)nbr < P.n_hydro)
                    own = pack_owner((uint32_t)nbr, 0);
                else
                    own = pack_owner(P.ghost_src[nbr - P.n_hydro], P.ghost_code[nbr - P.n_hydro]);
            }
            P.f_own[f] = own;
            P.f_geo[f] = make_double4(pe.x / nlen, pe.y / nlen, pe.z / nlen, ascale * area[pass]);
        }
    }
    if (lane == 0) {
        P.vol[e] = vscale * cell_vol;
        P.fptr[e] = fits ? (uint32_t)base : 0u;
        P.fcnt[e] = fits ? (uint32_t)nf : 0u;
        P.status[e] = ST_SUCCESS;
        P.certk[e] = certk;
        P.centroid[3 * (size_t)e] = (cen[0] + ox - 0.5) * uscale + 0.5;
        P.centroid[3 * (size_t)e + 1] = (cen[1] + oy - 0.5) * uscale + 0.5;
        P.centroid[3 * (size_t)e + 2] = D == 3 ? (cen[2] + oz - 0.5) * uscale + 0.5 : 0.0;
    }
}

// Cavity boundary of a 3D cut: the removed vertices are the triangles flagged in
// cm (nb_r of nb_t); a boundary edge is an edge of a removed triangle whose twin
// triangle is kept.  Each gives a new vertex (cur, x, y), staged in the order of
// the removed vertices and then of their three edges.  The removed triangles are
// first listed in order; with at most 32 of their edges, an edge is interior when
// its undirected key occurs twice (once per adjacent triangle, __match_any_sync),
// else the directed edges are marked in the per-plane rows of emask.  Returns the
// number of new vertices; src gets the OR of their first planes and, with
// WANT_NXT, nxt[x] = y (for the FP64 kernel's cycle check).
template <bool WANT_NXT, class Cell>
__device__ __forceinline__ int cavity_boundary3(Cell& W, int lane, const uint32_t (&cm)[3], int nb_t, int nb_r,
                                                uint32_t cur, unsigned long long& src) {
    uint32_t* rl = rl_of(W);  // removed triangles (scratch: MAX_T u32)
    uint32_t* stage = stage_of(W);
    unsigned long long* em = emask_of(W);
    int before = 0;
#pragma unroll
    for (int j = 0; j < 3; j++) {
        const int i = lane + 32 * j;
        if (i < nb_t && ((cm[j] >> lane) & 1u)) rl[before + __popc(cm[j] & ((1u << lane) - 1u))] = W.tri[i];
        before += __popc(cm[j]);
    }
    __syncwarp();
    const int ne = 3 * nb_r;
    const bool by_match = ne <= 32;
    if (!by_match) {
        for (int q = lane; q < ne; q += 32) {
            const int r = q / 3, ed = q - 3 * r;
            const uint32_t tv = rl[r];
            const uint32_t x = (tv >> (8 * ed)) & 255u, y = (tv >> (8 * (ed == 2 ? 0 : ed + 1))) & 255u;
            atomicOr(&em[x], 1ull << y);
        }
        __syncwarp();
    }
    int base = 0;
    uint32_t slo = 0u, shi = 0u;
    for (int c0 = 0; c0 < ne; c0 += 32) {
        const int q = c0 + lane;
        const bool valid = q < ne;
        uint32_t x = 0u, y = 0u;
        if (valid) {
            const int r = q / 3, ed = q - 3 * r;
            const uint32_t tv = rl[r];
            x = (tv >> (8 * ed)) & 255u;
            y = (tv >> (8 * (ed == 2 ? 0 : ed + 1))) & 255u;
        }
        bool isb;
        if (by_match) {
            // every lane takes part in the match (lanes without an edge carry a unique key)
            const uint32_t key = valid ? ((min(x, y) << 8) | max(x, y)) : (0x10000u | (uint32_t)lane);
            const unsigned same = __match_any_sync(FULL, key);
            isb = valid && __popc(same) == 1;
        } else {
            isb = valid && !((em[y] >> x) & 1ull);
        }
        const unsigned bal = __ballot_sync(FULL, isb);
        if (isb) {
            const int pos = base + __popc(bal & ((1u << lane) - 1u));
            if (pos < MAX_P) stage[pos] = pack3(cur, x, y);
            if (x < 32u) slo |= 1u << x; else shi |= 1u << (x - 32u);
            if (WANT_NXT) nxt_of(W)[x] = (unsigned char)y;
        }
        base += __popc(bal);
    }
    slo = __reduce_or_sync(FULL, slo);
    shi = __reduce_or_sync(FULL, shi);
    src = ((unsigned long long)shi << 32) | slo;
    if (!by_match) {
        __syncwarp();
        for (int q = lane; q < ne; q += 32) {
            const int r = q / 3, ed = q - 3 * r;
            em[(rl[r] >> (8 * ed)) & 255u] = 0ull;
        }
    }
    __syncwarp();
    return base;
}

// One step of ConvexCell::clip_by_plane (cell.cpp:120-205) in FP64: the
// bisector of the seed and ext point z = (bx, by, bz).  CLIP_FAIL sets status
// (and the vertex distance the final certificate uses); CLIP_NONE leaves the
// cell unchanged; CLIP_CUT updates the cell and v_dist.
// REUSE (grid walk only): with all MAX_P plane slots taken, a neighbour plane
// that no vertex uses any more gives its slot to the new plane instead of the
// cell failing with VERTEX_OVERFLOW as the reference does.
constexpr int CLIP_FAIL = -1, CLIP_NONE = 0, CLIP_CUT = 1;

template <int D, bool REUSE = false>
__device__ __forceinline__ int clip_by(WarpCell& W, int lane, uint32_t z, double bx, double by, double bz, double sx,
                                       double sy, double sz, int robust, int& nb_v, int& nb_t, int& status,
                                       double& v_dist, double& fail_vdist) {
    int cur = nb_v;
    if (nb_v >= MAX_P) {  // new_halfplane (cell.cpp:159-162)
        int slot = -1;
        if (REUSE) {
            unsigned long long used = (1ull << (2 * D)) - 1ull;  // the box planes keep their slots
#pragma unroll
            for (int j = 0; j < 3; j++) {
                const int i = lane + 32 * j;
                if (i < nb_t) {
                    const uint32_t tv = W.tri[i];
                    used |= (1ull << tri_a(tv)) | (1ull << tri_b(tv)) | (D == 3 ? (1ull << tri_c(tv)) : 0ull);
                }
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) used |= __shfl_xor_sync(FULL, used, o);
            if (~used) slot = __ffsll((long long)~used) - 1;
        }
        if (slot < 0) {
            status = ST_VERTEX_OVERFLOW;
            fail_vdist = v_dist;
            return CLIP_FAIL;
        }
        cur = slot;
    }
    // new_halfplane: bisector plane (cell.cpp:164-168)
    const double dx = sx - bx, dy = sy - by, dz = sz - bz;
    const double ax = sx + bx, ay = sy + by, az = sz + bz;
    const double dot = ax * dx + ay * dy + az * dz;
    const double4 eq = make_double4(dx, dy, dz, -dot / 2.0);
    if (lane == 0) W.hp[cur] = eq;

    // 1. conflicts
    uint32_t cm[3];
    bool near = false;
#pragma unroll
    for (int j = 0; j < 3; j++) {
        int i = lane + 32 * j;
        bool cf = false;
        if (i < nb_t) cf = in_conflict<D>(W.hp, W.tri[i], eq, &near, robust);
        cm[j] = __ballot_sync(FULL, cf);
    }
    const int nb_r = __popc(cm[0]) + __popc(cm[1]) + __popc(cm[2]);
    const uint32_t km[3] = {~cm[0], ~cm[1], ~cm[2]};
    if (__any_sync(FULL, near)) {  // needs_exact_predicates: the reference keeps only the kept vertices
        status = ST_NEEDS_EXACT_PREDICATES;
        fail_vdist = max_vd2(W, nb_t, lane, km);
        return CLIP_FAIL;
    }
    if (nb_r == 0) return CLIP_NONE;  // plane does not cut the cell: dropped (cell.cpp:133-136)
    __syncwarp();  // hp[cur] visible

    // 2. cavity boundary
    const int kept = nb_t - nb_r;
    int n_new = 0;
    bool bad = false;
    uint32_t* stage = W.u.b.stage;  // new vertices, written at their final position
    if (D == 2) {
        uint32_t lo = 0, hi = 0;  // XOR of the lines of removed vertices
#pragma unroll
        for (int j = 0; j < 3; j++) {
            int i = lane + 32 * j;
            if (i < nb_t && ((cm[j] >> lane) & 1u)) {
                uint32_t tv = W.tri[i];
                uint32_t a = tri_a(tv), b = tri_b(tv);
                if (a < 32) lo ^= 1u << a; else hi ^= 1u << (a - 32);
                if (b < 32) lo ^= 1u << b; else hi ^= 1u << (b - 32);
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            lo ^= __shfl_xor_sync(FULL, lo, o);
            hi ^= __shfl_xor_sync(FULL, hi, o);
        }
        unsigned long long xm = (unsigned long long)lo | ((unsigned long long)hi << 32);
        if (__popcll(xm) < 2) {
            bad = true;
        } else {
            int b0 = __ffsll((long long)xm) - 1;
            unsigned long long x2 = xm & (xm - 1);
            int b1 = __ffsll((long long)x2) - 1;
            n_new = 2;
            if (lane < 2) {
                int j = lane == 0 ? b0 : b1;
                const double4 hi_ = W.hp[cur], hj = W.hp[j];
                double rw = det2(hi_.x, hi_.y, hj.x, hj.y);  // new_vertex orientation (cell.cpp:351-359)
                stage[lane] = rw > 0 ? pack3(j, cur, 0) : pack3(cur, j, 0);
            }
        }
    } else {
        unsigned long long src = 0ull;
        n_new = cavity_boundary3<true>(W, lane, cm, nb_t, nb_r, (uint32_t)cur, src);
        // a simple cycle visits each source plane once
        bool ok = __popcll(src) == n_new && n_new >= 3;
        if (ok && lane == 0) {
            int x0 = __ffsll((long long)src) - 1, x = x0;
            for (int st = 1; st <= n_new; st++) {
                x = W.u.b.nxt[x];
                if (!((src >> x) & 1ull) || (x == x0 && st < n_new)) {
                    ok = false;
                    break;
                }
            }
            if (x != x0) ok = false;
        }
        ok = __shfl_sync(FULL, ok ? 1 : 0, 0) != 0;
        bad = !ok;
    }
    if (bad) {
        status = ST_INCONSISTENT_BOUNDARY;
        fail_vdist = max_vd2(W, nb_t, lane, km);
        return CLIP_FAIL;
    }
    // 3. new vertices and their certificate distances, one lane each
    __syncwarp();
    double newmax = 0.0;
    const int n_st = n_new < MAX_P ? n_new : MAX_P;
    for (int q = lane; q < n_st; q += 32) {
        double x, y, zz;
        vertex_pos<D>(W.hp, stage[q], x, y, zz);
        const double d2 = seed_d2(x, y, zz, sx, sy, sz);
        W.u.b.stage_d2[q] = d2;
        newmax = nan_max(newmax, d2);
    }
    if (kept + n_new >= MAX_T) {  // new_vertex overflow (cell.cpp:347-350)
        status = ST_TRIANGLE_OVERFLOW;
        fail_vdist = nan_max(max_vd2(W, nb_t, lane, km), warp_max(newmax));
        return CLIP_FAIL;
    }
    // compaction: kept vertices in order, then the new ones
    uint32_t kt[3];
    double kd[3];
    int kp[3];
    int before = 0;
#pragma unroll
    for (int j = 0; j < 3; j++) {
        const int i = lane + 32 * j;
        const int nvalid = nb_t - 32 * j;
        const uint32_t vm = nvalid >= 32 ? FULL : (nvalid > 0 ? ((1u << nvalid) - 1u) : 0u);
        const uint32_t kmj = km[j] & vm;
        const bool keep = (kmj >> lane) & 1u;
        kt[j] = keep ? W.tri[i] : 0u;
        kd[j] = keep ? W.vd2[i] : 0.0;
        kp[j] = keep ? before + __popc(kmj & ((1u << lane) - 1u)) : -1;
        before += __popc(kmj);
    }
    __syncwarp();
#pragma unroll
    for (int j = 0; j < 3; j++)
        if (kp[j] >= 0) {
            W.tri[kp[j]] = kt[j];
            W.vd2[kp[j]] = kd[j];
        }
    for (int q = lane; q < n_new; q += 32) {
        W.tri[kept + q] = stage[q];
        W.vd2[kept + q] = W.u.b.stage_d2[q];
    }
    if (lane == 0) W.vid[cur] = (int)z;
    if (cur == nb_v) nb_v++;
    nb_t = kept + n_new;
    __syncwarp();
    v_dist = max_vd2(W, nb_t, lane, nullptr);
    return CLIP_CUT;
}

template <int D, int CW>
__global__ void __launch_bounds__(CW * 32) k_clip(ClipParams P) {
    using PT = typename PointOf<D>::type;
    __shared__ WarpCell cells[CW];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int64_t t = (int64_t)blockIdx.x * CW + w;
    if (t >= P.nq) return;  // warp-uniform
    WarpCell& W = cells[w];
    const PT* spts = (const PT*)P.spts;
    const PT* ext = (const PT*)P.ext;
    const int64_t tq = P.slots ? (int64_t)P.slots[t] : t;
    const uint32_t s = P.qs[tq];
    const uint32_t e = P.perm[s];
    const PT sp = spts[s];
    const double sx = sp.x, sy = sp.y, sz = pz(sp);
    const int K = P.kq ? (int)P.kq[tq] : P.K;  // per-cell budget (learned K) within rows of P.K
    const uint32_t* kl = P.knn + (size_t)tq * P.K;

    // ---- ConvexCell::ConvexCell (cell.cpp:42-104): bounding box [-1e-14, 1 + 1e-14]^D
    const double beps = 1e-14;
    const double xmin = -beps, xmax = 1.0 + beps;
    if (lane < 2 * D) {
        double4 pl;
        switch (lane) {
            case 0: pl = make_double4(1.0, 0.0, 0.0, -xmin); break;
            case 1: pl = make_double4(-1.0, 0.0, 0.0, xmax); break;
            case 2: pl = make_double4(0.0, 1.0, 0.0, -xmin); break;
            case 3: pl = make_double4(0.0, -1.0, 0.0, xmax); break;
            case 4: pl = make_double4(0.0, 0.0, 1.0, -xmin); break;
            default: pl = make_double4(0.0, 0.0, -1.0, xmax); break;
        }
        W.hp[lane] = pl;
        W.vid[lane] = -1;
    }
    if (D == 3) {
        W.u.b.emask[lane] = 0ull;
        W.u.b.emask[lane + 32] = 0ull;
    }
    const int ntri0 = D == 2 ? 4 : 8;
    if (lane < ntri0) {
        uint32_t tv;
        if (D == 2) {
            const uint32_t t2[4] = {pack3(2, 0, 0), pack3(1, 2, 0), pack3(3, 1, 0), pack3(0, 3, 0)};
            tv = t2[lane & 3];
        } else {
            const uint32_t t3[8] = {pack3(2, 5, 0), pack3(5, 3, 0), pack3(1, 5, 2), pack3(5, 1, 3),
                                    pack3(4, 2, 0), pack3(4, 0, 3), pack3(2, 4, 1), pack3(4, 3, 1)};
            tv = t3[lane & 7];
        }
        W.tri[lane] = tv;
    }
    __syncwarp();
    if (lane < ntri0) {
        double x, y, z;
        vertex_pos<D>(W.hp, W.tri[lane], x, y, z);
        W.vd2[lane] = seed_d2(x, y, z, sx, sy, sz);
    }
    __syncwarp();
    int nb_v = 2 * D, nb_t = ntri0;
    int status = ST_SUCCESS, certk = 0;
    double v_dist = max_vd2(W, nb_t, lane, nullptr);
    double fail_vdist = 0.0;

    for (int k = 0; k < K; k++) {
        const uint32_t z = kl[k];
        if (z == NO_NEIGHBOR) break;
        const PT B = ext[z];
        const double bx = B.x, by = B.y, bz = pz(B);
        const double d2B = seed_d2(bx, by, bz, sx, sy, sz);  // (B - seed)^2 as cell.cpp:381-382
        if (clip_by<D>(W, lane, z, bx, by, bz, sx, sy, sz, P.robust, nb_v, nb_t, status, v_dist, fail_vdist) ==
            CLIP_FAIL)
            break;
        if (d2B > 4 * v_dist) {  // security radius reached (voronoi.cpp:138)
            certk = k + 1;
            break;
        }
    }
    // final certificate with the K-th neighbour (voronoi.cpp:145-147)
    {
        const double vdf = status == ST_SUCCESS ? v_dist : fail_vdist;
        const uint32_t zK = kl[K - 1];
        if (zK == NO_NEIGHBOR) {
            status = ST_SECURITY_RADIUS_NOT_REACHED;
        } else {
            const PT BK = ext[zK];
            if (!(seed_d2(BK.x, BK.y, pz(BK), sx, sy, sz) > 4 * vdf)) status = ST_SECURITY_RADIUS_NOT_REACHED;
        }
    }
    if (status != ST_SUCCESS) {
        store_failed(P, lane, e, status);
        return;
    }
    extract_and_store<D>(W, P, w, lane, nb_v, nb_t, e, certk, sx, sy, sz);
}


// ============================================================================
// Security-radius clipping without a neighbour budget (extension).  Cells whose
// certificate does not close within the K nearest neighbours -- large cells
// beside dense clumps, whose security sphere holds thousands of clump points --
// are clipped from the head of their own list and then by walking the grid:
// coarse bins in order of their distance lower bound, dense bins descended
// sub-bin by sub-bin, points already clipped from the list skipped.  A box
// is skipped when it lies beyond the security radius (2 sqrt(v_dist)) or when
// no point in it can cut the cell: a point q cuts the convex cell iff some
// vertex v is nearer to q than to the seed, so a box whose distance to every
// vertex exceeds that vertex's distance to the seed holds no cutting point.
// When the walk ends every point within the security radius has been clipped
// or excluded, which is the certificate.  The walk also takes the cells that
// failed for other reasons (predicates the absolute-frame determinants cannot
// decide, plane or vertex overflow): it clips in the seed's local frame and
// reuses plane slots, which removes most of those causes.  Points of a
// sub-bin are clipped in their sorted order (by extended id within the
// sub-bin), so the result is deterministic.
constexpr int PRUNE_STACK = 64;
constexpr int WALK_MAX_BOXES = 1 << 17;   // boxes popped per cell
constexpr int WALK_MAX_POINTS = 1 << 15;  // points clipped per cell

// squared distance from (x, y, z) to the box [lo, lo + side)^D
template <int D>
__device__ __forceinline__ double pt_box_d2(double x, double y, double z, const double (&lo)[3], double side) {
    const double c[3] = {x, y, z};
    double d2 = 0.0;
#pragma unroll
    for (int a = 0; a < D; a++) {
        const double hi = lo[a] + side;
        const double dd = c[a] < lo[a] ? lo[a] - c[a] : (c[a] > hi ? c[a] - hi : 0.0);
        d2 += dd * dd;
    }
    return d2;
}

template <int D>
__global__ void __launch_bounds__(CLIP_WARPS * 32)
    k_clip_pruned(ClipParams P, SubGrid g, const int2* __restrict__ table, int table_n, int table_r) {
    using PT = typename PointOf<D>::type;
    __shared__ WarpCell cells_sm[CLIP_WARPS];
    __shared__ int4 stack_sm[CLIP_WARPS][PRUNE_STACK];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int64_t t = (int64_t)blockIdx.x * CLIP_WARPS + w;
    if (t >= P.nq) return;  // warp-uniform
    WarpCell& W = cells_sm[w];
    int4* stk = stack_sm[w];
    const PT* spts = (const PT*)P.spts;
    const PT* ext = (const PT*)P.ext;
    const int64_t tq = P.slots[t];  // the cell's query slot: its sorted position and its neighbour list
    const uint32_t s = P.qs[tq];
    const uint32_t e = P.perm[s];
    const PT sp = spts[s];
    // absolute seed; the cell is clipped in the frame centred on it (planes (-b, |b|^2 / 2)
    // for b = B - seed), which keeps clump cells far from the origin well conditioned
    const double sx = sp.x, sy = sp.y, sz = pz(sp);
    if (!(isfinite(sx) && isfinite(sy) && isfinite(sz))) {
        store_failed(P, lane, e, ST_SECURITY_RADIUS_NOT_REACHED);
        return;
    }

    // ---- the bounding box cell (cell.cpp:42-104) in the local frame: w' = w + n . seed
    const double beps = 1e-14;
    const double xmin = -beps, xmax = 1.0 + beps;
    if (lane < 2 * D) {
        double4 pl;
        switch (lane) {
            case 0: pl = make_double4(1.0, 0.0, 0.0, sx - xmin); break;
            case 1: pl = make_double4(-1.0, 0.0, 0.0, xmax - sx); break;
            case 2: pl = make_double4(0.0, 1.0, 0.0, sy - xmin); break;
            case 3: pl = make_double4(0.0, -1.0, 0.0, xmax - sy); break;
            case 4: pl = make_double4(0.0, 0.0, 1.0, sz - xmin); break;
            default: pl = make_double4(0.0, 0.0, -1.0, xmax - sz); break;
        }
        W.hp[lane] = pl;
        W.vid[lane] = -1;
    }
    if (D == 3) {
        W.u.b.emask[lane] = 0ull;
        W.u.b.emask[lane + 32] = 0ull;
    }
    const int ntri0 = D == 2 ? 4 : 8;
    if (lane < ntri0) {
        uint32_t tv;
        if (D == 2) {
            const uint32_t t2[4] = {pack3(2, 0, 0), pack3(1, 2, 0), pack3(3, 1, 0), pack3(0, 3, 0)};
            tv = t2[lane & 3];
        } else {
            const uint32_t t3[8] = {pack3(2, 5, 0), pack3(5, 3, 0), pack3(1, 5, 2), pack3(5, 1, 3),
                                    pack3(4, 2, 0), pack3(4, 0, 3), pack3(2, 4, 1), pack3(4, 3, 1)};
            tv = t3[lane & 7];
        }
        W.tri[lane] = tv;
    }
    __syncwarp();
    if (lane < ntri0) {
        double x, y, z;
        vertex_pos<D>(W.hp, W.tri[lane], x, y, z);
        W.vd2[lane] = seed_d2(x, y, z, 0.0, 0.0, 0.0);
    }
    __syncwarp();
    int nb_v = 2 * D, nb_t = ntri0;
    int status = ST_SUCCESS;
    double v_dist = max_vd2(W, nb_t, lane, nullptr);
    double fail_vdist = 0.0;

    // vertex positions of this lane's vertices (lane, lane + 32, lane + 64)
    double vx[3], vy[3], vz[3];
    auto refresh = [&]() {
#pragma unroll
        for (int j = 0; j < 3; j++) {
            const int i = lane + 32 * j;
            if (i < nb_t) vertex_pos<D>(W.hp, W.tri[i], vx[j], vy[j], vz[j]);
        }
    };
    refresh();
    // 1. The first walk_prefix neighbours of the cell's own list, in list order (the
    // list-based clip's order) and in the local frame; the walk then adds only the points
    // beyond them (keys above the last one's), so the cell stays near its final shape
    // instead of collecting transient vertices box by box.  The prefix is the same in
    // every form (plain K, learned K), so the walk is too.
    double key_d2 = -1.0;  // (distance, id) of the last listed neighbour clipped
    uint32_t key_id = 0u;
    bool alive = true, done = false;
    {
        const int Kc = P.kq ? (int)P.kq[tq] : P.K;
        const int L = min(Kc, P.walk_prefix);
        const uint32_t* kl = P.knn + (size_t)tq * P.K;
        for (int k = 0; k < L; k++) {
            const uint32_t z = kl[k];
            if (z == NO_NEIGHBOR) break;
            const PT B = ext[z];
            const double bx = B.x - sx, by = B.y - sy, bz = pz(B) - sz;
            const double d2 = seed_d2(bx, by, bz, 0.0, 0.0, 0.0);  // the KNN's key, exactly
            key_d2 = d2;
            key_id = z;
            if (d2 > 4 * v_dist) {  // certified: every point not clipped yet is farther
                done = true;
                break;
            }
            if (clip_by<D, true>(W, lane, z, bx, by, bz, 0.0, 0.0, 0.0, P.robust, nb_v, nb_t, status, v_dist,
                                 fail_vdist) == CLIP_FAIL) {
                alive = false;
                break;
            }
        }
        if (alive && !done) refresh();
    }
    // true when no point of the box can cut the cell (with a relative margin for rounding)
    auto prunable = [&](const double (&lo)[3], double side) -> bool {
        const double ll[3] = {lo[0] - sx, lo[1] - sy, lo[2] - sz};  // the box in the local frame
        bool ok = true;
#pragma unroll
        for (int j = 0; j < 3; j++) {
            const int i = lane + 32 * j;
            if (i < nb_t) ok = ok && pt_box_d2<D>(vx[j], vy[j], vz[j], ll, side) > W.vd2[i] * (1.0 + 1e-9);
        }
        return __all_sync(FULL, ok);
    };
    const InstPar& ipc = g.ip[g.inst[e]];  // the cell's instance: its grid
    const int G = ipc.G;
    const uint32_t slot0 = ipc.slot0;
    const double h0 = 1.0 / (double)G;
    // work bounds: a cell that needs more is left uncertified (reported, not hung)
    int boxes = 0, points = 0;
    // clips by the points of level-L box (x, y, z), descending refined bins depth first
    auto visit = [&](int x0, int y0, int z0) -> bool {
        int sp_ = 0;
        if (lane == 0) stk[0] = make_int4(x0, y0, z0, 0);
        sp_ = 1;
        __syncwarp();
        while (sp_ > 0) {
            const int4 b = stk[--sp_];
            __syncwarp();
            const int L = b.w;
            if (++boxes > WALK_MAX_BOXES || v_dist != v_dist) return false;
            if (L > 0) {  // pushed while the cell was larger: test again
                const double side = 1.0 / (double)(G << L);
                const double lo[3] = {b.x * side, b.y * side, b.z * side};
                if (pt_box_d2<D>(sx, sy, sz, lo, side) * (1.0 - 1e-12) > 4 * v_dist) continue;
                if (prunable(lo, side)) continue;
            }
            const int cx = b.x >> L, cy = b.y >> L, cz = b.z >> L;
            const uint32_t m = slot0 + morton<D>(cx, cy, cz);
            const int Lb = g.lvl[m];
            if (L < Lb) {
                // children nearest first: pushed farthest first
                const double side = 1.0 / (double)(G << (L + 1));
                double cd[1 << D];
                int order[1 << D];
#pragma unroll
                for (int ch = 0; ch < (1 << D); ch++) {
                    const double lo[3] = {(2 * b.x + (ch & 1)) * side, (2 * b.y + ((ch >> 1) & 1)) * side,
                                          D == 3 ? (2 * b.z + ((ch >> 2) & 1)) * side : 0.0};
                    cd[ch] = pt_box_d2<D>(sx, sy, sz, lo, side);
                    order[ch] = ch;
                }
                for (int a = 1; a < (1 << D); a++)  // insertion sort, descending distance
                    for (int q = a; q > 0 && cd[order[q]] > cd[order[q - 1]]; q--) {
                        const int tmp = order[q];
                        order[q] = order[q - 1];
                        order[q - 1] = tmp;
                    }
                for (int a = 0; a < (1 << D); a++) {
                    const int ch = order[a];
                    if (cd[ch] * (1.0 - 1e-12) > 4 * v_dist) continue;
                    const int nx = 2 * b.x + (ch & 1), ny = 2 * b.y + ((ch >> 1) & 1),
                              nz = D == 3 ? 2 * b.z + ((ch >> 2) & 1) : 0;
                    const double lo[3] = {nx * side, ny * side, nz * side};
                    if (prunable(lo, side)) continue;
                    if (sp_ >= PRUNE_STACK) return false;
                    if (lane == 0) stk[sp_] = make_int4(nx, ny, nz, L + 1);
                    sp_++;
                }
                __syncwarp();
                continue;
            }
            // a leaf: one sub-bin of the bin's own level
            const uint32_t slot = g.sub_off[m] + (L > 0 ? morton<D>(b.x - (cx << L), b.y - (cy << L), b.z - (cz << L)) : 0u);
            const uint32_t a0 = g.sub_start[slot], a1 = g.sub_start[slot + 1];
            for (uint32_t q = a0; q < a1; q++) {
                if (q == s) continue;
                const PT B = spts[q];
                const double bx = B.x - sx, by = B.y - sy, bz = pz(B) - sz;
                const double d2 = seed_d2(bx, by, bz, 0.0, 0.0, 0.0);
                if (d2 > 4 * v_dist) continue;
                const uint32_t id = P.perm[q];
                if (d2 < key_d2 || (d2 == key_d2 && id <= key_id)) continue;  // clipped from the list
                if (++points > WALK_MAX_POINTS) return false;
                const int r = clip_by<D, true>(W, lane, id, bx, by, bz, 0.0, 0.0, 0.0, P.robust, nb_v, nb_t,
                                               status, v_dist, fail_vdist);
                if (r == CLIP_FAIL) return false;
                if (r == CLIP_CUT) refresh();
            }
        }
        return true;
    };
    // coarse bins around the seed's: the offset table (ascending lower bound), then rings
    const int bc[3] = {bin_coord(sx, G), bin_coord(sy, G), D == 3 ? bin_coord(sz, G) : 0};
    const double pc[3] = {sx, sy, sz};
    for (int ci = 0; ci < table_n && alive && !done; ci++) {
        const int2 ent = table[ci];
        if ((double)ent.y * h0 * h0 * (1.0 - 1e-12) > 4 * v_dist) break;
        const int x = bc[0] + (int)(signed char)(ent.x & 255), y = bc[1] + (int)(signed char)((ent.x >> 8) & 255),
                  z = D == 3 ? bc[2] + (int)(signed char)((ent.x >> 16) & 255) : 0;
        if (x < 0 || x >= G || y < 0 || y >= G || (D == 3 && (z < 0 || z >= G))) continue;
        const double lo[3] = {x * h0, y * h0, z * h0};
        if (pt_box_d2<D>(sx, sy, sz, lo, h0) * (1.0 - 1e-12) > 4 * v_dist) continue;
        if (prunable(lo, h0)) continue;
        alive = visit(x, y, z);
    }
    // a vertex without a position (three planes through one line, w = 0) makes v_dist
    // NaN and no radius bounds the walk: such a cell stays uncertified, as in k_clip
    if (v_dist != v_dist) alive = false;
    for (int r = table_r + 1; alive && !done; r++) {
        double lb = CUDART_INF;
        bool all = true;
#pragma unroll
        for (int a = 0; a < D; a++) {
            const int lo = bc[a] - (r - 1), hi = bc[a] + (r - 1);
            if (lo > 0) {
                all = false;
                lb = fmin(lb, pc[a] - (double)lo * h0);
            }
            if (hi < G - 1) {
                all = false;
                lb = fmin(lb, (double)(hi + 1) * h0 - pc[a]);
            }
        }
        if (all || r > G + 1) break;
        if (lb > 0.0 && 4 * v_dist < lb * lb * (1.0 - 1e-12)) break;
        if (v_dist != v_dist) {
            alive = false;
            break;
        }
        const int w1 = 2 * r + 1;
        const int ncube = D == 2 ? w1 * w1 : w1 * w1 * w1;
        for (int ci = 0; ci < ncube && alive; ci++) {
            const int dx = ci % w1 - r, rest = ci / w1;
            const int dy = rest % w1 - r, dz = D == 3 ? rest / w1 - r : 0;
            if (max(abs(dx), max(abs(dy), abs(dz))) != r) continue;
            if (++boxes > WALK_MAX_BOXES) {
                alive = false;
                break;
            }
            const int x = bc[0] + dx, y = bc[1] + dy, z = bc[2] + dz;
            if (x < 0 || x >= G || y < 0 || y >= G || (D == 3 && (z < 0 || z >= G))) continue;
            const double lo[3] = {x * h0, y * h0, z * h0};
            if (pt_box_d2<D>(sx, sy, sz, lo, h0) * (1.0 - 1e-12) > 4 * v_dist) continue;
            if (prunable(lo, h0)) continue;
            alive = visit(x, y, z);
        }
    }
    if (lane == 0) {
        atomicAdd(&P.walk_stats[0], (unsigned long long)points);
        atomicAdd(&P.walk_stats[1], (unsigned long long)boxes);
    }
    if (!alive || v_dist != v_dist) {
        store_failed(P, lane, e, status == ST_SUCCESS ? ST_SECURITY_RADIUS_NOT_REACHED : status);
        return;
    }
    // every point within the security radius was clipped or excluded: certified
    extract_and_store<D>(W, P, w, lane, nb_v, nb_t, e, P.walk_certk, 0.0, 0.0, 0.0, false, sx, sy, sz);
}

// ============================================================================
// FP32 local-frame clipping (the precision form).  The cell is clipped
// in single precision in a frame centred on its seed: a neighbour b = B - seed
// gives the plane (-b, |b|^2 / 2), the box planes get w + n.seed.  Every
// plane-vertex determinant is accepted only when it exceeds a bound on its
// rounding error, 64 u times an upper bound of the permanent of the absolute
// entries (u = 2^-24);
// otherwise, and on any overflow or inconsistent cavity, the cell is handed to
// the FP64 kernel (status ST_RECLIP).  Certified cells are extracted in FP64:
// the plane equations are recomputed from the points with the reference's
// formula, vertices follow in FP64 from the same triples, and the security
// radius is checked again in FP64 over the final vertex set, which also yields
// the exact certified K.  A cell whose FP64 check disagrees is re-clipped.  So
// topology, statuses and geometry are those of the FP64 path.
// ============================================================================

constexpr int ST_RECLIP = 7;
constexpr float F32_BOUND = 64.0f * 5.9604645e-8f;

__device__ __forceinline__ float det2f(float a11, float a12, float a21, float a22) {
    return fmaf(a11, a22, -(a12 * a21));
}
__device__ __forceinline__ float per2f(float a11, float a12, float a21, float a22) {
    return fabsf(a11 * a22) + fabsf(a12 * a21);
}
__device__ __forceinline__ float det3f(float a11, float a12, float a13, float a21, float a22, float a23, float a31,
                                       float a32, float a33) {
    float t = a11 * det2f(a22, a23, a32, a33);
    t = fmaf(-a21, det2f(a12, a13, a32, a33), t);
    return fmaf(a31, det2f(a12, a13, a22, a23), t);
}
__device__ __forceinline__ float per3f(float a11, float a12, float a13, float a21, float a22, float a23, float a31,
                                       float a32, float a33) {
    return fabsf(a11) * per2f(a22, a23, a32, a33) + fabsf(a21) * per2f(a12, a13, a32, a33) +
           fabsf(a31) * per2f(a12, a13, a22, a23);
}

// Homogeneous coordinates of a vertex in the local frame -- the cofactors of the
// plane-vertex determinant: det4(p1, p2, p3, e) = e . V (and det3 in 2D) -- and
// the permanents of the same minors, which bound their rounding errors.  The
// entries of a plane differ in scale (normal ~ h, offset ~ h^2), so the offset's
// cofactor keeps its own permanent and the three normal cofactors share their
// largest: (|e.x| + |e.y| + |e.z|) P_xyz + |e.w| P_w bounds the permanent of the
// full matrix (8 bytes a vertex instead of 16, for 28 warps per SM).
template <int D>
__device__ __forceinline__ void vertex_h32(const float4* hp, uint32_t t, float4& V, float2& Pb2) {
    float4 Pb;
    const float4 p1 = hp[tri_a(t)], p2 = hp[tri_b(t)];
    if (D == 2) {
        V.x = -det2f(p1.w, p1.y, p2.w, p2.y);
        V.y = -det2f(p1.x, p1.w, p2.x, p2.w);
        V.z = 0.0f;
        V.w = det2f(p1.x, p1.y, p2.x, p2.y);
        Pb = make_float4(per2f(p1.w, p1.y, p2.w, p2.y), per2f(p1.x, p1.w, p2.x, p2.w), 0.0f,
                         per2f(p1.x, p1.y, p2.x, p2.y));
        Pb2 = make_float2(fmaxf(Pb.x, Pb.y), Pb.w);
        return;
    }
    const float4 p3 = hp[tri_c(t)];
    V.x = -det3f(p1.w, p1.y, p1.z, p2.w, p2.y, p2.z, p3.w, p3.y, p3.z);
    V.y = -det3f(p1.x, p1.w, p1.z, p2.x, p2.w, p2.z, p3.x, p3.w, p3.z);
    V.z = -det3f(p1.x, p1.y, p1.w, p2.x, p2.y, p2.w, p3.x, p3.y, p3.w);
    V.w = det3f(p1.x, p1.y, p1.z, p2.x, p2.y, p2.z, p3.x, p3.y, p3.z);
    Pb = make_float4(per3f(p1.w, p1.y, p1.z, p2.w, p2.y, p2.z, p3.w, p3.y, p3.z),
                     per3f(p1.x, p1.w, p1.z, p2.x, p2.w, p2.z, p3.x, p3.w, p3.z),
                     per3f(p1.x, p1.y, p1.w, p2.x, p2.y, p2.w, p3.x, p3.y, p3.w),
                     per3f(p1.x, p1.y, p1.z, p2.x, p2.y, p2.z, p3.x, p3.y, p3.z));
    Pb2 = make_float2(fmaxf(fmaxf(Pb.x, Pb.y), Pb.z), Pb.w);
}

// Squared distance to the seed (the origin of the local frame) of a vertex given
// in homogeneous coordinates.
__device__ __forceinline__ float vd2_of(const float4& V) {
    const float x = V.x / V.w, y = V.y / V.w, z = V.z / V.w;
    return fmaf(x, x, fmaf(y, y, z * z));
}

// Plane-vertex predicate from the cached cofactors: 0 = not in conflict,
// 1 = in conflict, 2 = undecided in FP32.  The bound covers the cofactors'
// rounding, the dot product's and the planes' own entry errors (all first order
// in the permanent |e| . P).
__device__ __forceinline__ int conflict_h32(const float4& V, const float2& P, const float4& e) {
    const float t = fmaf(e.w, V.w, fmaf(e.z, V.z, fmaf(e.y, V.y, e.x * V.x)));
    // |e.x| P.x + |e.y| P.y + |e.z| P.z + |e.w| P.w <= (|e.x| + |e.y| + |e.z|) max(P.x, P.y, P.z) + |e.w| P.w
    const float per = fmaf(fabsf(e.w), P.y, (fabsf(e.x) + fabsf(e.y) + fabsf(e.z)) * P.x);
    if (!(fabsf(t) > F32_BOUND * per)) return 2;
    return t > 0.0f ? 1 : 0;
}

// The squared distances are >= +0 or NaN, so their bit patterns order as unsigned
// integers (any NaN above every number): one integer max-reduction gives the
// maximum, NaN when any is NaN.
template <class Cell>
__device__ __forceinline__ float max_vd2f(const Cell& W, int n, int lane) {
    uint32_t m = 0u;
    const float* d32 = D32_of(W);
#pragma unroll
    for (int j = 0; j < 3; j++) {
        const int i = lane + 32 * j;
        if (i < n) m = max(m, __float_as_uint(d32[i]));
    }
    return __uint_as_float(__reduce_max_sync(FULL, m));
}

// The reference's FP64 plane p of the cell (box planes, or the bisector with
// extended point vid), global coordinates (cell.cpp:75-82, 164-168).
template <int D>
__device__ __forceinline__ double4 plane64(int p, int vid, const typename PointOf<D>::type* ext, double sx, double sy,
                                           double sz) {
    const double beps = 1e-14, xmin = -beps, xmax = 1.0 + beps;
    if (vid < 0) {
        switch (p) {
            case 0: return make_double4(1.0, 0.0, 0.0, -xmin);
            case 1: return make_double4(-1.0, 0.0, 0.0, xmax);
            case 2: return make_double4(0.0, 1.0, 0.0, -xmin);
            case 3: return make_double4(0.0, -1.0, 0.0, xmax);
            case 4: return make_double4(0.0, 0.0, 1.0, -xmin);
            default: return make_double4(0.0, 0.0, -1.0, xmax);
        }
    }
    const typename PointOf<D>::type B = ext[vid];
    const double bx = B.x, by = B.y, bz = pz(B);
    const double dx = sx - bx, dy = sy - by, dz = sz - bz;
    const double ax = sx + bx, ay = sy + by, az = sz + bz;
    const double dot = ax * dx + ay * dy + az * dz;
    return make_double4(dx, dy, dz, -dot / 2.0);
}

// Resident warps per SM: 32 in 3D (64 registers a thread, 6.9 KB of shared memory a
// warp: the overlaid cell), 28 in 2D (72 registers, 7.8 KB).  One cell per block: 28
// one-warp blocks fit an SM's shared memory (each block also reserves 1 KB), so the
// registers are set for 28 (72 a thread, nearly no spills).
template <int D, int CW>
__global__ void __launch_bounds__(CW * 32, CW == 1 ? 28 : (D == 3 ? 32 : 28) / CW) k_clip32(ClipParams P) {
    using PT = typename PointOf<D>::type;
    using Cell = typename std::conditional<D == 3, WarpCell32, WarpCell>::type;
    __shared__ Cell cells[CW];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int64_t t = (int64_t)blockIdx.x * CW + w;
    if (t >= P.nq) return;  // warp-uniform
    Cell& W = cells[w];
    float4* hp = hp32_of(W);
    float4* V32 = V32_of(W);
    float2* P32 = P32_of(W);
    float* D32 = D32_of(W);
    const PT* spts = (const PT*)P.spts;
    const PT* ext = (const PT*)P.ext;
    const int64_t tq = P.slots ? (int64_t)P.slots[t] : t;
    const uint32_t s = P.qs[tq];
    const uint32_t e = P.perm[s];
    const PT sp = spts[s];
    const double sx = sp.x, sy = sp.y, sz = pz(sp);
    const int K = P.kq ? (int)P.kq[tq] : P.K;  // per-cell budget (learned K) within rows of P.K
    const uint32_t* kl = P.knn + (size_t)tq * P.K;

    // bounding box in the local frame: w' = w + n . seed
    const double beps = 1e-14;
    const double xmin = -beps, xmax = 1.0 + beps;
    if (lane < 2 * D) {
        float4 pl;
        switch (lane) {
            case 0: pl = make_float4(1.f, 0.f, 0.f, (float)(sx - xmin)); break;
            case 1: pl = make_float4(-1.f, 0.f, 0.f, (float)(xmax - sx)); break;
            case 2: pl = make_float4(0.f, 1.f, 0.f, (float)(sy - xmin)); break;
            case 3: pl = make_float4(0.f, -1.f, 0.f, (float)(xmax - sy)); break;
            case 4: pl = make_float4(0.f, 0.f, 1.f, (float)(sz - xmin)); break;
            default: pl = make_float4(0.f, 0.f, -1.f, (float)(xmax - sz)); break;
        }
        hp[lane] = pl;
        W.vid[lane] = -1;
    }
    if (D == 3) {
        emask_of(W)[lane] = 0ull;
        emask_of(W)[lane + 32] = 0ull;
    }
    const int ntri0 = D == 2 ? 4 : 8;
    if (lane < ntri0) {
        uint32_t tv;
        if (D == 2) {
            const uint32_t t2[4] = {pack3(2, 0, 0), pack3(1, 2, 0), pack3(3, 1, 0), pack3(0, 3, 0)};
            tv = t2[lane & 3];
        } else {
            const uint32_t t3[8] = {pack3(2, 5, 0), pack3(5, 3, 0), pack3(1, 5, 2), pack3(5, 1, 3),
                                    pack3(4, 2, 0), pack3(4, 0, 3), pack3(2, 4, 1), pack3(4, 3, 1)};
            tv = t3[lane & 7];
        }
        W.tri[lane] = tv;
    }
    __syncwarp();
    if (lane < ntri0) {
        vertex_h32<D>(hp, W.tri[lane], V32[lane], P32[lane]);
        D32[lane] = vd2_of(V32[lane]);
    }
    __syncwarp();
    int nb_v = 2 * D, nb_t = ntri0;
    bool reclip = false, certified = false;
    int k_stop = 0, k_last = 0;
    float v_dist = max_vd2f(W, nb_t, lane);

    // neighbours are fetched 32 at a time, one per lane; each lane forms its
    // neighbour's local-frame plane and distance, broadcast plane by plane
    uint32_t zc = NO_NEIGHBOR;
    float cfx = 0.f, cfy = 0.f, cfz = 0.f, cfw = 0.f, cd2 = 0.f;
    for (int k = 0; k < K; k++) {
        if ((k & 31) == 0) {
            const int kk = k + lane;
            zc = kk < K ? kl[kk] : NO_NEIGHBOR;
            if (zc != NO_NEIGHBOR) {
                const PT Bc = ext[zc];
                const double bx = Bc.x - sx, by = Bc.y - sy, bz = pz(Bc) - sz;  // local frame, exact in FP64
                cfx = (float)bx;
                cfy = (float)by;
                cfz = (float)bz;
                cfw = 0.5f * fmaf(cfx, cfx, fmaf(cfy, cfy, cfz * cfz));
                cd2 = (float)seed_d2(Bc.x, Bc.y, pz(Bc), sx, sy, sz);
            }
            if constexpr (D == 3) {
                __syncwarp();
                W.c.sb_eq[lane] = make_float4(-cfx, -cfy, -cfz, cfw);
                W.c.sb_d2[lane] = cd2;
                W.c.sb_z[lane] = zc;
                __syncwarp();
            }
        }
        uint32_t z;
        float d2Bf;
        float4 eq;
        if constexpr (D == 3) {
            z = W.c.sb_z[k & 31];
            d2Bf = W.c.sb_d2[k & 31];
            eq = W.c.sb_eq[k & 31];
        } else {
            z = __shfl_sync(FULL, zc, k & 31);
            d2Bf = __shfl_sync(FULL, cd2, k & 31);
            eq = make_float4(-__shfl_sync(FULL, cfx, k & 31), -__shfl_sync(FULL, cfy, k & 31),
                             -__shfl_sync(FULL, cfz, k & 31), __shfl_sync(FULL, cfw, k & 31));
        }
        if (z == NO_NEIGHBOR) break;
        k_stop = k + 1;
        if (nb_v >= MAX_P) {
            reclip = true;
            break;
        }
        const int cur = nb_v;
        if constexpr (D == 2) {
            if (lane == 0) hp[cur] = eq;
            __syncwarp();
        }

        uint32_t cm[3];
        bool undecided = false;
#pragma unroll
        for (int j = 0; j < 3; j++) {
            const int i = lane + 32 * j;
            bool cf = false;
            if (i < nb_t) {
                const int c = conflict_h32(V32[i], P32[i], eq);
                undecided |= c == 2;
                cf = c == 1;
            }
            cm[j] = __ballot_sync(FULL, cf);
        }
        if (__any_sync(FULL, undecided)) {
            reclip = true;
            break;
        }
        const int nb_r = __popc(cm[0]) + __popc(cm[1]) + __popc(cm[2]);
        const uint32_t km[3] = {~cm[0], ~cm[1], ~cm[2]};
        if (nb_r == 0) {
            if (d2Bf > 4.004f * v_dist) {
                certified = true;
                break;
            }
            continue;
        }
        k_last = k + 1;
        if constexpr (D == 3) {  // the plane cuts: it joins the cell's plane list
            if (lane == 0) hp[cur] = eq;
            __syncwarp();
        }
        const int kept = nb_t - nb_r;
        int n_new = 0;
        bool bad = false;
        uint32_t* stage = stage_of(W);  // new vertices, written at their final position
        if (D == 2) {
            uint32_t lo = 0, hi = 0;
#pragma unroll
            for (int j = 0; j < 3; j++) {
                const int i = lane + 32 * j;
                if (i < nb_t && ((cm[j] >> lane) & 1u)) {
                    const uint32_t tv = W.tri[i];
                    const uint32_t a = tri_a(tv), b = tri_b(tv);
                    if (a < 32) lo ^= 1u << a; else hi ^= 1u << (a - 32);
                    if (b < 32) lo ^= 1u << b; else hi ^= 1u << (b - 32);
                }
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                lo ^= __shfl_xor_sync(FULL, lo, o);
                hi ^= __shfl_xor_sync(FULL, hi, o);
            }
            const unsigned long long xm = (unsigned long long)lo | ((unsigned long long)hi << 32);
            if (__popcll(xm) < 2) {
                bad = true;
            } else {
                const int b0 = __ffsll((long long)xm) - 1;
                const unsigned long long x2 = xm & (xm - 1);
                const int b1 = __ffsll((long long)x2) - 1;
                n_new = 2;
                bool und = false;
                if (lane < 2) {
                    const int j = lane == 0 ? b0 : b1;
                    const float4 hi_ = hp[cur], hj = hp[j];
                    const float rw = det2f(hi_.x, hi_.y, hj.x, hj.y);
                    und = !(fabsf(rw) > F32_BOUND * per2f(hi_.x, hi_.y, hj.x, hj.y));
                    stage[lane] = rw > 0 ? pack3(j, cur, 0) : pack3(cur, j, 0);
                }
                if (__any_sync(FULL, und)) bad = true;
            }
        } else {
            unsigned long long src = 0ull;
            n_new = cavity_boundary3<false>(W, lane, cm, nb_t, nb_r, (uint32_t)cur, src);
            // Every predicate that reached this point was decided beyond its error
            // bound, so the conflict set is the exact one and (no vertex lies on the
            // plane: that would have been undecided) the cavity boundary is one simple
            // cycle; the reference's walk (cell.cpp:262-300), which the FP64 kernel
            // replays, cannot fail here.  Each source plane appearing once is checked.
            bad = !(__popcll(src) == n_new && n_new >= 3);
        }
        if (bad || kept + n_new >= MAX_T || n_new > MAX_P) {
            reclip = true;
            break;
        }
        uint32_t kt[3];
        float4 kd[3];
        float2 kb[3];
        float kr[3];
        int kp[3];
        int before = 0;
#pragma unroll
        for (int j = 0; j < 3; j++) {
            const int i = lane + 32 * j;
            const int nvalid = nb_t - 32 * j;
            const uint32_t vm = nvalid >= 32 ? FULL : (nvalid > 0 ? ((1u << nvalid) - 1u) : 0u);
            const uint32_t kmj = km[j] & vm;
            const bool keep = (kmj >> lane) & 1u;
            kt[j] = keep ? W.tri[i] : 0u;
            kd[j] = keep ? V32[i] : make_float4(0.f, 0.f, 0.f, 0.f);
            kb[j] = keep ? P32[i] : make_float2(0.f, 0.f);
            kr[j] = keep ? D32[i] : 0.0f;
            kp[j] = keep ? before + __popc(kmj & ((1u << lane) - 1u)) : -1;
            before += __popc(kmj);
        }
        __syncwarp();
#pragma unroll
        for (int j = 0; j < 3; j++)
            if (kp[j] >= 0) {
                W.tri[kp[j]] = kt[j];
                V32[kp[j]] = kd[j];
                P32[kp[j]] = kb[j];
                D32[kp[j]] = kr[j];
            }
        // new vertices after the kept ones, one lane each
        for (int q = lane; q < n_new; q += 32) {
            const uint32_t tv = stage[q];
            float4 V;
            float2 Pb;
            vertex_h32<D>(hp, tv, V, Pb);
            W.tri[kept + q] = tv;
            V32[kept + q] = V;
            P32[kept + q] = Pb;
            D32[kept + q] = vd2_of(V);
        }
        if (lane == 0) W.vid[cur] = (int)z;
        nb_v++;
        nb_t = kept + n_new;
        __syncwarp();
        v_dist = max_vd2f(W, nb_t, lane);
        if (d2Bf > 4.004f * v_dist) {
            certified = true;
            break;
        }
    }
    if (reclip) {
        if (lane == 0) {
            P.status[e] = ST_RECLIP;
            atomicAdd(P.reclip, 1u);
        }
        return;
    }
    // ---- FP64: planes, vertices and the certificate over the final vertex set
    __syncwarp();
#pragma unroll
    for (int pass = 0; pass < 2; pass++) {
        const int p = lane + 32 * pass;
        if (p < nb_v) hp_of(W)[p] = plane64<D>(p, W.vid[p], ext, sx, sy, sz);
    }
    compute_vpos<D>(W, lane, nb_t);
    double vm64 = 0.0;
#pragma unroll
    for (int j = 0; j < 3; j++) {
        const int i = lane + 32 * j;
        if (i < nb_t) vm64 = nan_max(vm64, seed_d2(vpos_of(W)[i][0], vpos_of(W)[i][1], vpos_of(W)[i][2], sx, sy, sz));
    }
    vm64 = warp_max(vm64);
    // first k >= k_last (1-based) whose neighbour lies beyond twice the farthest vertex
    int certk = 0;
    const int k_lo = k_last > 0 ? k_last : 1;
    for (int k0 = k_lo; k0 <= k_stop && certk == 0; k0 += 32) {
        const int k = k0 + lane;
        bool pass = false;
        if (k <= k_stop) {
            const uint32_t z = kl[k - 1];
            const PT B = ext[z];
            pass = seed_d2(B.x, B.y, pz(B), sx, sy, sz) > 4 * vm64;
        }
        const unsigned bal = __ballot_sync(FULL, pass);
        if (bal) certk = k0 + __ffs(bal) - 1;
    }
    const bool last_valid = kl[K - 1] != NO_NEIGHBOR;
    if (certk == 0 || !last_valid) {
        if (certified && last_valid) {  // FP32 stopped before FP64 agrees: clip again in FP64
            if (lane == 0) {
                P.status[e] = ST_RECLIP;
                atomicAdd(P.reclip, 1u);
            }
            return;
        }
        store_failed(P, lane, e, ST_SECURITY_RADIUS_NOT_REACHED);
        return;
    }
    extract_and_store<D>(W, P, w, lane, nb_v, nb_t, e, certk, sx, sy, sz, true);
}

// ============================================================================
// Thread-per-cell 2D clipping.  A 2D cell has ~6 vertices, so the warp-per-cell
// kernel leaves most lanes idle; here each thread clips one cell with the same
// arithmetic in the same order (vertex list, predicates, new-vertex orientation,
// stable compaction, certificate, angle-ordered area, plane-ordered faces), so
// the result is the warp kernel's bit for bit.  Cells needing more than
// T2P planes or T2T vertices are marked ST_RECLIP and re-run by the warp kernel.
constexpr int T2P = 24;
constexpr int T2T = 24;
constexpr int T2_THREADS = 128;

__global__ void __launch_bounds__(T2_THREADS) k_clip2t(ClipParams P) {
    const int64_t t = (int64_t)blockIdx.x * T2_THREADS + threadIdx.x;
    if (t >= P.nq) return;
    const int64_t tq = P.slots ? (int64_t)P.slots[t] : t;
    const uint32_t s = P.qs[tq];
    const uint32_t e = P.perm[s];
    const double2* spts = (const double2*)P.spts;
    const double2* ext = (const double2*)P.ext;
    const double2 sp = spts[s];
    const double sx = sp.x, sy = sp.y, sz = 0.0;
    const int K = P.kq ? (int)P.kq[tq] : P.K;
    const uint32_t* kl = P.knn + (size_t)tq * P.K;

    double4 hp[T2P];
    int vid[T2P];
    uint32_t tri[T2T];
    double vd2[T2T];
    const double beps = 1e-14;
    const double xmin = -beps, xmax = 1.0 + beps;
    hp[0] = make_double4(1.0, 0.0, 0.0, -xmin);
    hp[1] = make_double4(-1.0, 0.0, 0.0, xmax);
    hp[2] = make_double4(0.0, 1.0, 0.0, -xmin);
    hp[3] = make_double4(0.0, -1.0, 0.0, xmax);
    for (int i = 0; i < 4; i++) vid[i] = -1;
    tri[0] = pack3(2, 0, 0);
    tri[1] = pack3(1, 2, 0);
    tri[2] = pack3(3, 1, 0);
    tri[3] = pack3(0, 3, 0);
    double v_dist = 0.0;
    for (int i = 0; i < 4; i++) {
        double x, y, z;
        vertex_pos<2>(hp, tri[i], x, y, z);
        vd2[i] = seed_d2(x, y, z, sx, sy, sz);
        v_dist = nan_max(v_dist, vd2[i]);
    }
    int nb_v = 4, nb_t = 4;
    int status = ST_SUCCESS, certk = 0;
    double fail_vdist = 0.0;
    bool too_big = false;
    for (int k = 0; k < K; k++) {
        const uint32_t z = kl[k];
        if (z == NO_NEIGHBOR) break;
        const double2 B = ext[z];
        const double bx = B.x, by = B.y, bz = 0.0;
        const double d2B = seed_d2(bx, by, bz, sx, sy, sz);
        if (nb_v >= MAX_P) {
            status = ST_VERTEX_OVERFLOW;
            fail_vdist = v_dist;
            break;
        }
        if (nb_v >= T2P) {
            too_big = true;
            break;
        }
        const double dx = sx - bx, dy = sy - by, dz = sz - bz;
        const double ax = sx + bx, ay = sy + by, az = sz + bz;
        const double dot = ax * dx + ay * dy + az * dz;
        const double4 eq = make_double4(dx, dy, dz, -dot / 2.0);
        const int cur = nb_v;
        hp[cur] = eq;
        uint32_t cm = 0;  // vertices in conflict (nb_t <= T2T < 32)
        bool near = false;
        for (int i = 0; i < nb_t; i++)
            if (in_conflict<2>(hp, tri[i], eq, &near, P.robust)) cm |= 1u << i;
        const int nb_r = __popc(cm);
        if (near) {
            status = ST_NEEDS_EXACT_PREDICATES;
            double m = 0.0;
            for (int i = 0; i < nb_t; i++)
                if (!((cm >> i) & 1u)) m = nan_max(m, vd2[i]);
            fail_vdist = m;
            break;
        }
        if (nb_r == 0) {
            if (d2B > 4 * v_dist) {
                certk = k + 1;
                break;
            }
            continue;
        }
        unsigned long long xm = 0ull;
        for (int i = 0; i < nb_t; i++)
            if ((cm >> i) & 1u) xm ^= (1ull << tri_a(tri[i])) ^ (1ull << tri_b(tri[i]));
        const int kept = nb_t - nb_r;
        if (__popcll(xm) < 2) {
            status = ST_INCONSISTENT_BOUNDARY;
            double m = 0.0;
            for (int i = 0; i < nb_t; i++)
                if (!((cm >> i) & 1u)) m = nan_max(m, vd2[i]);
            fail_vdist = m;
            break;
        }
        const int b0 = __ffsll((long long)xm) - 1;
        const unsigned long long x2 = xm & (xm - 1);
        const int b1 = __ffsll((long long)x2) - 1;
        uint32_t nt[2];
        double nd[2];
        double newmax = 0.0;
        for (int q = 0; q < 2; q++) {
            const int j = q == 0 ? b0 : b1;
            const double rw = det2(hp[cur].x, hp[cur].y, hp[j].x, hp[j].y);  // new_vertex orientation
            nt[q] = rw > 0 ? pack3(j, cur, 0) : pack3(cur, j, 0);
            double x, y, zz;
            vertex_pos<2>(hp, nt[q], x, y, zz);
            nd[q] = seed_d2(x, y, zz, sx, sy, sz);
            newmax = nan_max(newmax, nd[q]);
        }
        if (kept + 2 >= MAX_T) {
            status = ST_TRIANGLE_OVERFLOW;
            double m = 0.0;
            for (int i = 0; i < nb_t; i++)
                if (!((cm >> i) & 1u)) m = nan_max(m, vd2[i]);
            fail_vdist = nan_max(m, newmax);
            break;
        }
        if (kept + 2 > T2T) {
            too_big = true;
            break;
        }
        int w = 0;
        for (int i = 0; i < nb_t; i++)
            if (!((cm >> i) & 1u)) {
                tri[w] = tri[i];
                vd2[w] = vd2[i];
                w++;
            }
        tri[kept] = nt[0];
        vd2[kept] = nd[0];
        tri[kept + 1] = nt[1];
        vd2[kept + 1] = nd[1];
        vid[cur] = (int)z;
        nb_v++;
        nb_t = kept + 2;
        double m = 0.0;
        for (int i = 0; i < nb_t; i++) m = nan_max(m, vd2[i]);
        v_dist = m;
        if (d2B > 4 * v_dist) {
            certk = k + 1;
            break;
        }
    }
    if (too_big) {
        P.status[e] = ST_RECLIP;
        atomicAdd(P.reclip, 1u);
        return;
    }
    {
        const double vdf = status == ST_SUCCESS ? v_dist : fail_vdist;
        const uint32_t zK = kl[K - 1];
        if (zK == NO_NEIGHBOR) {
            status = ST_SECURITY_RADIUS_NOT_REACHED;
        } else {
            const double2 BK = ext[zK];
            if (!(seed_d2(BK.x, BK.y, 0.0, sx, sy, sz) > 4 * vdf)) status = ST_SECURITY_RADIUS_NOT_REACHED;
        }
    }
    if (status != ST_SUCCESS) {
        if (status == ST_SECURITY_RADIUS_NOT_REACHED && (int64_t)e < P.n_hydro) atomicAdd(P.uncertified, 1u);
        P.vol[e] = 0.0;
        P.fptr[e] = 0;
        P.fcnt[e] = 0;
        P.status[e] = status;
        P.certk[e] = 0;
        P.centroid[3 * (size_t)e] = P.centroid[3 * (size_t)e + 1] = P.centroid[3 * (size_t)e + 2] = 0.0;
        return;
    }
    // ---- extraction (cell.cpp:416-669), the warp kernel's 2D branch in one thread
    double vx[T2T], vy[T2T];
    for (int i = 0; i < nb_t; i++) {
        double z;
        vertex_pos<2>(hp, tri[i], vx[i], vy[i], z);
    }
    double cx = 0, cy = 0;
    for (int i = 0; i < nb_t; i++) cx += vx[i], cy += vy[i];
    cx /= nb_t;
    cy /= nb_t;
    double ang[T2T];
    for (int i = 0; i < nb_t; i++) ang[i] = atan2(vy[i] - cy, vx[i] - cx);
    unsigned char order[T2T];
    for (int i = 0; i < nb_t; i++) {
        int rank = 0;
        for (int q = 0; q < nb_t; q++) rank += (ang[q] < ang[i] || (ang[q] == ang[i] && q < i)) ? 1 : 0;
        order[rank] = (unsigned char)i;
    }
    double a = 0, mx = 0, my = 0, sa = 0;
    for (int i = 0; i < nb_t; i++) {
        const int j = (i + 1) % nb_t;
        const int pi = order[i], qi = order[j];
        a += vx[pi] * vy[qi];
        a -= vx[qi] * vy[pi];
        const double cr = (vx[pi] - cx) * (vy[qi] - cy) - (vx[qi] - cx) * (vy[pi] - cy);
        mx += (vx[pi] + vx[qi] - 2 * cx) * cr;
        my += (vy[pi] + vy[qi] - 2 * cy) * cr;
        sa += cr;
    }
    const double cell_vol = fabs(a) / 2.0;
    const double cen0 = cx + mx / (3.0 * sa), cen1 = cy + my / (3.0 * sa);
    // faces: planes in order, the first two vertices on each give its edge
    double area[T2P];
    unsigned valid = 0;
    int nf = 0;
    for (int p = 0; p < nb_v; p++) {
        int cnt = 0, v0 = -1, v1 = -1;
        for (int i = 0; i < nb_t; i++)
            if ((int)tri_a(tri[i]) == p || (int)tri_b(tri[i]) == p) {
                if (cnt == 0) v0 = i; else if (cnt == 1) v1 = i;
                cnt++;
            }
        if (cnt >= 2) {
            const double ddx = vx[v1] - vx[v0], ddy = vy[v1] - vy[v0];
            area[p] = sqrt(ddx * ddx + ddy * ddy);
            valid |= 1u << p;
            nf++;
        }
    }
    const double uscale = P.ip[P.inst[e]].scale_out;
    const double vscale = uscale * uscale, ascale = uscale;
    const unsigned long long base = atomicAdd(P.face_counter, (unsigned long long)nf);
    const bool fits = base + (unsigned long long)nf <= P.face_cap;
    if (!fits) {
        atomicOr(P.overflow, 1u);
    } else {
        int idx = 0;
        for (int p = 0; p < nb_v; p++) {
            if (!((valid >> p) & 1u)) continue;
            const size_t f = base + idx++;
            const double4 pe = hp[p];
            const double nlen = sqrt(pe.x * pe.x + pe.y * pe.y + pe.z * pe.z);  // compute_face_normal
            const int nbr = vid[p];
            P.f_nb[f] = nbr;
            uint32_t own = BOX_FACE;
            if (nbr >= 0) {
                if ((int64_t)nbr < P.n_hydro)
                    own = pack_owner((uint32_t)nbr, 0);
                else
                    own = pack_owner(P.ghost_src[nbr - P.n_hydro], P.ghost_code[nbr - P.n_hydro]);
            }
            P.f_own[f] = own;
            P.f_geo[f] = make_double4(pe.x / nlen, pe.y / nlen, pe.z / nlen, ascale * area[p]);
        }
    }
    P.vol[e] = vscale * cell_vol;
    P.fptr[e] = fits ? (uint32_t)base : 0u;
    P.fcnt[e] = fits ? (uint32_t)nf : 0u;
    P.status[e] = ST_SUCCESS;
    P.certk[e] = certk;
    P.centroid[3 * (size_t)e] = (cen0 - 0.5) * uscale + 0.5;
    P.centroid[3 * (size_t)e + 1] = (cen1 - 0.5) * uscale + 0.5;
    P.centroid[3 * (size_t)e + 2] = 0.0;
}

}  // namespace

namespace {

inline unsigned nblk(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

__global__ void k_mark_not_computed(int* __restrict__ status, int* __restrict__ certk, int64_t from, int64_t to) {
    int64_t e = from + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= to) return;
    status[e] = ST_NOT_COMPUTED;
    certk[e] = 0;
}

// out[off[t]] = qs[t] (sorted positions) or t (query slots) for flagged t
__global__ void k_compact_list(const uint32_t* __restrict__ qs, const uint32_t* __restrict__ flag,
                               const uint32_t* __restrict__ off, int64_t nq, int as_slots, uint32_t* __restrict__ out) {
    int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nq) return;
    if (flag[t]) out[off[t]] = as_slots ? (uint32_t)t : qs[t];
}

// flag[t] = cell of query slot t (hydro only if hydro_only) has status `code`
__global__ void k_flag_status(const uint32_t* __restrict__ qs, const uint32_t* __restrict__ perm,
                              const int* __restrict__ status, int64_t nq, int64_t n_hydro, int hydro_only, int code,
                              uint32_t* __restrict__ flag) {
    int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nq) return;
    const uint32_t e = perm[qs[t]];
    const int st = status[e];
    // code < 0: any failure (not SUCCESS, not skipped, not waiting for the FP64 re-clip)
    const bool match = code >= 0 ? st == code : (st != ST_SUCCESS && st != ST_NOT_COMPUTED && st != ST_RECLIP);
    flag[t] = ((!hydro_only || e < (uint32_t)n_hydro) && match) ? 1u : 0u;
}

// Compacts the cells whose status is `code` into `out` (query slots, or sorted
// positions when as_slots is false); returns the count.
cudaError_t select_cells(pgpu_ctx* c, int code, bool hydro_only, bool as_slots, uint32_t* out, uint32_t* count) {
    cudaError_t e = cudaSuccess;
    const int64_t nq = c->n_query;
    uint32_t* flag = ensure<uint32_t>(c->qflag, nq + 1, &e);
    uint32_t* off = ensure<uint32_t>(c->qoff, nq + 1, &e);
    if (e) return e;
    k_flag_status<<<nblk(nq, 256), 256, 0, c->stream>>>((const uint32_t*)c->qs.p, (const uint32_t*)c->perm.p,
                                                         (const int*)c->status.p, nq, c->n_hydro, hydro_only ? 1 : 0,
                                                         code, flag);
    if ((e = exclusive_scan_u32(flag, off, nq, c->scan_tmp, c->stream))) return e;
    k_compact_list<<<nblk(nq, 256), 256, 0, c->stream>>>((const uint32_t*)c->qs.p, flag, off, nq, as_slots ? 1 : 0,
                                                          out);
    count_launches(2);
    if ((e = cudaMemcpyAsync(count, off + nq, sizeof(uint32_t), cudaMemcpyDeviceToHost, c->stream))) return e;
    return cudaStreamSynchronize(c->stream);
}


// One clipping pass over the query list qs[0, nq) with K-neighbour lists `knn`.
// reset: start a fresh face array (else faces are appended to the current one).
cudaError_t clip_pass(pgpu_ctx* c, const uint32_t* qs, int64_t nq, int K, const uint32_t* knn, bool reset,
                      unsigned long long* fc, unsigned* overflow, unsigned* uncert, bool fp32 = false,
                      unsigned* reclip = nullptr, const uint32_t* slots = nullptr, const uint16_t* kq = nullptr,
                      bool pruned = false, bool thread2d = false) {
    const int D = c->prm.dim;
    cudaError_t e = cudaSuccess;
    DevScalars* sc = (DevScalars*)c->scalars.p;
    if (reset && (e = cudaMemsetAsync(&sc->face_count, 0, sizeof(unsigned long long), c->stream))) return e;
    if ((e = cudaMemsetAsync(&sc->overflow, 0, sizeof(unsigned int), c->stream))) return e;
    if ((e = cudaMemsetAsync(&sc->uncertified, 0, sizeof(unsigned int), c->stream))) return e;
    if ((e = cudaMemsetAsync(&sc->reclip, 0, sizeof(unsigned int), c->stream))) return e;
    ClipParams P;
    P.qs = qs;
    P.slots = slots;
    P.perm = (const uint32_t*)c->perm.p;
    P.spts = c->spts.p;
    P.ext = c->ext.p;
    P.knn = knn;
    P.kq = kq;
    P.ghost_src = (const uint32_t*)c->ghost_src.p;
    P.ghost_code = (const uint32_t*)c->ghost_code.p;
    P.nq = nq;
    P.n_hydro = c->n_hydro;
    P.K = K;
    P.robust = c->prm.predicates == PGPU_PRED_ROBUST;
    P.uncertified = &sc->uncertified;
    P.reclip = &sc->reclip;
    P.ip = (const InstPar*)c->inst.d_par.p;
    P.inst = (const uint16_t*)c->inst.d_inst_e.p;
    P.vol = (double*)c->vol.p;
    P.fptr = (uint32_t*)c->fptr.p;
    P.fcnt = (uint32_t*)c->fcnt.p;
    P.status = (int*)c->status.p;
    P.certk = (int*)c->certk.p;
    P.centroid = (double*)c->centroid.p;
    P.f_nb = (int32_t*)c->f_nb.p;
    P.f_own = (uint32_t*)c->f_own.p;
    P.f_geo = (double4*)c->f_geo.p;
    P.face_counter = &sc->face_count;
    P.walk_stats = &sc->walk_points;
    P.overflow = &sc->overflow;
    P.face_cap = c->face_cap;
    // the shortest list any form builds: the smallest learned class (capped at k)
    P.walk_prefix = std::min(c->prm.k, D == 3 ? 32 : 12);
    P.walk_certk = c->prm.k + 1;
    if (nq > 0) {
        const unsigned blocks = (unsigned)((nq + CLIP_WARPS - 1) / CLIP_WARPS);
        const int CW = c->tune.clip_warps;  // cells (warps) per block: autotuned, 1, 2 or 4
        const unsigned blocks_cw = (unsigned)((nq + CW - 1) / CW);
        if (thread2d && D == 2 && !slots) {
            k_clip2t<<<(unsigned)((nq + T2_THREADS - 1) / T2_THREADS), T2_THREADS, 0, c->stream>>>(P);
        } else if (pruned) {
            const SubGrid g = {(const InstPar*)c->inst.d_par.p, (const uint16_t*)c->inst.d_inst_e.p,
                               (const uint8_t*)c->bin_lvl.p, (const uint32_t*)c->sub_off.p,
                               (const uint32_t*)c->sub_start.p};
            const int2* tab = (const int2*)c->knn_table.p;
            if (D == 2)
                k_clip_pruned<2><<<blocks, CLIP_WARPS * 32, 0, c->stream>>>(P, g, tab, c->knn_table_n,
                                                                            c->knn_table_r);
            else
                k_clip_pruned<3><<<blocks, CLIP_WARPS * 32, 0, c->stream>>>(P, g, tab, c->knn_table_n,
                                                                            c->knn_table_r);
        } else if (fp32) {
            // one cell per block frees each warp's slot as soon as its own cell is done
            // (no warp waits for its block mates); the autotuner picks
            if (D == 2) {
                if (CW == 1) k_clip32<2, 1><<<blocks_cw, 32, 0, c->stream>>>(P);
                else if (CW == 2) k_clip32<2, 2><<<blocks_cw, 64, 0, c->stream>>>(P);
                else k_clip32<2, 4><<<blocks_cw, 128, 0, c->stream>>>(P);
            } else {
                if (CW == 1) k_clip32<3, 1><<<blocks_cw, 32, 0, c->stream>>>(P);
                else if (CW == 2) k_clip32<3, 2><<<blocks_cw, 64, 0, c->stream>>>(P);
                else k_clip32<3, 4><<<blocks_cw, 128, 0, c->stream>>>(P);
            }
        } else {
            if (D == 2) {
                if (CW == 1) k_clip<2, 1><<<blocks_cw, 32, 0, c->stream>>>(P);
                else if (CW == 2) k_clip<2, 2><<<blocks_cw, 64, 0, c->stream>>>(P);
                else k_clip<2, 4><<<blocks_cw, 128, 0, c->stream>>>(P);
            } else {
                if (CW == 1) k_clip<3, 1><<<blocks_cw, 32, 0, c->stream>>>(P);
                else if (CW == 2) k_clip<3, 2><<<blocks_cw, 64, 0, c->stream>>>(P);
                else k_clip<3, 4><<<blocks_cw, 128, 0, c->stream>>>(P);
            }
        }
        count_launches(1);
    }
    if ((e = cudaGetLastError())) return e;
    if ((e = cudaMemcpyAsync(fc, &sc->face_count, sizeof(*fc), cudaMemcpyDeviceToHost, c->stream))) return e;
    if ((e = cudaMemcpyAsync(overflow, &sc->overflow, sizeof(*overflow), cudaMemcpyDeviceToHost, c->stream))) return e;
    if ((e = cudaMemcpyAsync(uncert, &sc->uncertified, sizeof(*uncert), cudaMemcpyDeviceToHost, c->stream))) return e;
    if (reclip && (e = cudaMemcpyAsync(reclip, &sc->reclip, sizeof(*reclip), cudaMemcpyDeviceToHost, c->stream)))
        return e;
    return cudaStreamSynchronize(c->stream);
}

}  // namespace

cudaError_t launch_clip(pgpu_ctx* c) {
    const int D = c->prm.dim;
    cudaError_t e = cudaSuccess;
    const int64_t n = c->n_ext;
    ensure<double>(c->vol, n + 1, &e);
    ensure<uint32_t>(c->fptr, n + 1, &e);
    ensure<uint32_t>(c->fcnt, n + 1, &e);
    ensure<int>(c->status, n + 1, &e);
    ensure<int>(c->certk, n + 1, &e);
    ensure<double>(c->centroid, 3 * n + 3, &e);
    if (e) return e;
    if (!c->all_cells && c->n_ext > c->n_hydro) {
        // ghost cells are not computed in the per-step path
        if ((e = cudaMemsetAsync(c->fcnt.p, 0, (n + 1) * sizeof(uint32_t), c->stream))) return e;
        if ((e = cudaMemsetAsync(c->vol.p, 0, (n + 1) * sizeof(double), c->stream))) return e;
        k_mark_not_computed<<<nblk(n - c->n_hydro, 256), 256, 0, c->stream>>>((int*)c->status.p, (int*)c->certk.p,
                                                                              c->n_hydro, n);
        count_launches(1);
    }
    for (int attempt = 0; attempt < 3; attempt++) {
        size_t want = c->face_cap;
        const size_t est = (size_t)c->n_query * (D == 2 ? 8 : 20) + 1024;
        if (want < est) want = est;
        ensure<int32_t>(c->f_nb, want, &e);
        ensure<uint32_t>(c->f_own, want, &e);
        ensure<double4>(c->f_geo, want, &e);
        if (e) return e;
        c->face_cap = want;
        unsigned long long fc = 0;
        unsigned of = 0, unc = 0, rc = 0;
        const bool fp32 = c->prm.precision == PGPU_CLIP_FP32;
        const uint16_t* kq = c->use_kq ? (const uint16_t*)c->kq.p : nullptr;
        // 2D: a thread per cell when the autotuner chose it (cells beyond its capacity come back as RECLIP)
        if ((e = clip_pass(c, (const uint32_t*)c->qs.p, c->n_query, c->knn_stride, (const uint32_t*)c->knn.p, true, &fc,
                           &of, &unc, fp32, &rc, nullptr, kq, false, c->tune.clip_thread && D == 2)))
            return e;
        c->n_reclip = rc;
        if (!of && rc > 0) {
            // cells the FP32 clip could not decide (or too big for a thread): the FP64 warp kernel, faces appended
            uint32_t* fq = ensure<uint32_t>(c->fb_qs, c->n_query + 1, &e);
            if (e) return e;
            uint32_t nr = 0;
            if ((e = select_cells(c, ST_RECLIP, false, true, fq, &nr))) return e;
            unsigned unc2 = 0, rc2 = 0;
            if ((e = clip_pass(c, (const uint32_t*)c->qs.p, nr, c->knn_stride, (const uint32_t*)c->knn.p, false, &fc, &of,
                               &unc2, false, &rc2, fq, kq)))
                return e;
            unc += unc2;
        }
        c->num_faces = (int64_t)fc;
        c->n_uncertified = unc;
        c->n_refit = 0;
        if (!of) return cudaSuccess;
        c->face_cap = (size_t)fc * 5 / 4 + 1024;  // retry with room for all faces
    }
    return cudaErrorMemoryAllocation;
}

cudaError_t launch_fallback(pgpu_ctx* c, int K2) {
    cudaError_t e = cudaSuccess;
    const int64_t nq = c->n_query;
    c->n_refit = 0;
    uint32_t* fq = ensure<uint32_t>(c->fb_qs, nq + 1, &e);
    if (e) return e;
    uint32_t nf = 0;
    if ((e = select_cells(c, ST_SECURITY_RADIUS_NOT_REACHED, true, false, fq, &nf))) return e;
    if (nf == 0) return cudaSuccess;
    uint32_t* kl = ensure<uint32_t>(c->fb_knn, (size_t)nf * K2 + 1, &e);
    if (e) return e;
    if ((e = launch_knn_list(c, fq, nf, K2, kl, nullptr, K2))) return e;
    unsigned long long fc = 0;
    unsigned of = 0, unc = 0;
    if ((e = clip_pass(c, fq, nf, K2, kl, false, &fc, &of, &unc))) return e;
    if (of) return cudaErrorMemoryAllocation;
    c->num_faces = (int64_t)fc;
    c->n_uncertified = unc;
    c->n_refit = nf;
    return cudaSuccess;
}

// Hydro cells still failed after the neighbour lists (uncertified, or any other
// failure): clipped again by the grid walk of k_clip_pruned, faces appended.
cudaError_t launch_pruned(pgpu_ctx* c) {
    cudaError_t e = cudaSuccess;
    const int64_t nq = c->n_query;
    uint32_t* fq = ensure<uint32_t>(c->fb_qs, nq + 1, &e);
    if (e) return e;
    uint32_t nf = 0;
    c->n_pruned = 0;
    DevScalars* sc = (DevScalars*)c->scalars.p;
    if ((e = cudaMemsetAsync(&sc->walk_points, 0, 2 * sizeof(unsigned long long), c->stream))) return e;
    if ((e = select_cells(c, -1, true, true, fq, &nf))) return e;
    if (nf == 0) return cudaSuccess;
    unsigned long long fc = 0;
    unsigned of = 0, unc = 0;
    // work items are query slots: the walk starts from each cell's own neighbour list
    const uint16_t* kq = c->use_kq ? (const uint16_t*)c->kq.p : nullptr;
    if ((e = clip_pass(c, (const uint32_t*)c->qs.p, nf, c->knn_stride, (const uint32_t*)c->knn.p, false, &fc, &of,
                       &unc, false, nullptr, fq, kq, true)))
        return e;
    if (of) return cudaErrorMemoryAllocation;
    c->num_faces = (int64_t)fc;
    c->n_uncertified = unc;
    c->n_pruned = nf;
    return cudaSuccess;
}

}  // namespace pgpu
