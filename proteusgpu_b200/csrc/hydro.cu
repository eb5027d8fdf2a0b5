// Hydro on the device mesh.
//
// Reference semantics (src/hydro/finite_volume_solver.cpp:43-186):
//   k_dt_ref    hydro::dt_CFL   min over cells of CFL R_i / (c_i + |v_i|)
//   k_hydro_ref hydro::hydro_step: per cell, sum over its faces of the HLL flux
//               (riemann.cpp:7-45) times the face area, then
//               rho' = rho - dt/V F_rho, v' = (rho v - dt/V F_m) / rho',
//               E' = E - dt/V F_E, written to a second buffer.
// Moving-mesh form (extension; the reference never moves its mesh):
//   k_prim_dt     primitives from the conserved mass, momentum and energy on
//                 the new mesh, and the CFL step in the same pass;
//   k_flux_update HLL fluxes with the conserved update and the drift of the
//                 generating point, one thread per cell gathering its faces
//                 (no atomics).  In PGPU_FLUX_PHYSICAL mode the normal is the
//                 outward one and the area is the one the lower hydro id
//                 computed for that face, so each face's flux cancels exactly
//                 between its two cells.
// All arithmetic is FP64 without FMA, operation for operation the reference's,
// so a flux computed from the same inputs is bit-identical.
#include <math_constants.h>

#include <mutex>

#include "pgpu_common.cuh"
#include "pgpu_ctx.h"

namespace pgpu {
namespace {

constexpr int HT = 256;  // threads per block

inline unsigned nblk(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

__device__ __forceinline__ double block_min(double v) {
    __shared__ double sm[HT / 32];
    for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
    if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x < 32) {
        v = threadIdx.x < HT / 32 ? sm[threadIdx.x] : CUDART_INF;
        for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
    }
    return v;
}

template <int D>
__device__ __forceinline__ double dt_cell(const Prim& s, double V, double cfl, double gamma) {
    double P = pressure<D>(s, gamma);
    double c = sqrt(gamma * P / s.rho);
    double R, va;
    if (D == 2) {
        R = sqrt(V / CUDART_PI);
        va = sqrt(s.vx * s.vx + s.vy * s.vy);
    } else {
        R = cbrt(3.0 * V / (4.0 * CUDART_PI));
        va = sqrt(s.vx * s.vx + s.vy * s.vy + s.vz * s.vz);
    }
    return cfl * (R / (c + va));
}

template <int D>
__device__ __forceinline__ Prim load_prim(const double* rho, const double* v, const double* E, int64_t i) {
    Prim s;
    s.rho = rho[i];
    s.vx = v[i * D];
    s.vy = v[i * D + 1];
    s.vz = D == 3 ? v[i * D + 2] : 0.0;
    s.E = E[i];
    return s;
}

// ---- reference hydro::dt_CFL
template <int D>
__global__ void k_dt_ref(const double* __restrict__ rho, const double* __restrict__ v, const double* __restrict__ E,
                         const double* __restrict__ vol, int64_t n, double cfl, double gamma,
                         unsigned long long* __restrict__ dt_bits) {
    int64_t i = (int64_t)blockIdx.x * HT + threadIdx.x;
    double d = 1e100;
    if (i < n) d = dt_cell<D>(load_prim<D>(rho, v, E, i), vol[i], cfl, gamma);
    d = block_min(d);
    if (threadIdx.x == 0) atomicMin(dt_bits, dbits(d));
}

// ---- reference hydro::hydro_step on primitives (rho, v, E) -> (rho2, v2, E2)
template <int D, bool PHYSICAL>
__global__ void k_hydro_ref(const double* __restrict__ rho, const double* __restrict__ v,
                            const double* __restrict__ E, const double* __restrict__ vol,
                            const uint32_t* __restrict__ fptr, const uint32_t* __restrict__ fcnt,
                            const uint32_t* __restrict__ f_own, const double4* __restrict__ f_geo, int64_t n,
                            double dt, double gamma, double* __restrict__ rho2, double* __restrict__ v2,
                            double* __restrict__ E2, unsigned int* __restrict__ box_faces) {
    int64_t i = (int64_t)blockIdx.x * HT + threadIdx.x;
    if (i >= n) return;
    const Prim si = load_prim<D>(rho, v, E, i);
    double tr = 0, tx = 0, ty = 0, tz = 0, te = 0;
    const uint32_t fp = fptr[i], nf = fcnt[i];
    unsigned nbox = 0;
    for (uint32_t q = 0; q < nf; q++) {
        const uint32_t own = f_own[fp + q];
        const double4 g = f_geo[fp + q];
        int64_t h = i;
        if (own == BOX_FACE) nbox++;
        else h = own & OWNER_MASK;
        const Prim sj = load_prim<D>(rho, v, E, h);
        const Flux fl = PHYSICAL ? hll<D>(si, sj, -g.x, -g.y, -g.z, gamma) : hll<D>(si, sj, g.x, g.y, g.z, gamma);
        const double A = g.w;
        tr += fl.rho * A;
        tx += fl.mx * A;
        ty += fl.my * A;
        if (D == 3) tz += fl.mz * A;
        te += fl.E * A;
    }
    if (nbox) atomicAdd(box_faces, nbox);
    const double V = vol[i];
    const double frac = dt / V;
    const double nr = si.rho - frac * tr;
    const double inv = 1.0 / nr;
    rho2[i] = nr;
    v2[i * D] = (si.rho * si.vx - frac * tx) * inv;
    v2[i * D + 1] = (si.rho * si.vy - frac * ty) * inv;
    if (D == 3) v2[i * D + 2] = (si.rho * si.vz - frac * tz) * inv;
    E2[i] = si.E - frac * te;
}

// ---- moving mesh: conserved variables from primitives on the first mesh
template <int D>
__global__ void k_cons_from_prim(const double* __restrict__ rho, const double* __restrict__ v,
                                 const double* __restrict__ E, const double* __restrict__ dep,
                                 const double* __restrict__ vol, int64_t n, double* __restrict__ mass,
                                 double* __restrict__ mom, double* __restrict__ en) {
    int64_t i = (int64_t)blockIdx.x * HT + threadIdx.x;
    if (i >= n) return;
    const double V = vol[i];
    mass[i] = rho[i] * V;
#pragma unroll
    for (int a = 0; a < D; a++) mom[i * D + a] = (rho[i] * v[i * D + a]) * V;
    double e = E[i] * V;
    if (dep) e = e + dep[i];
    en[i] = e;
}

// ---- moving mesh: primitives + CFL step (+ failed-cell and cert-K statistics)
template <int D>
__global__ void k_prim_dt(const double* __restrict__ mass, const double* __restrict__ mom,
                          const double* __restrict__ en, const double* __restrict__ vol,
                          const int* __restrict__ status, const int* __restrict__ certk, int64_t n, double cfl,
                          const InstPar* __restrict__ ip, const uint16_t* __restrict__ inst,
                          unsigned long long* __restrict__ dt_inst, double4* __restrict__ w4,
                          double* __restrict__ we, DevScalars* __restrict__ sc) {
    int64_t i = (int64_t)blockIdx.x * HT + threadIdx.x;
    double d = 1e100;
    const int b = i < n ? inst[i] : -1;
    if (i < n) {
        const double gamma = ip[b].gamma;
        const double V = vol[i];
        const double m = mass[i];
        if (status[i] != ST_SUCCESS || !(V > 0.0)) {
            // a cell without a mesh cell this step keeps its conserved state: density -1
            // marks it for k_flux_update (no fluxes, its faces are walls), it drifts with
            // its velocity and takes no part in the time step
            const double im = m > 0.0 ? 1.0 / m : 0.0;
            w4[i] = make_double4(-1.0, mom[i * D] * im, mom[i * D + 1] * im, D == 3 ? mom[i * D + 2] * im : 0.0);
            we[i] = 0.0;
            atomicAdd(&sc->failed, 1u);
        } else {
            Prim s;
            s.rho = m / V;
            s.vx = mom[i * D] / m;
            s.vy = mom[i * D + 1] / m;
            s.vz = D == 3 ? mom[i * D + 2] / m : 0.0;
            s.E = en[i] / V;
            w4[i] = make_double4(s.rho, s.vx, s.vy, s.vz);
            we[i] = s.E;
            d = dt_cell<D>(s, V, cfl, gamma);
            atomicMax(&sc->cert_k_max, certk[i]);
        }
    }
    // each instance has its own time step; a block inside one instance reduces first
    __shared__ int s_b0;
    if (threadIdx.x == 0) s_b0 = b;
    __syncthreads();
    const int b0 = s_b0;
    const bool uniform = __syncthreads_and(b == b0 || b < 0) != 0;
    if (uniform) {
        const double m = block_min(d);
        if (threadIdx.x == 0) {
            atomicMin(&sc->dt_bits, dbits(m));
            if (b0 >= 0) atomicMin(&dt_inst[b0], dbits(m));
        }
    } else {
        const double m = block_min(d);
        if (threadIdx.x == 0) atomicMin(&sc->dt_bits, dbits(m));
        if (b >= 0) atomicMin(&dt_inst[b], dbits(d));
    }
}

// Index in its cell's face list (records hp .. hp + hn - 1) of the first face whose
// owner record is want, or -1.  Eight records are loaded per step, independently of one
// another, so a search costs about one dependent load round trip per eight records
// instead of one per record (16.8M clustered cells: flux 28.4 -> 22.6 ms).
__device__ __forceinline__ int partner_face(const uint32_t* __restrict__ f_own, uint32_t hp, uint32_t hn,
                                            uint32_t want) {
    constexpr int W = 8;
    for (uint32_t r0 = 0; r0 < hn; r0 += W) {
        uint32_t v[W];
#pragma unroll
        for (int j = 0; j < W; j++) v[j] = r0 + j < hn ? f_own[hp + r0 + j] : BOX_FACE;
        int hit = -1;
#pragma unroll
        for (int j = W - 1; j >= 0; j--)
            if (v[j] == want) hit = (int)(r0 + j);
        if (hit >= 0) return hit;
    }
    return -1;
}

// 24 warps per SM (at most 85 registers a thread; the HLL arithmetic spills a little):
// the gathers of the neighbours' states and faces are latency bound, more resident
// warps hide more of them (16.8M points: 31.4 -> 28.4 ms).  Blocks of two warps, so that
// a block's slot is free again soon after its own slowest cell (23.7 -> 23.1 ms).
constexpr int FT = 64;  // flux threads per block
template <int D, bool PHYSICAL, int MIRROR>
__global__ void __launch_bounds__(FT, 12) k_flux_update(const double4* __restrict__ w4, const double* __restrict__ we,
                              const uint32_t* __restrict__ fptr, const uint32_t* __restrict__ fcnt,
                              const uint32_t* __restrict__ f_own, const double4* __restrict__ f_geo, int64_t n,
                              const InstPar* __restrict__ ip, const uint16_t* __restrict__ inst,
                              const unsigned long long* __restrict__ dt_inst, double fixed_dt,
                              double* __restrict__ mass, double* __restrict__ mom, double* __restrict__ en,
                              double* __restrict__ pos, DevScalars* __restrict__ sc,
                              const uint32_t* __restrict__ order, const uint32_t* __restrict__ perm) {
    const int64_t t = (int64_t)blockIdx.x * FT + threadIdx.x;
    if (t >= n) return;
    // cells in the mesh's spatial order when given (the query list: sorted positions of
    // the hydro cells): neighbouring threads then read neighbouring faces and share
    // neighbour states in cache.  Every cell's arithmetic is the same either way.
    const int64_t i = order ? (int64_t)perm[order[t]] : t;
    const int b = inst[i];
    const double gamma = ip[b].gamma;
    // MIRROR 0 / 1: every instance periodic / walled; 2: per instance
    const bool mirror = MIRROR == 2 ? ip[b].mirror != 0 : MIRROR == 1;
    const double dt = fixed_dt > 0 ? fixed_dt : __longlong_as_double((long long)dt_inst[b]);
    const double4 wi = w4[i];
    const Prim si = {wi.x, wi.y, wi.z, wi.w, we[i]};
    double tr = 0, tx = 0, ty = 0, tz = 0, te = 0;
    const bool alive = wi.x >= 0.0;  // density -1: no mesh cell this step
    const uint32_t fp = fptr[i], nf = alive ? fcnt[i] : 0u;
    unsigned nbox = 0, nunp = 0;
    for (uint32_t q = 0; q < nf; q++) {
        const uint32_t own = f_own[fp + q];
        const double4 g = f_geo[fp + q];
        uint32_t h = (uint32_t)i;
        uint32_t code = 0;
        double A = g.w;
        if (own == BOX_FACE) {
            nbox++;
        } else {
            h = own & OWNER_MASK;
            code = own >> OWNER_BITS;
            if (PHYSICAL && h < (uint32_t)i) {
                // the lower hydro id's value of this face's area
                const uint32_t want = pack_owner((uint32_t)i, reverse_code(code, D, !mirror));
                const uint32_t hp = fptr[h];
                const int r = partner_face(f_own, hp, fcnt[h], want);
                if (r >= 0)
                    A = f_geo[hp + r].w;
                else if (w4[h].x >= 0.0)
                    nunp++;
            }
        }
        const double4 wj4 = w4[h];
        if (wj4.x < 0.0) continue;  // the neighbour has no mesh cell this step: a wall
        Prim sj = {wj4.x, wj4.y, wj4.z, wj4.w, we[h]};
        if (mirror && code) {
            uint32_t cd = code;
            if (cd % 3) sj.vx = -sj.vx;
            cd /= 3;
            if (cd % 3) sj.vy = -sj.vy;
            cd /= 3;
            if (D == 3 && (cd % 3)) sj.vz = -sj.vz;
        }
        const Flux fl = PHYSICAL ? hll<D>(si, sj, -g.x, -g.y, -g.z, gamma) : hll<D>(si, sj, g.x, g.y, g.z, gamma);
        tr += fl.rho * A;
        tx += fl.mx * A;
        ty += fl.my * A;
        if (D == 3) tz += fl.mz * A;
        te += fl.E * A;
    }
    if (nbox) atomicAdd(&sc->box_faces, nbox);
    if (nunp) atomicAdd(&sc->unpaired, nunp);
    mass[i] = mass[i] - dt * tr;
    mom[i * D] = mom[i * D] - dt * tx;
    mom[i * D + 1] = mom[i * D + 1] - dt * ty;
    if (D == 3) mom[i * D + 2] = mom[i * D + 2] - dt * tz;
    en[i] = en[i] - dt * te;
    // drift with the cell's velocity at the start of the step, then wrap or reflect
    const double vv[3] = {si.vx, si.vy, si.vz};
#pragma unroll
    for (int a = 0; a < D; a++) {
        double p = pos[i * D + a] + vv[a] * dt;
        if (!mirror) {
            if (p < 0.0) p += 1.0;
            if (p >= 1.0) p -= 1.0;
        } else {
            if (p < 0.0) p = -p;
            if (p >= 1.0) p = 2.0 - p;
            if (p >= 1.0) p = 0x1.fffffffffffffp-1;
        }
        pos[i * D + a] = p;
    }
}

// ---- moving faces (extension): the faces move with the generators, so the
// Riemann problem is solved in the face's frame (Pakmor et al. 2011); second
// order by MUSCL-Hancock with least-squares gradients (Springel 2010,
// Pakmor et al. 2016).  Periodic boxes.  Primitives W = (rho, v, P), NV = D + 2.
// The operation order follows the oracle's om_step_ale.
template <int D>
__device__ __forceinline__ void ale_prim(const double4* __restrict__ w4, const double* __restrict__ we, uint32_t h,
                                         double gamma, double* W) {
    const double4 a = w4[h];
    const Prim s = {a.x, a.y, a.z, a.w, we[h]};
    W[0] = s.rho;
    W[1] = s.vx;
    W[2] = s.vy;
    if (D == 3) W[3] = s.vz;
    W[D + 1] = pressure<D>(s, gamma);
}

template <int D>
__device__ __forceinline__ double dotd(const double* a, const double* b) {
    double s = a[0] * b[0] + a[1] * b[1];
    if (D == 3) s = s + a[2] * b[2];
    return s;
}

// generator offset of a face: the neighbour's image minus the cell, physical units
template <int D>
__device__ __forceinline__ void ale_offset(const typename PointOf<D>::type* __restrict__ ext, int32_t nb, uint32_t i,
                                           double scale, double* d) {
    const typename PointOf<D>::type pe = ext[nb], pc = ext[i];
    d[0] = (pe.x - pc.x) * scale;
    d[1] = (pe.y - pc.y) * scale;
    d[2] = D == 3 ? (pz(pe) - pz(pc)) * scale : 0.0;
}

// Per cell: least-squares gradients of W, the limiter, and the half-step prediction in
// the cell's frame: wp[i * NV + k], grad[(i * NV + k) * D + a].
template <int D>
__global__ void k_ale_grad(const double4* __restrict__ w4, const double* __restrict__ we,
                           const uint32_t* __restrict__ fptr, const uint32_t* __restrict__ fcnt,
                           const uint32_t* __restrict__ f_own, const int32_t* __restrict__ f_nb,
                           const double4* __restrict__ f_geo, const typename PointOf<D>::type* __restrict__ ext,
                           int64_t n, const InstPar* __restrict__ ip, const uint16_t* __restrict__ inst,
                           const unsigned long long* __restrict__ dt_inst, double fixed_dt,
                           double* __restrict__ wp, double* __restrict__ grad, const uint32_t* __restrict__ order,
                           const uint32_t* __restrict__ perm) {
    constexpr int NV = D + 2, IP = D + 1;
    const int64_t t = (int64_t)blockIdx.x * HT + threadIdx.x;
    if (t >= n) return;
    const int64_t i = order ? (int64_t)perm[order[t]] : t;
    const int b = inst[i];
    const double gamma = ip[b].gamma, scale = ip[b].scale_out;
    const double dt = fixed_dt > 0 ? fixed_dt : __longlong_as_double((long long)dt_inst[b]);
    double Wi[NV];
    ale_prim<D>(w4, we, (uint32_t)i, gamma, Wi);
    double* gi = grad + (size_t)i * NV * D;
    if (!(Wi[0] >= 0.0)) {  // no mesh cell this step
        for (int k = 0; k < NV; k++) {
            wp[i * NV + k] = Wi[k];
            for (int a = 0; a < D; a++) gi[k * D + a] = 0.0;
        }
        return;
    }
    double M[6] = {0, 0, 0, 0, 0, 0}, bb[NV][3], wmax[NV], wmin[NV];
    for (int k = 0; k < NV; k++) {
        bb[k][0] = bb[k][1] = bb[k][2] = 0.0;
        wmax[k] = wmin[k] = Wi[k];
    }
    const uint32_t fp = fptr[i], nf = fcnt[i];
    for (uint32_t q = 0; q < nf; q++) {
        const uint32_t own = f_own[fp + q];
        if (own == BOX_FACE) continue;
        const uint32_t h = own & OWNER_MASK;
        if (w4[h].x < 0.0) continue;
        double d[3], Wh[NV];
        ale_offset<D>(ext, f_nb[fp + q], (uint32_t)i, scale, d);
        ale_prim<D>(w4, we, h, gamma, Wh);
        const double wgt = f_geo[fp + q].w / dotd<D>(d, d);
        M[0] += wgt * d[0] * d[0];
        M[1] += wgt * d[0] * d[1];
        M[3] += wgt * d[1] * d[1];
        if (D == 3) {
            M[2] += wgt * d[0] * d[2];
            M[4] += wgt * d[1] * d[2];
            M[5] += wgt * d[2] * d[2];
        }
#pragma unroll
        for (int k = 0; k < NV; k++) {
            const double dw = Wh[k] - Wi[k];
            for (int a = 0; a < D; a++) bb[k][a] += wgt * dw * d[a];
            wmax[k] = dmax_ref(wmax[k], Wh[k]);
            wmin[k] = dmin_ref(wmin[k], Wh[k]);
        }
    }
    double g[NV][3];
#pragma unroll
    for (int k = 0; k < NV; k++) {
        if (D == 2) {
            const double det = M[0] * M[3] - M[1] * M[1];
            g[k][0] = (M[3] * bb[k][0] - M[1] * bb[k][1]) / det;
            g[k][1] = (M[0] * bb[k][1] - M[1] * bb[k][0]) / det;
            g[k][2] = 0.0;
        } else {
            const double c00 = M[3] * M[5] - M[4] * M[4];
            const double c01 = M[2] * M[4] - M[1] * M[5];
            const double c02 = M[1] * M[4] - M[2] * M[3];
            const double c11 = M[0] * M[5] - M[2] * M[2];
            const double c12 = M[1] * M[2] - M[0] * M[4];
            const double c22 = M[0] * M[3] - M[1] * M[1];
            const double det = M[0] * c00 + M[1] * c01 + M[2] * c02;
            g[k][0] = (c00 * bb[k][0] + c01 * bb[k][1] + c02 * bb[k][2]) / det;
            g[k][1] = (c01 * bb[k][0] + c11 * bb[k][1] + c12 * bb[k][2]) / det;
            g[k][2] = (c02 * bb[k][0] + c12 * bb[k][1] + c22 * bb[k][2]) / det;
        }
    }
    // limiter: the reconstructed value at every face midpoint stays within the
    // neighbourhood's extrema
    double alpha[NV];
    for (int k = 0; k < NV; k++) alpha[k] = 1.0;
    for (uint32_t q = 0; q < nf; q++) {
        const uint32_t own = f_own[fp + q];
        if (own == BOX_FACE) continue;
        if (w4[own & OWNER_MASK].x < 0.0) continue;
        double d[3];
        ale_offset<D>(ext, f_nb[fp + q], (uint32_t)i, scale, d);
#pragma unroll
        for (int k = 0; k < NV; k++) {
            const double dw = dotd<D>(g[k], d) * 0.5;
            double psi = 1.0;
            if (dw > 0.0)
                psi = (wmax[k] - Wi[k]) / dw;
            else if (dw < 0.0)
                psi = (wmin[k] - Wi[k]) / dw;
            alpha[k] = dmin_ref(alpha[k], psi);
        }
    }
#pragma unroll
    for (int k = 0; k < NV; k++)
        for (int a = 0; a < 3; a++) g[k][a] = alpha[k] * g[k][a];
    double div = g[1][0] + g[2][1];
    if (D == 3) div = div + g[3][2];
    const double hdt = 0.5 * dt;
    const double r = Wi[0], P = Wi[IP];
    wp[i * NV] = r - hdt * (r * div);
    for (int a = 0; a < D; a++) wp[i * NV + 1 + a] = Wi[1 + a] - hdt * (g[IP][a] / r);
    wp[i * NV + IP] = P - hdt * (gamma * P * div);
#pragma unroll
    for (int k = 0; k < NV; k++)
        for (int a = 0; a < D; a++) gi[k * D + a] = g[k][a];
}

// Per cell: moving-face HLL fluxes (face states reconstructed to the generators'
// midpoint with ORDER 2), the conserved update and the drift.  For a face whose
// other cell has the lower hydro id, the offset and area are that cell's (its
// partner face's), so both cells evaluate the same face and the fluxes cancel.
template <int D, int ORDER>
__global__ void k_ale_flux(const double4* __restrict__ w4, const double* __restrict__ we,
                           const uint32_t* __restrict__ fptr, const uint32_t* __restrict__ fcnt,
                           const uint32_t* __restrict__ f_own, const int32_t* __restrict__ f_nb,
                           const double4* __restrict__ f_geo, const typename PointOf<D>::type* __restrict__ ext,
                           int64_t n, const InstPar* __restrict__ ip, const uint16_t* __restrict__ inst,
                           const unsigned long long* __restrict__ dt_inst, double fixed_dt,
                           const double* __restrict__ wp, const double* __restrict__ grad, double* __restrict__ mass,
                           double* __restrict__ mom, double* __restrict__ en, double* __restrict__ pos,
                           DevScalars* __restrict__ sc, const uint32_t* __restrict__ order,
                           const uint32_t* __restrict__ perm) {
    constexpr int NV = D + 2, IP = D + 1;
    const int64_t t = (int64_t)blockIdx.x * HT + threadIdx.x;
    if (t >= n) return;
    const int64_t i = order ? (int64_t)perm[order[t]] : t;
    const int b = inst[i];
    const double gamma = ip[b].gamma, scale = ip[b].scale_out;
    const double dt = fixed_dt > 0 ? fixed_dt : __longlong_as_double((long long)dt_inst[b]);
    const double4 wi = w4[i];
    const bool alive = wi.x >= 0.0;
    double tr = 0, tx = 0, ty = 0, tz = 0, te = 0;
    const uint32_t fp = fptr[i], nf = alive ? fcnt[i] : 0u;
    unsigned nbox = 0, nunp = 0;
    double Wi[NV];
    if (ORDER == 1) ale_prim<D>(w4, we, (uint32_t)i, gamma, Wi);
    for (uint32_t q = 0; q < nf; q++) {
        const uint32_t own = f_own[fp + q];
        if (own == BOX_FACE) {
            nbox++;
            continue;
        }
        const uint32_t h = own & OWNER_MASK, code = own >> OWNER_BITS;
        const double4 wh = w4[h];
        if (wh.x < 0.0) continue;  // the neighbour has no mesh cell this step: a wall
        double d[3];
        double A = f_geo[fp + q].w;
        ale_offset<D>(ext, f_nb[fp + q], (uint32_t)i, scale, d);
        if (h < (uint32_t)i) {
            const uint32_t want = pack_owner((uint32_t)i, reverse_code(code, D, true));
            const uint32_t hp = fptr[h];
            const int r = partner_face(f_own, hp, fcnt[h], want);
            if (r >= 0) {
                double dh[3];
                ale_offset<D>(ext, f_nb[hp + r], h, scale, dh);
                d[0] = -dh[0];
                d[1] = -dh[1];
                d[2] = -dh[2];
                A = f_geo[hp + r].w;
            } else {
                nunp++;
            }
        }
        double L[NV], R[NV];
        if (ORDER == 1) {
            for (int k = 0; k < NV; k++) L[k] = Wi[k];
            ale_prim<D>(w4, we, h, gamma, R);
        } else {
            const double* gi = grad + (size_t)i * NV * D;
            const double* gh = grad + (size_t)h * NV * D;
            double gk[3] = {0.0, 0.0, 0.0};
#pragma unroll
            for (int k = 0; k < NV; k++) {
                for (int a = 0; a < D; a++) gk[a] = gi[k * D + a];
                L[k] = wp[i * NV + k] + dotd<D>(gk, d) * 0.5;
                for (int a = 0; a < D; a++) gk[a] = gh[k * D + a];
                R[k] = wp[(size_t)h * NV + k] - dotd<D>(gk, d) * 0.5;
            }
            if (!(L[0] > 0.0 && L[IP] > 0.0 && R[0] > 0.0 && R[IP] > 0.0)) {
                for (int k = 0; k < NV; k++) {
                    L[k] = wp[i * NV + k];
                    R[k] = wp[(size_t)h * NV + k];
                }
            }
        }
        double w[3] = {(wi.y + wh.y) * 0.5, (wi.z + wh.z) * 0.5, D == 3 ? (wi.w + wh.w) * 0.5 : 0.0};
        Prim sl = {L[0], L[1] - w[0], L[2] - w[1], D == 3 ? L[3] - w[2] : 0.0, 0.0};
        Prim sr = {R[0], R[1] - w[0], R[2] - w[1], D == 3 ? R[3] - w[2] : 0.0, 0.0};
        const double vl[3] = {sl.vx, sl.vy, sl.vz}, vr[3] = {sr.vx, sr.vy, sr.vz};
        sl.E = L[IP] / (gamma - 1.0) + 0.5 * sl.rho * dotd<D>(vl, vl);
        sr.E = R[IP] / (gamma - 1.0) + 0.5 * sr.rho * dotd<D>(vr, vr);
        const double4 g = f_geo[fp + q];
        Flux fl = hll<D>(sl, sr, -g.x, -g.y, -g.z, gamma);
        const double fm[3] = {fl.mx, fl.my, fl.mz};
        const double wm = dotd<D>(w, fm), ww = dotd<D>(w, w);
        fl.E = fl.E + wm + 0.5 * ww * fl.rho;
        fl.mx = fl.mx + w[0] * fl.rho;
        fl.my = fl.my + w[1] * fl.rho;
        if (D == 3) fl.mz = fl.mz + w[2] * fl.rho;
        tr += fl.rho * A;
        tx += fl.mx * A;
        ty += fl.my * A;
        if (D == 3) tz += fl.mz * A;
        te += fl.E * A;
    }
    if (nbox) atomicAdd(&sc->box_faces, nbox);
    if (nunp) atomicAdd(&sc->unpaired, nunp);
    mass[i] = mass[i] - dt * tr;
    mom[i * D] = mom[i * D] - dt * tx;
    mom[i * D + 1] = mom[i * D + 1] - dt * ty;
    if (D == 3) mom[i * D + 2] = mom[i * D + 2] - dt * tz;
    en[i] = en[i] - dt * te;
    const double vv[3] = {wi.y, wi.z, wi.w};
#pragma unroll
    for (int a = 0; a < D; a++) {
        double p = pos[i * D + a] + vv[a] * dt;
        if (p < 0.0) p += 1.0;
        if (p >= 1.0) p -= 1.0;
        pos[i * D + a] = p;
    }
}

// Deterministic sums (mass, momentum, energy) over hydro cells: fixed block
// partials, then one ordered pass.
template <int D>
__global__ void k_partial_sums(const double* __restrict__ mass, const double* __restrict__ mom,
                               const double* __restrict__ en, int64_t n, double* __restrict__ part) {
    __shared__ double sm[5][HT];
    int64_t i = (int64_t)blockIdx.x * HT + threadIdx.x;
    double v[5] = {0, 0, 0, 0, 0};
    if (i < n) {
        v[0] = mass[i];
        for (int a = 0; a < D; a++) v[1 + a] = mom[i * D + a];
        v[4] = en[i];
    }
    for (int k = 0; k < 5; k++) sm[k][threadIdx.x] = v[k];
    __syncthreads();
    for (int s = HT / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s)
            for (int k = 0; k < 5; k++) sm[k][threadIdx.x] += sm[k][threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int k = 0; k < 5; k++) part[blockIdx.x * 5 + k] = sm[k][0];
}

__global__ void k_final_sums(const double* __restrict__ part, int64_t nb, double* __restrict__ out) {
    if (threadIdx.x >= 5) return;
    double s = 0;
    for (int64_t b = 0; b < nb; b++) s += part[b * 5 + threadIdx.x];
    out[threadIdx.x] = s;
}

}  // namespace

cudaError_t launch_dt_ref(pgpu_ctx* c, double cfl) {
    DevScalars* sc = (DevScalars*)c->scalars.p;
    const unsigned long long init = 0x54B249AD2594C37Dull;  // bit pattern of 1e100
    cudaError_t e = cudaMemcpyAsync(&sc->dt_bits, &init, sizeof(init), cudaMemcpyHostToDevice, c->stream);
    if (e) return e;
    const int64_t n = c->n_hydro;
    if (n > 0) {
        if (c->prm.dim == 2)
            k_dt_ref<2><<<nblk(n, HT), HT, 0, c->stream>>>((const double*)c->rho.p, (const double*)c->vel.p,
                                                            (const double*)c->energy.p, (const double*)c->vol.p, n,
                                                            cfl, c->prm.gamma, &sc->dt_bits);
        else
            k_dt_ref<3><<<nblk(n, HT), HT, 0, c->stream>>>((const double*)c->rho.p, (const double*)c->vel.p,
                                                            (const double*)c->energy.p, (const double*)c->vol.p, n,
                                                            cfl, c->prm.gamma, &sc->dt_bits);
        count_launches(1);
    }
    return cudaGetLastError();
}

cudaError_t launch_hydro_ref(pgpu_ctx* c, double dt) {
    cudaError_t e = cudaSuccess;
    const int D = c->prm.dim;
    const int64_t n = c->n_hydro;
    double* r2 = ensure<double>(c->rho2, n + 1, &e);
    double* v2 = ensure<double>(c->vel2, n * D + 1, &e);
    double* e2 = ensure<double>(c->energy2, n + 1, &e);
    if (e) return e;
    DevScalars* sc = (DevScalars*)c->scalars.p;
    const bool phys = c->prm.flux_mode != PGPU_FLUX_REFERENCE;
    if (n > 0) {
#define PGPU_HREF(DD, PH)                                                                                         \
    k_hydro_ref<DD, PH><<<nblk(n, HT), HT, 0, c->stream>>>(                                                      \
        (const double*)c->rho.p, (const double*)c->vel.p, (const double*)c->energy.p, (const double*)c->vol.p, \
        (const uint32_t*)c->fptr.p, (const uint32_t*)c->fcnt.p, (const uint32_t*)c->f_own.p,                   \
        (const double4*)c->f_geo.p, n, dt, c->prm.gamma, r2, v2, e2, &sc->box_faces)
        if (D == 2) {
            if (phys) PGPU_HREF(2, true); else PGPU_HREF(2, false);
        } else {
            if (phys) PGPU_HREF(3, true); else PGPU_HREF(3, false);
        }
#undef PGPU_HREF
        count_launches(1);
    }
    if ((e = cudaGetLastError())) return e;
    std::swap(c->rho, c->rho2);
    std::swap(c->vel, c->vel2);
    std::swap(c->energy, c->energy2);
    return cudaSuccess;
}

cudaError_t launch_cons_from_prim(pgpu_ctx* c, const double* dep) {
    cudaError_t e = cudaSuccess;
    const int D = c->prm.dim;
    const int64_t n = c->n_hydro;
    ensure<double>(c->mass, n + 1, &e);
    ensure<double>(c->mom, n * D + 1, &e);
    ensure<double>(c->en, n + 1, &e);
    if (e) return e;
    if (n > 0) {
        if (D == 2)
            k_cons_from_prim<2><<<nblk(n, HT), HT, 0, c->stream>>>(
                (const double*)c->rho.p, (const double*)c->vel.p, (const double*)c->energy.p, dep,
                (const double*)c->vol.p, n, (double*)c->mass.p, (double*)c->mom.p, (double*)c->en.p);
        else
            k_cons_from_prim<3><<<nblk(n, HT), HT, 0, c->stream>>>(
                (const double*)c->rho.p, (const double*)c->vel.p, (const double*)c->energy.p, dep,
                (const double*)c->vol.p, n, (double*)c->mass.p, (double*)c->mom.p, (double*)c->en.p);
        count_launches(1);
    }
    return cudaGetLastError();
}

cudaError_t launch_prim_dt(pgpu_ctx* c, double cfl, double fixed_dt) {
    cudaError_t e = cudaSuccess;
    const int64_t n = c->n_hydro;
    double4* w4 = ensure<double4>(c->w4, n + 1, &e);
    double* we = ensure<double>(c->we, n + 1, &e);
    if (e) return e;
    DevScalars* sc = (DevScalars*)c->scalars.p;
    // reset the per-step statistics and the dt accumulators (1e100 as the reference's start value)
    DevScalars init{};
    init.dt_bits = 0x54B249AD2594C37Dull;
    if ((e = cudaMemcpyAsync(&sc->dt_bits, &init.dt_bits, sizeof(init.dt_bits), cudaMemcpyHostToDevice, c->stream)))
        return e;
    c->inst.dt_init.assign(c->inst.n, init.dt_bits);
    if ((e = cudaMemcpyAsync(c->inst.d_dt.p, c->inst.dt_init.data(), c->inst.n * sizeof(unsigned long long),
                             cudaMemcpyHostToDevice, c->stream)))
        return e;
    if ((e = cudaMemsetAsync(&sc->overflow, 0, offsetof(DevScalars, dt) - offsetof(DevScalars, overflow),
                             c->stream)))
        return e;
    (void)fixed_dt;
    if (n > 0) {
        if (c->prm.dim == 2)
            k_prim_dt<2><<<nblk(n, HT), HT, 0, c->stream>>>((const double*)c->mass.p, (const double*)c->mom.p,
                                                            (const double*)c->en.p, (const double*)c->vol.p,
                                                            (const int*)c->status.p, (const int*)c->certk.p, n, cfl,
                                                            (const InstPar*)c->inst.d_par.p,
                                                            (const uint16_t*)c->inst.d_inst_h.p,
                                                            (unsigned long long*)c->inst.d_dt.p, w4, we, sc);
        else
            k_prim_dt<3><<<nblk(n, HT), HT, 0, c->stream>>>((const double*)c->mass.p, (const double*)c->mom.p,
                                                            (const double*)c->en.p, (const double*)c->vol.p,
                                                            (const int*)c->status.p, (const int*)c->certk.p, n, cfl,
                                                            (const InstPar*)c->inst.d_par.p,
                                                            (const uint16_t*)c->inst.d_inst_h.p,
                                                            (unsigned long long*)c->inst.d_dt.p, w4, we, sc);
        count_launches(1);
    }
    return cudaGetLastError();
}

// moving faces: gradients (second order), then fluxes + update + drift
static cudaError_t launch_ale(pgpu_ctx* c, double fixed_dt) {
    const int D = c->prm.dim;
    const int64_t n = c->n_hydro;
    const int order2 = c->prm.flux_mode == PGPU_FLUX_ALE2;
    const int NV = D + 2;
    cudaError_t e = cudaSuccess;
    double* wp = ensure<double>(c->ale_wp, (size_t)n * NV + 1, &e);
    double* gr = ensure<double>(c->ale_grad, (size_t)n * NV * D + 1, &e);
    if (e) return e;
    DevScalars* sc = (DevScalars*)c->scalars.p;
    const uint32_t* order = c->have_mesh && !c->all_cells && c->n_query == n ? (const uint32_t*)c->qs.p : nullptr;
    const InstPar* ip = (const InstPar*)c->inst.d_par.p;
    const uint16_t* inst = (const uint16_t*)c->inst.d_inst_h.p;
    const unsigned long long* dti = (const unsigned long long*)c->inst.d_dt.p;
    const double4* w4 = (const double4*)c->w4.p;
    const double* we = (const double*)c->we.p;
    const uint32_t* fptr = (const uint32_t*)c->fptr.p;
    const uint32_t* fcnt = (const uint32_t*)c->fcnt.p;
    const uint32_t* fown = (const uint32_t*)c->f_own.p;
    const int32_t* fnb = (const int32_t*)c->f_nb.p;
    const double4* fgeo = (const double4*)c->f_geo.p;
    const uint32_t* perm = (const uint32_t*)c->perm.p;
    int launches = 0;
    if (D == 2) {
        const double2* ext = (const double2*)c->ext.p;
        if (order2) {
            k_ale_grad<2><<<nblk(n, HT), HT, 0, c->stream>>>(w4, we, fptr, fcnt, fown, fnb, fgeo, ext, n, ip, inst,
                                                             dti, fixed_dt, wp, gr, order, perm);
            k_ale_flux<2, 2><<<nblk(n, HT), HT, 0, c->stream>>>(w4, we, fptr, fcnt, fown, fnb, fgeo, ext, n, ip, inst,
                                                                dti, fixed_dt, wp, gr, (double*)c->mass.p,
                                                                (double*)c->mom.p, (double*)c->en.p,
                                                                (double*)c->pos.p, sc, order, perm);
            launches = 2;
        } else {
            k_ale_flux<2, 1><<<nblk(n, HT), HT, 0, c->stream>>>(w4, we, fptr, fcnt, fown, fnb, fgeo, ext, n, ip, inst,
                                                                dti, fixed_dt, wp, gr, (double*)c->mass.p,
                                                                (double*)c->mom.p, (double*)c->en.p,
                                                                (double*)c->pos.p, sc, order, perm);
            launches = 1;
        }
    } else {
        const double4* ext = (const double4*)c->ext.p;
        if (order2) {
            k_ale_grad<3><<<nblk(n, HT), HT, 0, c->stream>>>(w4, we, fptr, fcnt, fown, fnb, fgeo, ext, n, ip, inst,
                                                             dti, fixed_dt, wp, gr, order, perm);
            k_ale_flux<3, 2><<<nblk(n, HT), HT, 0, c->stream>>>(w4, we, fptr, fcnt, fown, fnb, fgeo, ext, n, ip, inst,
                                                                dti, fixed_dt, wp, gr, (double*)c->mass.p,
                                                                (double*)c->mom.p, (double*)c->en.p,
                                                                (double*)c->pos.p, sc, order, perm);
            launches = 2;
        } else {
            k_ale_flux<3, 1><<<nblk(n, HT), HT, 0, c->stream>>>(w4, we, fptr, fcnt, fown, fnb, fgeo, ext, n, ip, inst,
                                                                dti, fixed_dt, wp, gr, (double*)c->mass.p,
                                                                (double*)c->mom.p, (double*)c->en.p,
                                                                (double*)c->pos.p, sc, order, perm);
            launches = 1;
        }
    }
    count_launches(launches);
    return cudaGetLastError();
}

cudaError_t launch_flux_update(pgpu_ctx* c, double fixed_dt) {
    const int D = c->prm.dim;
    const int64_t n = c->n_hydro;
    if (n <= 0) return cudaSuccess;
    if (c->prm.flux_mode == PGPU_FLUX_ALE1 || c->prm.flux_mode == PGPU_FLUX_ALE2) return launch_ale(c, fixed_dt);
    DevScalars* sc = (DevScalars*)c->scalars.p;
    const bool phys = c->prm.flux_mode == PGPU_FLUX_PHYSICAL;
    // the current mesh's query list covers exactly the hydro cells, in spatial order
    const uint32_t* order = c->have_mesh && !c->all_cells && c->n_query == n ? (const uint32_t*)c->qs.p : nullptr;
    // walls: 0 all periodic, 1 all reflective, 2 mixed across the instances of a batch
    int mir = c->inst.par[0].mirror;
    for (const auto& q : c->inst.par)
        if (q.mirror != c->inst.par[0].mirror) mir = 2;
#define PGPU_FLUX(DD, PH, MI)                                                                                     \
    k_flux_update<DD, PH, MI><<<nblk(n, FT), FT, 0, c->stream>>>(                                                \
        (const double4*)c->w4.p, (const double*)c->we.p, (const uint32_t*)c->fptr.p, (const uint32_t*)c->fcnt.p, \
        (const uint32_t*)c->f_own.p, (const double4*)c->f_geo.p, n, (const InstPar*)c->inst.d_par.p,              \
        (const uint16_t*)c->inst.d_inst_h.p, (const unsigned long long*)c->inst.d_dt.p, fixed_dt,                 \
        (double*)c->mass.p, (double*)c->mom.p, (double*)c->en.p, (double*)c->pos.p, sc, order,             \
        (const uint32_t*)c->perm.p)
#define PGPU_FLUX_M(DD, PH) \
    do {                    \
        if (mir == 0)       \
            PGPU_FLUX(DD, PH, 0); \
        else if (mir == 1)  \
            PGPU_FLUX(DD, PH, 1); \
        else                \
            PGPU_FLUX(DD, PH, 2); \
    } while (0)
    if (D == 2) {
        if (phys) PGPU_FLUX_M(2, true); else PGPU_FLUX_M(2, false);
    } else {
        if (phys) PGPU_FLUX_M(3, true); else PGPU_FLUX_M(3, false);
    }
#undef PGPU_FLUX_M
#undef PGPU_FLUX
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_sums(pgpu_ctx* c) {
    cudaError_t e = cudaSuccess;
    const int64_t n = c->n_hydro;
    const int64_t nb = (n + HT - 1) / HT;
    double* part = ensure<double>(c->red_tmp, 5 * (nb + 1), &e);
    if (e) return e;
    DevScalars* sc = (DevScalars*)c->scalars.p;
    if (n > 0) {
        if (c->prm.dim == 2)
            k_partial_sums<2><<<(unsigned)nb, HT, 0, c->stream>>>((const double*)c->mass.p, (const double*)c->mom.p,
                                                                  (const double*)c->en.p, n, part);
        else
            k_partial_sums<3><<<(unsigned)nb, HT, 0, c->stream>>>((const double*)c->mass.p, (const double*)c->mom.p,
                                                                  (const double*)c->en.p, n, part);
        k_final_sums<<<1, 32, 0, c->stream>>>(part, nb, sc->sums);
        count_launches(2);
    }
    return cudaGetLastError();
}

}  // namespace pgpu

// ---------------------------------------------------------------------------
// pgpu_dt_cfl_static: hydro::dt_CFL on the caller's device arrays, with no
// allocation.  Its scratch is a file-scope device array: one partial minimum
// per block of DT_STATIC_CELLS_PER_BLOCK cells, then the result.  Every slot is
// written before it is read in the same call, so nothing has to start at zero;
// two calls that overlap on one device share the array and race.
namespace pgpu {
namespace {

constexpr int DT_STATIC_CELLS_PER_THREAD = 4;
constexpr int64_t DT_STATIC_CELLS_PER_BLOCK = (int64_t)HT * DT_STATIC_CELLS_PER_THREAD;
constexpr int DT_STATIC_MAX_BLOCKS = (int)(PGPU_DT_STATIC_MAX_CELLS / DT_STATIC_CELLS_PER_BLOCK);
static_assert((int64_t)DT_STATIC_MAX_BLOCKS * DT_STATIC_CELLS_PER_BLOCK == PGPU_DT_STATIC_MAX_CELLS,
              "the cell limit is a whole number of blocks");

// 16384 partials + the result: 128 KiB + 8 bytes of the library's device image.
static __device__ __align__(256) double g_dt_scratch[DT_STATIC_MAX_BLOCKS + 1];

template <int D>
__global__ void k_dt_static_partial(const double* __restrict__ rho, const double* __restrict__ v,
                                    const double* __restrict__ E, const double* __restrict__ vol, int64_t n,
                                    double cfl, double gamma, double* __restrict__ partial) {
    const int64_t base = (int64_t)blockIdx.x * DT_STATIC_CELLS_PER_BLOCK + threadIdx.x;
    double d = 1e100;  // the reference's starting value of the minimum
#pragma unroll
    for (int j = 0; j < DT_STATIC_CELLS_PER_THREAD; j++) {
        const int64_t i = base + (int64_t)j * HT;
        if (i < n) d = fmin(d, dt_cell<D>(load_prim<D>(rho, v, E, i), vol[i], cfl, gamma));
    }
    d = block_min(d);
    if (threadIdx.x == 0) partial[blockIdx.x] = d;
}

__global__ void k_dt_static_final(const double* __restrict__ partial, int nb, double* __restrict__ out) {
    double d = 1e100;
    for (int b = threadIdx.x; b < nb; b += HT) d = fmin(d, partial[b]);
    d = block_min(d);
    if (threadIdx.x == 0) *out = d;
}

std::mutex g_dt_static_mu;
double* g_dt_static_ptr[PGPU_DT_STATIC_MAX_DEVICES];

}  // namespace
}  // namespace pgpu

extern "C" int pgpu_dt_cfl_static(int dim, double gamma, double cfl, const double* rho, const double* v,
                                  const double* E, const double* volumes, int64_t n, void* stream, double* dt) {
    using namespace pgpu;
    if ((dim != 2 && dim != 3) || !rho || !v || !E || !volumes || !dt || n <= 0) return PGPU_EINVAL;
    if (n > PGPU_DT_STATIC_MAX_CELLS) return PGPU_ECAPACITY;
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess) return PGPU_ECUDA;
    if (dev < 0 || dev >= PGPU_DT_STATIC_MAX_DEVICES) return PGPU_ECAPACITY;
    double* scratch;
    {
        std::lock_guard<std::mutex> lock(g_dt_static_mu);
        if (!g_dt_static_ptr[dev]) {
            void* p = nullptr;
            if (cudaGetSymbolAddress(&p, g_dt_scratch) != cudaSuccess || !p) return PGPU_ECUDA;
            g_dt_static_ptr[dev] = (double*)p;
        }
        scratch = g_dt_static_ptr[dev];
    }
    cudaStream_t s = (cudaStream_t)stream;
    const int nb = (int)((n + DT_STATIC_CELLS_PER_BLOCK - 1) / DT_STATIC_CELLS_PER_BLOCK);
    if (dim == 2)
        k_dt_static_partial<2><<<nb, HT, 0, s>>>(rho, v, E, volumes, n, cfl, gamma, scratch);
    else
        k_dt_static_partial<3><<<nb, HT, 0, s>>>(rho, v, E, volumes, n, cfl, gamma, scratch);
    k_dt_static_final<<<1, HT, 0, s>>>(scratch, nb, scratch + DT_STATIC_MAX_BLOCKS);
    count_launches(2);
    if (cudaGetLastError() != cudaSuccess) return PGPU_ECUDA;
    if (cudaMemcpyAsync(dt, scratch + DT_STATIC_MAX_BLOCKS, sizeof(double), cudaMemcpyDeviceToHost, s) !=
        cudaSuccess)
        return PGPU_ECUDA;
    if (cudaStreamSynchronize(s) != cudaSuccess) return PGPU_ECUDA;
    return PGPU_OK;
}
