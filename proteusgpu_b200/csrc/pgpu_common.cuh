// Shared device code of the sm_100a mesh-and-flux path.
//
// Everything in this file is compiled with -fmad=false (see build.py): the
// parity contract with the reference's CPU build is bit-identical predicates,
// vertex coordinates and fluxes, and the reference's x86-64 build executes
// plain multiplies and adds, never fused ones.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "pgpu_ctx.h"

namespace pgpu {

constexpr int MAX_P = 64;   // clipping planes per cell (reference _MAX_P_, Config.sh:37)
constexpr int MAX_T = 96;   // vertices per cell (reference _MAX_T_, Config.sh:38)
constexpr int MAX_K = 256;  // neighbour budget limit of this implementation
constexpr uint32_t NO_NEIGHBOR = 0xFFFFFFFFu;

enum Status : int {
    ST_TRIANGLE_OVERFLOW = 0,
    ST_VERTEX_OVERFLOW = 1,
    ST_INCONSISTENT_BOUNDARY = 2,
    ST_SECURITY_RADIUS_NOT_REACHED = 3,
    ST_SUCCESS = 4,
    ST_NEEDS_EXACT_PREDICATES = 5,
    ST_NOT_COMPUTED = 6
};

// Point storage: 2D points as double2 (16 B), 3D points as double4 (32 B,
// w unused) so that one point is one aligned vector load.
template <int D> struct PointOf;
template <> struct PointOf<2> { using type = double2; };
template <> struct PointOf<3> { using type = double4; };

__device__ __forceinline__ double pz(const double2&) { return 0.0; }
__device__ __forceinline__ double pz(const double4& p) { return p.z; }

template <int D>
__device__ __forceinline__ typename PointOf<D>::type make_pt(double x, double y, double z);
template <> __device__ __forceinline__ double2 make_pt<2>(double x, double y, double) { return make_double2(x, y); }
template <> __device__ __forceinline__ double4 make_pt<3>(double x, double y, double z) {
    return make_double4(x, y, z, 0.0);
}

// ---- the reference's determinant expansions (src/global/allvars.h:168-195).
// The association order is part of the parity contract.
__device__ __forceinline__ double det2(double a11, double a12, double a21, double a22) {
    return a11 * a22 - a12 * a21;
}
__device__ __forceinline__ double det3(double a11, double a12, double a13, double a21, double a22, double a23,
                                       double a31, double a32, double a33) {
    return a11 * det2(a22, a23, a32, a33) - a21 * det2(a12, a13, a32, a33) + a31 * det2(a12, a13, a22, a23);
}
__device__ __forceinline__ double det4(double a11, double a12, double a13, double a14, double a21, double a22,
                                       double a23, double a24, double a31, double a32, double a33, double a34,
                                       double a41, double a42, double a43, double a44) {
    double m12 = a21 * a12 - a11 * a22;
    double m13 = a31 * a12 - a11 * a32;
    double m14 = a41 * a12 - a11 * a42;
    double m23 = a31 * a22 - a21 * a32;
    double m24 = a41 * a22 - a21 * a42;
    double m34 = a41 * a32 - a31 * a42;
    double m123 = m23 * a13 - m13 * a23 + m12 * a33;
    double m124 = m24 * a13 - m14 * a23 + m12 * a43;
    double m134 = m34 * a13 - m14 * a33 + m13 * a43;
    double m234 = m34 * a23 - m24 * a33 + m23 * a43;
    return (m234 * a14 - m134 * a24 + m124 * a34 - m123 * a44);
}

// ---- Morton codes of grid bins (bit interleave) ----
__device__ __forceinline__ uint32_t spread2(uint32_t x) {  // 16 bits -> even bits
    x &= 0xFFFFu;
    x = (x | (x << 8)) & 0x00FF00FFu;
    x = (x | (x << 4)) & 0x0F0F0F0Fu;
    x = (x | (x << 2)) & 0x33333333u;
    x = (x | (x << 1)) & 0x55555555u;
    return x;
}
__device__ __forceinline__ uint32_t spread3(uint32_t x) {  // 10 bits -> every third bit
    x &= 0x3FFu;
    x = (x | (x << 16)) & 0x030000FFu;
    x = (x | (x << 8)) & 0x0300F00Fu;
    x = (x | (x << 4)) & 0x030C30C3u;
    x = (x | (x << 2)) & 0x09249249u;
    return x;
}
template <int D> __device__ __forceinline__ uint32_t morton(int i, int j, int k);
template <> __device__ __forceinline__ uint32_t morton<2>(int i, int j, int) {
    return spread2((uint32_t)i) | (spread2((uint32_t)j) << 1);
}
template <> __device__ __forceinline__ uint32_t morton<3>(int i, int j, int k) {
    return spread3((uint32_t)i) | (spread3((uint32_t)j) << 1) | (spread3((uint32_t)k) << 2);
}

__device__ __forceinline__ int bin_coord(double x, int G) {
    int i = (int)floor(x * (double)G);
    return i < 0 ? 0 : (i > G - 1 ? G - 1 : i);
}

// Sub-bins of dense coarse bins: a bin with more than SUB_SPLIT points gets the
// smallest level L (<= SUB_LMAX) with at most SUB_FILL points per sub-bin on
// average.  Coordinates at level L run over [0, G << L); a point's level-L
// coordinate is clamped into its own coarse bin so both levels agree.
constexpr int SUB_SPLIT = 16;
constexpr int SUB_FILL = 4;
constexpr int SUB_LMAX = 5;
// The grid as the search kernels see it: per instance, coarse Morton bins, dense
// ones split into Morton-ordered sub-bins.
struct SubGrid {
    const InstPar* ip;          // per instance: G, first slot
    const uint16_t* inst;       // instance of each extended id
    const uint8_t* lvl;         // refinement level per coarse bin
    const uint32_t* sub_off;    // first sub-bin slot per coarse bin
    const uint32_t* sub_start;  // first sorted point per sub-bin slot (one past the last: n)
};

__device__ __forceinline__ int sub_coord(double x, int G, int L) {
    const int b = bin_coord(x, G);
    const int i = (int)floor(x * (double)(G << L));
    const int lo = b << L, hi = lo + (1 << L) - 1;
    return i < lo ? lo : (i > hi ? hi : i);
}

// ---- hydro: the reference's HLL solver (src/hydro/riemann.cpp:7-124) ----
struct Prim {
    double rho, vx, vy, vz, E;
};
struct Flux {
    double rho, mx, my, mz, E;
};

__host__ __device__ __forceinline__ double dmin_ref(double a, double b) { return (b < a) ? b : a; }  // std::min
__host__ __device__ __forceinline__ double dmax_ref(double a, double b) { return (a < b) ? b : a; }  // std::max

template <int D>
__host__ __device__ __forceinline__ double pressure(const Prim& s, double gamma) {
    if (D == 2) return (gamma - 1) * (s.E - (0.5 * s.rho * (s.vx * s.vx + s.vy * s.vy)));
    return (gamma - 1) * (s.E - (0.5 * s.rho * (s.vx * s.vx + s.vy * s.vy + s.vz * s.vz)));
}

struct Frame {
    double nx, ny, nz, mx, my, mz, px, py, pz;
};

// compute_geom (riemann.cpp:75-97)
__host__ __device__ __forceinline__ Frame make_frame(double ax, double ay, double az) {
    Frame g;
    double nn = sqrt(ax * ax + ay * ay + az * az);
    g.nx = ax / nn;
    g.ny = ay / nn;
    g.nz = az / nn;
    double mx, my, mz;
    if (g.nx != 0.0 || g.ny != 0.0) {
        mx = -g.ny;
        my = g.nx;
        mz = 0.0;
    } else {
        mx = 1.0;
        my = 0.0;
        mz = 0.0;
    }
    double mm = sqrt(mx * mx + my * my + mz * mz);
    g.mx = mx / mm;
    g.my = my / mm;
    g.mz = mz / mm;
    g.px = g.ny * g.mz - g.nz * g.my;
    g.py = g.nz * g.mx - g.nx * g.mz;
    g.pz = g.nx * g.my - g.ny * g.mx;
    return g;
}

template <int D>
__host__ __device__ __forceinline__ void to_face(Prim& s, const Frame& g) {  // rotate_to_face
    double vx = s.vx, vy = s.vy;
    if (D == 2) {
        s.vx = vx * g.nx + vy * g.ny;
        s.vy = vx * g.mx + vy * g.my;
    } else {
        double vz = s.vz;
        s.vx = vx * g.nx + vy * g.ny + vz * g.nz;
        s.vy = vx * g.mx + vy * g.my + vz * g.mz;
        s.vz = vx * g.px + vy * g.py + vz * g.pz;
    }
}

template <int D>
__host__ __device__ __forceinline__ Flux phys_flux(const Prim& s, double gamma) {  // get_flux
    double P = pressure<D>(s, gamma);
    Flux f;
    f.rho = s.rho * s.vx;
    f.mx = s.rho * s.vx * s.vx + P;
    f.my = s.rho * s.vx * s.vy;
    f.mz = (D == 3) ? s.rho * s.vx * s.vz : 0.0;
    f.E = (s.E + P) * s.vx;
    return f;
}

// riemann_hll with the face normal (ax, ay, az); returns the lab-frame flux.
template <int D>
__host__ __device__ __forceinline__ Flux hll(Prim L, Prim R, double ax, double ay, double az, double gamma) {
    Frame g = make_frame(ax, ay, az);
    to_face<D>(L, g);
    to_face<D>(R, g);
    Flux fl = phys_flux<D>(L, gamma), fr = phys_flux<D>(R, gamma);
    double cl = sqrt((gamma * pressure<D>(L, gamma)) / L.rho);
    double cr = sqrt((gamma * pressure<D>(R, gamma)) / R.rho);
    double SL = dmin_ref(L.vx - cl, R.vx - cr);
    double SR = dmax_ref(L.vx + cl, R.vx + cr);
    Flux f = {0.0, 0.0, 0.0, 0.0, 0.0};
    if (SL >= 0) {
        f = fl;
    } else if (SL < 0 && SR > 0) {
        f.rho = (SR * fl.rho - SL * fr.rho + SL * SR * (R.rho - L.rho)) / (SR - SL);
        f.mx = (SR * fl.mx - SL * fr.mx + SL * SR * (R.rho * R.vx - L.rho * L.vx)) / (SR - SL);
        f.my = (SR * fl.my - SL * fr.my + SL * SR * (R.rho * R.vy - L.rho * L.vy)) / (SR - SL);
        if (D == 3) f.mz = (SR * fl.mz - SL * fr.mz + SL * SR * (R.rho * R.vz - L.rho * L.vz)) / (SR - SL);
        f.E = (SR * fl.E - SL * fr.E + SL * SR * (R.E - L.E)) / (SR - SL);
    } else if (SR <= 0) {
        f = fr;
    }
    // rotate_from_face
    double vx = f.mx, vy = f.my;
    if (D == 2) {
        f.mx = vx * g.nx + vy * g.mx;
        f.my = vx * g.ny + vy * g.my;
    } else {
        double vz = f.mz;
        f.mx = vx * g.nx + vy * g.mx + vz * g.px;
        f.my = vx * g.ny + vy * g.my + vz * g.py;
        f.mz = vx * g.nz + vy * g.mz + vz * g.pz;
    }
    return f;
}

// Face owner/code word: bits 0..26 owner hydro id, bits 27..31 image code
// (base-3 digits per axis: 0 none, 1 low wall, 2 high wall).  Box faces: ~0u.
constexpr uint32_t OWNER_BITS = 27;
constexpr uint32_t OWNER_MASK = (1u << OWNER_BITS) - 1u;
constexpr uint32_t BOX_FACE = 0xFFFFFFFFu;

__device__ __forceinline__ uint32_t pack_owner(uint32_t owner, uint32_t code) {
    return owner | (code << OWNER_BITS);
}

// Reverse image code: a periodic shift swaps digits 1 <-> 2; a mirror is its own inverse.
__device__ __forceinline__ uint32_t reverse_code(uint32_t code, int dim, bool periodic) {
    if (!periodic) return code;
    uint32_t out = 0, mul = 1;
    for (int a = 0; a < dim; a++) {
        uint32_t d = code % 3;
        code /= 3;
        out += (d == 0 ? 0 : 3 - d) * mul;
        mul *= 3;
    }
    return out;
}

// Order-preserving map of a non-negative double to uint64 (for atomicMin on dt).
__device__ __forceinline__ unsigned long long dbits(double x) { return (unsigned long long)__double_as_longlong(x); }

}  // namespace pgpu
