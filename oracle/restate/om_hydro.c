#define _GNU_SOURCE
/*
 * CFL time step, HLL fluxes and updates (test-infrastructure oracle).
 *
 * om_dt_cfl and om_hydro_step_ref restate hydro::dt_CFL and hydro::hydro_step
 * (src/hydro/finite_volume_solver.cpp:43-186) with riemann_hll and its helpers
 * (src/hydro/riemann.cpp:7-124) in the same FP64 operation order.  Primitive
 * state: rho, v, E with E the total energy per unit volume.
 *
 * om_step_moving is an extension (the reference never moves its mesh): it
 * carries conserved mass, momentum and energy per cell across re-meshing, uses
 * the outward normal and face-pair-symmetric areas so that every face flux
 * cancels exactly between its two cells, and drifts each generating point with
 * its cell's velocity.
 */
#include "om.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
    double rho, v[3], E;
} prim_t;

typedef struct {
    double n[3], m[3], p[3];
} geom_t;

static inline double dmin(double a, double b) { return (b < a) ? b : a; } /* std::min */
static inline double dmax(double a, double b) { return (a < b) ? b : a; } /* std::max */

/* get_P_ideal_gas (riemann.cpp:118-124) */
static inline double pressure(const prim_t *s, int dim, double gamma) {
    if (dim == 2) return (gamma - 1) * (s->E - (0.5 * s->rho * (s->v[0] * s->v[0] + s->v[1] * s->v[1])));
    return (gamma - 1) * (s->E - (0.5 * s->rho * (s->v[0] * s->v[0] + s->v[1] * s->v[1] + s->v[2] * s->v[2])));
}

/* compute_geom (riemann.cpp:75-97) */
static geom_t make_geom(const double *normal) {
    geom_t g;
    double nn = sqrt(normal[0] * normal[0] + normal[1] * normal[1] + normal[2] * normal[2]);
    g.n[0] = normal[0] / nn;
    g.n[1] = normal[1] / nn;
    g.n[2] = normal[2] / nn;
    if (g.n[0] != 0.0 || g.n[1] != 0.0) {
        g.m[0] = -g.n[1];
        g.m[1] = g.n[0];
        g.m[2] = 0.0;
    } else {
        g.m[0] = 1.0;
        g.m[1] = 0.0;
        g.m[2] = 0.0;
    }
    double mm = sqrt(g.m[0] * g.m[0] + g.m[1] * g.m[1] + g.m[2] * g.m[2]);
    g.m[0] /= mm;
    g.m[1] /= mm;
    g.m[2] /= mm;
    g.p[0] = g.n[1] * g.m[2] - g.n[2] * g.m[1];
    g.p[1] = g.n[2] * g.m[0] - g.n[0] * g.m[2];
    g.p[2] = g.n[0] * g.m[1] - g.n[1] * g.m[0];
    return g;
}

/* rotate_to_face / rotate_from_face (riemann.cpp:47-73) */
static void to_face(prim_t *s, const geom_t *g, int dim) {
    double vx = s->v[0], vy = s->v[1];
    if (dim == 2) {
        s->v[0] = vx * g->n[0] + vy * g->n[1];
        s->v[1] = vx * g->m[0] + vy * g->m[1];
    } else {
        double vz = s->v[2];
        s->v[0] = vx * g->n[0] + vy * g->n[1] + vz * g->n[2];
        s->v[1] = vx * g->m[0] + vy * g->m[1] + vz * g->m[2];
        s->v[2] = vx * g->p[0] + vy * g->p[1] + vz * g->p[2];
    }
}

static void from_face(prim_t *s, const geom_t *g, int dim) {
    double vx = s->v[0], vy = s->v[1];
    if (dim == 2) {
        s->v[0] = vx * g->n[0] + vy * g->m[0];
        s->v[1] = vx * g->n[1] + vy * g->m[1];
    } else {
        double vz = s->v[2];
        s->v[0] = vx * g->n[0] + vy * g->m[0] + vz * g->p[0];
        s->v[1] = vx * g->n[1] + vy * g->m[1] + vz * g->p[1];
        s->v[2] = vx * g->n[2] + vy * g->m[2] + vz * g->p[2];
    }
}

/* get_flux (riemann.cpp:99-116) */
static prim_t phys_flux(const prim_t *s, int dim, double gamma) {
    double P = pressure(s, dim, gamma);
    prim_t f;
    memset(&f, 0, sizeof(f));
    f.rho = s->rho * s->v[0];
    f.v[0] = s->rho * s->v[0] * s->v[0] + P;
    f.v[1] = s->rho * s->v[0] * s->v[1];
    if (dim == 3) f.v[2] = s->rho * s->v[0] * s->v[2];
    f.E = (s->E + P) * s->v[0];
    return f;
}

/* riemann_hll (riemann.cpp:7-45) with the face normal passed in */
static prim_t hll(prim_t L, prim_t R, const double *normal, int dim, double gamma) {
    geom_t g = make_geom(normal);
    to_face(&L, &g, dim);
    to_face(&R, &g, dim);
    prim_t fl = phys_flux(&L, dim, gamma), fr = phys_flux(&R, dim, gamma);
    double SL = dmin(L.v[0] - sqrt((gamma * pressure(&L, dim, gamma)) / L.rho),
                     R.v[0] - sqrt((gamma * pressure(&R, dim, gamma)) / R.rho));
    double SR = dmax(L.v[0] + sqrt((gamma * pressure(&L, dim, gamma)) / L.rho),
                     R.v[0] + sqrt((gamma * pressure(&R, dim, gamma)) / R.rho));
    prim_t f;
    memset(&f, 0, sizeof(f));
    if (SL >= 0) {
        f = fl;
    } else if (SL < 0 && SR > 0) {
        f.rho = (SR * fl.rho - SL * fr.rho + SL * SR * (R.rho - L.rho)) / (SR - SL);
        f.v[0] = (SR * fl.v[0] - SL * fr.v[0] + SL * SR * (R.rho * R.v[0] - L.rho * L.v[0])) / (SR - SL);
        f.v[1] = (SR * fl.v[1] - SL * fr.v[1] + SL * SR * (R.rho * R.v[1] - L.rho * L.v[1])) / (SR - SL);
        if (dim == 3)
            f.v[2] = (SR * fl.v[2] - SL * fr.v[2] + SL * SR * (R.rho * R.v[2] - L.rho * L.v[2])) / (SR - SL);
        f.E = (SR * fl.E - SL * fr.E + SL * SR * (R.E - L.E)) / (SR - SL);
    } else if (SR <= 0) {
        f = fr;
    }
    from_face(&f, &g, dim);
    return f;
}

static prim_t load(const double *rho, const double *v, const double *E, long i, int dim) {
    prim_t s;
    memset(&s, 0, sizeof(s));
    s.rho = rho[i];
    s.E = E[i];
    for (int k = 0; k < dim; k++) s.v[k] = v[i * dim + k];
    return s;
}

double om_dt_cfl(const om_mesh *m, double cfl, double gamma, const double *rho, const double *v, const double *E) {
    const int dim = m->dim;
    double min_dt = 1e100;
    for (long i = 0; i < m->n_hydro; i++) {
        prim_t s = load(rho, v, E, i, dim);
        double P = pressure(&s, dim, gamma);
        double c = sqrt(gamma * P / s.rho);
        double R, va;
        if (dim == 2) {
            R = sqrt(m->volumes[i] / M_PI);
            va = sqrt(s.v[0] * s.v[0] + s.v[1] * s.v[1]);
        } else {
            R = cbrt(3.0 * m->volumes[i] / (4.0 * M_PI));
            va = sqrt(s.v[0] * s.v[0] + s.v[1] * s.v[1] + s.v[2] * s.v[2]);
        }
        double dt_i = cfl * (R / (c + va));
        if (dt_i < min_dt) min_dt = dt_i;
    }
    return min_dt;
}

/* hydro id owning extended id e */
static inline long owner_of(const om_mesh *m, long e) { return e < m->n_hydro ? e : m->ghost_ids[e - m->n_hydro]; }
static inline int code_of(const om_mesh *m, long e) { return e < m->n_hydro ? 0 : m->ghost_code[e - m->n_hydro]; }

long om_hydro_step_ref(const om_mesh *m, double dt, double gamma, double *rho, double *v, double *E) {
    const int dim = m->dim;
    const long nh = m->n_hydro;
    double *nr = (double *)malloc(nh * sizeof(double));
    double *nv = (double *)malloc(nh * dim * sizeof(double));
    double *nE = (double *)malloc(nh * sizeof(double));
    long box_faces = 0;
#pragma omp parallel for reduction(+ : box_faces)
    for (long i = 0; i < nh; i++) {
        prim_t si = load(rho, v, E, i, dim), tot;
        memset(&tot, 0, sizeof(tot));
        for (long j = 0; j < m->face_counts[i]; j++) {
            long f = m->face_ptr[i] + j;
            long e = m->neighbor[f];
            if (e < 0) {
                box_faces++;
                e = i;
            }
            prim_t sj = load(rho, v, E, owner_of(m, e), dim);
            prim_t fl = hll(si, sj, m->normal + 3 * f, dim, gamma);
            double A = m->area[f];
            tot.rho += fl.rho * A;
            tot.v[0] += fl.v[0] * A;
            tot.v[1] += fl.v[1] * A;
            if (dim == 3) tot.v[2] += fl.v[2] * A;
            tot.E += fl.E * A;
        }
        double V = m->volumes[i];
        double frac = dt / V;
        nr[i] = si.rho - frac * tot.rho;
        double inv = 1.0 / nr[i];
        for (int k = 0; k < dim; k++) nv[i * dim + k] = (si.rho * si.v[k] - frac * tot.v[k]) * inv;
        nE[i] = si.E - frac * tot.E;
    }
    memcpy(rho, nr, nh * sizeof(double));
    memcpy(v, nv, nh * dim * sizeof(double));
    memcpy(E, nE, nh * sizeof(double));
    free(nr);
    free(nv);
    free(nE);
    return box_faces;
}

/* Reverse image code: a periodic shift +1 <-> -1 swaps digits 1 and 2; a
 * mirror is its own inverse. */
static int reverse_code(int code, int dim, int periodic) {
    if (!periodic) return code;
    int out = 0, mul = 1;
    for (int a = 0; a < dim; a++) {
        int d = code % 3;
        code /= 3;
        out += (d == 0 ? 0 : 3 - d) * mul;
        mul *= 3;
    }
    return out;
}

static long symmetric_area_impl(const om_mesh *m, double *out, int periodic) {
    long unpaired = 0;
    const int dim = m->dim;
#pragma omp parallel for reduction(+ : unpaired)
    for (long i = 0; i < m->n_hydro; i++) {
        for (long j = 0; j < m->face_counts[i]; j++) {
            long f = m->face_ptr[i] + j;
            out[f] = m->area[f];
            long e = m->neighbor[f];
            if (e < 0) continue;
            long h = owner_of(m, e);
            if (h >= i) continue;
            int want = reverse_code(code_of(m, e), dim, periodic);
            int found = 0;
            for (long q = 0; q < m->face_counts[h]; q++) {
                long g = m->face_ptr[h] + q;
                long e2 = m->neighbor[g];
                if (e2 < 0) continue;
                if (owner_of(m, e2) == i && code_of(m, e2) == want) {
                    out[f] = m->area[g];
                    found = 1;
                    break;
                }
            }
            if (!found) unpaired++;
        }
    }
    return unpaired;
}

long om_symmetric_area(const om_mesh *m, double *out) { return symmetric_area_impl(m, out, 1); }

static long symmetric_area_mode(const om_mesh *m, double *out, int boundary) {
    return symmetric_area_impl(m, out, boundary == OM_PERIODIC);
}

double om_step_moving(const om_mesh *m, double cfl, double fixed_dt, double gamma, int boundary, double *x,
                      double *mass, double *mom, double *energy, long *n_unpaired) {
    const int dim = m->dim;
    const long nh = m->n_hydro;
    double *rho = (double *)malloc(nh * sizeof(double));
    double *v = (double *)malloc(nh * dim * sizeof(double));
    double *E = (double *)malloc(nh * sizeof(double));
    for (long i = 0; i < nh; i++) {
        double V = m->volumes[i];
        rho[i] = mass[i] / V;
        for (int k = 0; k < dim; k++) v[i * dim + k] = mom[i * dim + k] / mass[i];
        E[i] = energy[i] / V;
    }
    double dt = fixed_dt > 0 ? fixed_dt : om_dt_cfl(m, cfl, gamma, rho, v, E);
    double *As = (double *)malloc((m->num_faces + 1) * sizeof(double));
    long unp = symmetric_area_mode(m, As, boundary);
    if (n_unpaired) *n_unpaired = unp;
#pragma omp parallel for
    for (long i = 0; i < nh; i++) {
        prim_t si = load(rho, v, E, i, dim), tot;
        memset(&tot, 0, sizeof(tot));
        for (long j = 0; j < m->face_counts[i]; j++) {
            long f = m->face_ptr[i] + j;
            long e = m->neighbor[f];
            if (e < 0) e = i;
            prim_t sj = load(rho, v, E, owner_of(m, e), dim);
            if (boundary == OM_REFLECTIVE) {
                int code = code_of(m, e);
                for (int a = 0; a < dim; a++, code /= 3)
                    if (code % 3) sj.v[a] = -sj.v[a];
            }
            double nout[3] = {-m->normal[3 * f], -m->normal[3 * f + 1], -m->normal[3 * f + 2]};
            prim_t fl = hll(si, sj, nout, dim, gamma);
            double A = As[f];
            tot.rho += fl.rho * A;
            tot.v[0] += fl.v[0] * A;
            tot.v[1] += fl.v[1] * A;
            if (dim == 3) tot.v[2] += fl.v[2] * A;
            tot.E += fl.E * A;
        }
        mass[i] = mass[i] - dt * tot.rho;
        for (int k = 0; k < dim; k++) mom[i * dim + k] = mom[i * dim + k] - dt * tot.v[k];
        energy[i] = energy[i] - dt * tot.E;
        for (int k = 0; k < dim; k++) {
            double p = x[i * dim + k] + v[i * dim + k] * dt;
            if (boundary == OM_PERIODIC) {
                if (p < 0.0) p += 1.0;
                if (p >= 1.0) p -= 1.0;
            } else {
                if (p < 0.0) p = -p;
                if (p >= 1.0) p = 2.0 - p;
                if (p >= 1.0) p = 0x1.fffffffffffffp-1;
            }
            x[i * dim + k] = p;
        }
    }
    free(As);
    free(rho);
    free(v);
    free(E);
    return dt;
}

/* ---- second-order moving-mesh step (extension; see om.h) ---- */

#define MUSCL_NV 5 /* rho, vx, vy, vz, P (vz unused in 2D) */

typedef struct {
    double w[MUSCL_NV];
} wvec_t;

/* partner face g of face f (cell i, neighbour image of h < i) in h's face list, or -1 */
static long partner_face(const om_mesh *m, long i, long f) {
    long e = m->neighbor[f];
    long h = owner_of(m, e);
    int want = reverse_code(code_of(m, e), m->dim, 1);
    for (long q = 0; q < m->face_counts[h]; q++) {
        long g = m->face_ptr[h] + q;
        long e2 = m->neighbor[g];
        if (e2 < 0) continue;
        if (owner_of(m, e2) == i && code_of(m, e2) == want) return g;
    }
    return -1;
}

/* generator offset d (physical units) of face f of hydro cell i, seen from i */
static void face_offset(const om_mesh *m, long i, long f, double *d) {
    const int dim = m->dim;
    const long e = m->neighbor[f];
    for (int a = 0; a < 3; a++) d[a] = 0.0;
    for (int a = 0; a < dim; a++) d[a] = (m->ext[e * dim + a] - m->ext[i * dim + a]) * m->unit_scale;
}

/* solves the symmetric normal equations M g = b (dim 2 or 3) by cofactors */
static void solve_sym(int dim, const double *M, const double *b, double *g) {
    /* M: xx, xy, xz, yy, yz, zz */
    if (dim == 2) {
        double det = M[0] * M[3] - M[1] * M[1];
        g[0] = (M[3] * b[0] - M[1] * b[1]) / det;
        g[1] = (M[0] * b[1] - M[1] * b[0]) / det;
        g[2] = 0.0;
        return;
    }
    double c00 = M[3] * M[5] - M[4] * M[4];
    double c01 = M[2] * M[4] - M[1] * M[5];
    double c02 = M[1] * M[4] - M[2] * M[3];
    double c11 = M[0] * M[5] - M[2] * M[2];
    double c12 = M[1] * M[2] - M[0] * M[4];
    double c22 = M[0] * M[3] - M[1] * M[1];
    double det = M[0] * c00 + M[1] * c01 + M[2] * c02;
    g[0] = (c00 * b[0] + c01 * b[1] + c02 * b[2]) / det;
    g[1] = (c01 * b[0] + c11 * b[1] + c12 * b[2]) / det;
    g[2] = (c02 * b[0] + c12 * b[1] + c22 * b[2]) / det;
}

static inline double dot_d(const double *a, const double *b, int dim) {
    double s = a[0] * b[0] + a[1] * b[1];
    if (dim == 3) s = s + a[2] * b[2];
    return s;
}

double om_step_ale(const om_mesh *m, int order, double cfl, double fixed_dt, double gamma, double *x, double *mass,
                   double *mom, double *energy, long *n_unpaired) {
    if (!m->ext || !(m->unit_scale > 0.0) || (order != 1 && order != 2)) return -1.0;
    const int dim = m->dim;
    const long nh = m->n_hydro;
    const int nv = dim == 3 ? 5 : 4;       /* variables: rho, v (dim), P */
    const int ip = dim == 3 ? 4 : 3;       /* index of P */
    double *rho = (double *)malloc(nh * sizeof(double));
    double *v = (double *)malloc(nh * dim * sizeof(double));
    double *E = (double *)malloc(nh * sizeof(double));
    wvec_t *W = (wvec_t *)calloc(nh, sizeof(wvec_t));
    wvec_t *Wp = (wvec_t *)calloc(nh, sizeof(wvec_t));
    double *G = (double *)calloc((size_t)nh * MUSCL_NV * 3, sizeof(double)); /* gradients, var-major */
    for (long i = 0; i < nh; i++) {
        double V = m->volumes[i];
        rho[i] = mass[i] / V;
        for (int k = 0; k < dim; k++) v[i * dim + k] = mom[i * dim + k] / mass[i];
        E[i] = energy[i] / V;
        prim_t s = load(rho, v, E, i, dim);
        W[i].w[0] = s.rho;
        for (int k = 0; k < dim; k++) W[i].w[1 + k] = s.v[k];
        W[i].w[ip] = pressure(&s, dim, gamma);
    }
    double dt = fixed_dt > 0 ? fixed_dt : om_dt_cfl(m, cfl, gamma, rho, v, E);
    long unp = 0;
    /* gradients (least squares), limiter, half-step prediction; first order: none */
    if (order == 1) memcpy(Wp, W, nh * sizeof(wvec_t));
#pragma omp parallel for
    for (long i = 0; i < (order == 2 ? nh : 0); i++) {
        double M[6] = {0, 0, 0, 0, 0, 0}, b[MUSCL_NV][3], wmax[MUSCL_NV], wmin[MUSCL_NV];
        for (int k = 0; k < nv; k++) {
            b[k][0] = b[k][1] = b[k][2] = 0.0;
            wmax[k] = wmin[k] = W[i].w[k];
        }
        for (long j = 0; j < m->face_counts[i]; j++) {
            long f = m->face_ptr[i] + j;
            if (m->neighbor[f] < 0) continue;
            long h = owner_of(m, m->neighbor[f]);
            double d[3];
            face_offset(m, i, f, d);
            double wgt = m->area[f] / dot_d(d, d, dim);
            M[0] += wgt * d[0] * d[0];
            M[1] += wgt * d[0] * d[1];
            M[3] += wgt * d[1] * d[1];
            if (dim == 3) {
                M[2] += wgt * d[0] * d[2];
                M[4] += wgt * d[1] * d[2];
                M[5] += wgt * d[2] * d[2];
            }
            for (int k = 0; k < nv; k++) {
                double dw = W[h].w[k] - W[i].w[k];
                for (int a = 0; a < dim; a++) b[k][a] += wgt * dw * d[a];
                wmax[k] = dmax(wmax[k], W[h].w[k]);
                wmin[k] = dmin(wmin[k], W[h].w[k]);
            }
        }
        double *g = G + (size_t)i * MUSCL_NV * 3;
        for (int k = 0; k < nv; k++) solve_sym(dim, M, b[k], g + 3 * k);
        /* limiter */
        double alpha[MUSCL_NV];
        for (int k = 0; k < nv; k++) alpha[k] = 1.0;
        for (long j = 0; j < m->face_counts[i]; j++) {
            long f = m->face_ptr[i] + j;
            if (m->neighbor[f] < 0) continue;
            double d[3];
            face_offset(m, i, f, d);
            for (int k = 0; k < nv; k++) {
                double dw = dot_d(g + 3 * k, d, dim) * 0.5;
                double psi = 1.0;
                if (dw > 0.0)
                    psi = (wmax[k] - W[i].w[k]) / dw;
                else if (dw < 0.0)
                    psi = (wmin[k] - W[i].w[k]) / dw;
                alpha[k] = dmin(alpha[k], psi);
            }
        }
        for (int k = 0; k < nv; k++)
            for (int a = 0; a < 3; a++) g[3 * k + a] = alpha[k] * g[3 * k + a];
        /* half-step prediction in the frame moving with the cell */
        double div = g[3 * 1 + 0] + g[3 * 2 + 1];
        if (dim == 3) div = div + g[3 * 3 + 2];
        const double hdt = 0.5 * dt;
        const double r = W[i].w[0], P = W[i].w[ip];
        Wp[i].w[0] = r - hdt * (r * div);
        for (int a = 0; a < dim; a++) Wp[i].w[1 + a] = W[i].w[1 + a] - hdt * (g[3 * ip + a] / r);
        Wp[i].w[ip] = P - hdt * (gamma * P * div);
    }
    /* fluxes and update */
#pragma omp parallel for reduction(+ : unp)
    for (long i = 0; i < nh; i++) {
        prim_t tot;
        memset(&tot, 0, sizeof(tot));
        const double *gi = G + (size_t)i * MUSCL_NV * 3;
        for (long j = 0; j < m->face_counts[i]; j++) {
            long f = m->face_ptr[i] + j;
            long e = m->neighbor[f];
            if (e < 0) continue;
            long h = owner_of(m, e);
            double d[3], A = m->area[f];
            face_offset(m, i, f, d);
            if (h < i) {
                long g2 = partner_face(m, i, f);
                if (g2 >= 0) {
                    double dh[3];
                    face_offset(m, h, g2, dh);
                    for (int a = 0; a < 3; a++) d[a] = -dh[a];
                    A = m->area[g2];
                } else {
                    unp++;
                }
            }
            const double *gh = G + (size_t)h * MUSCL_NV * 3;
            wvec_t L = Wp[i], R = Wp[h];
            if (order == 2) {
                for (int k = 0; k < nv; k++) {
                    L.w[k] = Wp[i].w[k] + dot_d(gi + 3 * k, d, dim) * 0.5;
                    R.w[k] = Wp[h].w[k] - dot_d(gh + 3 * k, d, dim) * 0.5;
                }
                if (!(L.w[0] > 0.0 && L.w[ip] > 0.0 && R.w[0] > 0.0 && R.w[ip] > 0.0)) {
                    L = Wp[i];
                    R = Wp[h];
                }
            }
            double w[3] = {0, 0, 0};
            for (int a = 0; a < dim; a++) w[a] = (v[i * dim + a] + v[h * dim + a]) * 0.5;
            prim_t sl, sr;
            memset(&sl, 0, sizeof(sl));
            memset(&sr, 0, sizeof(sr));
            sl.rho = L.w[0];
            sr.rho = R.w[0];
            for (int a = 0; a < dim; a++) {
                sl.v[a] = L.w[1 + a] - w[a];
                sr.v[a] = R.w[1 + a] - w[a];
            }
            sl.E = L.w[ip] / (gamma - 1.0) + 0.5 * sl.rho * dot_d(sl.v, sl.v, dim);
            sr.E = R.w[ip] / (gamma - 1.0) + 0.5 * sr.rho * dot_d(sr.v, sr.v, dim);
            double nout[3] = {-m->normal[3 * f], -m->normal[3 * f + 1], -m->normal[3 * f + 2]};
            prim_t fl = hll(sl, sr, nout, dim, gamma);
            /* back to the lab frame */
            double wm = dot_d(w, fl.v, dim), ww = dot_d(w, w, dim);
            fl.E = fl.E + wm + 0.5 * ww * fl.rho;
            for (int a = 0; a < dim; a++) fl.v[a] = fl.v[a] + w[a] * fl.rho;
            tot.rho += fl.rho * A;
            tot.v[0] += fl.v[0] * A;
            tot.v[1] += fl.v[1] * A;
            if (dim == 3) tot.v[2] += fl.v[2] * A;
            tot.E += fl.E * A;
        }
        mass[i] = mass[i] - dt * tot.rho;
        for (int k = 0; k < dim; k++) mom[i * dim + k] = mom[i * dim + k] - dt * tot.v[k];
        energy[i] = energy[i] - dt * tot.E;
    }
    for (long i = 0; i < nh; i++)
        for (int k = 0; k < dim; k++) {
            double p = x[i * dim + k] + v[i * dim + k] * dt;
            if (p < 0.0) p += 1.0;
            if (p >= 1.0) p -= 1.0;
            x[i * dim + k] = p;
        }
    if (n_unpaired) *n_unpaired = unp;
    free(rho);
    free(v);
    free(E);
    free(W);
    free(Wp);
    free(G);
    return dt;
}
