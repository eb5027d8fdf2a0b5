#define _GNU_SOURCE
/*
 * Voronoi cells by half-space clipping + extraction (test-infrastructure oracle).
 *
 * Restates the reference's ConvexCell (src/voronoi/cell.cpp:42-411), the cell
 * loop of cpu_compute_cell (src/voronoi/voronoi.cpp:115-155) and
 * extract_cell_to_vmesh (src/voronoi/cell.cpp:416-669), which follow Ray,
 * Sokolov, Lefebvre, Levy, "Meshless Voronoi on the GPU", ACM TOG 37(6), 2018.
 * A cell is kept in dual form: planes (a, b, c, d) with a.x + d >= 0 inside,
 * and vertices as triples (pairs in 2D) of plane indices.  The steps, the list
 * manipulation order and the FP64 operation sequence are those of the
 * reference so that vertex order, and therefore every area and volume, come out
 * bit-identical; every determinant is evaluated with the reference's
 * expansion.  Extension: per-cell certified K and centroid.
 */
#include "om.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define END_OF_LIST 255

/* Predicate mode (extension): 0 = the reference's (a near-zero determinant
 * fails the cell), 1 = robust (the vertex is kept, i.e. not cut, and a vertex
 * with w = 0 blocks the security-radius certificate). */
int om_predicate_mode = 0;
void om_set_predicate_mode(int m) { om_predicate_mode = m; }

extern long om_counters_g[4];

typedef struct {
    int dim;
    const double *pts;
    double seed[4];
    int nb_v, nb_t, nb_r;
    int first;
    int status;
    double hp[OM_MAX_P][4];
    int vid[OM_MAX_P];
    unsigned char tri[OM_MAX_T][3];
    unsigned char bnext[OM_MAX_P];
    long n_pred, n_newv;
} cell_t;

/* ---- the reference's determinant expansions (allvars.h:168-195) ---- */
static inline double det2(double a11, double a12, double a21, double a22) { return a11 * a22 - a12 * a21; }

static inline double det3(double a11, double a12, double a13, double a21, double a22, double a23, double a31,
                          double a32, double a33) {
    return a11 * det2(a22, a23, a32, a33) - a21 * det2(a12, a13, a32, a33) + a31 * det2(a12, a13, a22, a23);
}

static inline double det4(double a11, double a12, double a13, double a14, double a21, double a22, double a23,
                          double a24, double a31, double a32, double a33, double a34, double a41, double a42,
                          double a43, double a44) {
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

static inline double fmax3(double a, double b, double c) {
    double m = a > b ? a : b;
    return m > c ? m : c;
}

static void point4(const double *p, int dim, double *o) {
    o[0] = p[0];
    o[1] = p[1];
    o[2] = dim == 3 ? p[2] : 0.0;
    o[3] = 1.0;
}

/* ---- ConvexCell::ConvexCell (cell.cpp:42-104): the bounding box ---- */
static void cell_init(cell_t *c, int dim, const double *pts, long id) {
    const double eps = 1e-14;
    const double xmin = -eps, xmax = 1.0 + eps;
    c->dim = dim;
    c->pts = pts;
    c->first = END_OF_LIST;
    for (int i = 0; i < OM_MAX_P; i++) c->bnext[i] = END_OF_LIST, c->vid[i] = -1;
    c->status = OM_SUCCESS;
    point4(pts + dim * id, dim, c->seed);
    double box[6][4] = {{1.0, 0.0, 0.0, -xmin}, {-1.0, 0.0, 0.0, xmax}, {0.0, 1.0, 0.0, -xmin},
                        {0.0, -1.0, 0.0, xmax}, {0.0, 0.0, 1.0, -xmin}, {0.0, 0.0, -1.0, xmax}};
    for (int p = 0; p < 2 * dim; p++) memcpy(c->hp[p], box[p], sizeof(box[p]));
    if (dim == 2) {
        static const unsigned char t2[4][2] = {{2, 0}, {1, 2}, {3, 1}, {0, 3}};
        for (int t = 0; t < 4; t++) c->tri[t][0] = t2[t][0], c->tri[t][1] = t2[t][1], c->tri[t][2] = 0;
        c->nb_v = 4;
        c->nb_t = 4;
    } else {
        static const unsigned char t3[8][3] = {{2, 5, 0}, {5, 3, 0}, {1, 5, 2}, {5, 1, 3},
                                               {4, 2, 0}, {4, 0, 3}, {2, 4, 1}, {4, 3, 1}};
        for (int t = 0; t < 8; t++) memcpy(c->tri[t], t3[t], 3);
        c->nb_v = 6;
        c->nb_t = 8;
    }
    c->nb_r = 0;
}

/* ConvexCell::compute_vertex_point with the perspective divide (cell.cpp:388-411) */
static void vertex_point(const cell_t *c, const unsigned char *v, double *o) {
    const double *p1 = c->hp[v[0]], *p2 = c->hp[v[1]];
    if (c->dim == 2) {
        double x = -det2(p1[3], p1[1], p2[3], p2[1]);
        double y = -det2(p1[0], p1[3], p2[0], p2[3]);
        double w = det2(p1[0], p1[1], p2[0], p2[1]);
        o[0] = x / w;
        o[1] = y / w;
        o[2] = 0;
        o[3] = 1;
        return;
    }
    const double *p3 = c->hp[v[2]];
    double x = -det3(p1[3], p1[1], p1[2], p2[3], p2[1], p2[2], p3[3], p3[1], p3[2]);
    double y = -det3(p1[0], p1[3], p1[2], p2[0], p2[3], p2[2], p3[0], p3[3], p3[2]);
    double z = -det3(p1[0], p1[1], p1[3], p2[0], p2[1], p2[3], p3[0], p3[1], p3[3]);
    double w = det3(p1[0], p1[1], p1[2], p2[0], p2[1], p2[2], p3[0], p3[1], p3[2]);
    o[0] = x / w;
    o[1] = y / w;
    o[2] = z / w;
    o[3] = 1;
}

static inline double dot3(const double *a, const double *b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

/* is_security_radius_reached (cell.cpp:369-384) */
static int security_reached(const cell_t *c, const double *nb) {
    double v_dist = 0;
    for (int i = 0; i < c->nb_t; i++) {
        double pc[4], d[4];
        vertex_point(c, c->tri[i], pc);
        for (int k = 0; k < 4; k++) d[k] = pc[k] - c->seed[k];
        double d2 = dot3(d, d);
        if (om_predicate_mode == 1) {
            /* robust mode: a vertex without a position (w = 0) blocks the certificate */
            v_dist = (d2 != d2 || v_dist != v_dist) ? d2 + v_dist : (d2 > v_dist ? d2 : v_dist);
        } else {
            v_dist = (d2 < v_dist) ? v_dist : d2; /* std::max(d2, v_dist) */
        }
    }
    double d[4];
    for (int k = 0; k < 4; k++) d[k] = nb[k] - c->seed[k];
    return dot3(d, d) > 4 * v_dist;
}

/* vert_is_in_conflict (cell.cpp:175-221) */
static int in_conflict(cell_t *c, const unsigned char *v, const double *e) {
    const double *p1 = c->hp[v[0]], *p2 = c->hp[v[1]];
    double det, eps;
    if (c->dim == 2) {
        det = det3(p1[0], p2[0], e[0], p1[1], p2[1], e[1], p1[3], p2[3], e[3]);
        double maxx = fmax3(fabs(p1[0]), fabs(p2[0]), fabs(e[0]));
        double maxy = fmax3(fabs(p1[1]), fabs(p2[1]), fabs(e[1]));
        double maxw = fmax3(fabs(p1[3]), fabs(p2[3]), fabs(e[3]));
        double max_max = fmax3(maxx, maxy, maxw);
        eps = 1e-14 * maxx * maxy * maxw;
        eps *= max_max;
    } else {
        const double *p3 = c->hp[v[2]];
        det = det4(p1[0], p2[0], p3[0], e[0], p1[1], p2[1], p3[1], e[1], p1[2], p2[2], p3[2], e[2], p1[3], p2[3],
                   p3[3], e[3]);
        double maxx = fmax3(fmax3(fabs(p1[0]), fabs(p2[0]), fabs(p3[0])), fabs(e[0]), 0.0);
        double maxy = fmax3(fmax3(fabs(p1[1]), fabs(p2[1]), fabs(p3[1])), fabs(e[1]), 0.0);
        double maxz = fmax3(fmax3(fabs(p1[2]), fabs(p2[2]), fabs(p3[2])), fabs(e[2]), 0.0);
        eps = 1e-14 * maxx * maxy * maxz;
        double max_max = fmax3(maxx, maxy, maxz);
        eps *= (max_max * max_max);
    }
    if (fabs(det) < eps) {
        if (om_predicate_mode == 1) return 0;
        c->status = OM_NEEDS_EXACT_PREDICATES;
    }
    return det > 0.0;
}

/* compute_boundary, 2D branch (cell.cpp:226-264) */
static void boundary_2d(cell_t *c) {
    for (int i = 0; i < OM_MAX_P; i++) c->bnext[i] = END_OF_LIST;
    c->first = END_OF_LIST;
    int count[OM_MAX_P] = {0};
    for (int r = 0; r < c->nb_r; r++) {
        count[c->tri[c->nb_t + r][0]]++;
        count[c->tri[c->nb_t + r][1]]++;
    }
    int lines[2], nb = 0;
    for (int p = 0; p < c->nb_v; p++)
        if (count[p] == 1 && nb < 2) lines[nb++] = p;
    if (nb != 2) {
        c->status = OM_INCONSISTENT_BOUNDARY;
        return;
    }
    c->first = lines[0];
    c->bnext[lines[0]] = (unsigned char)lines[1];
    c->bnext[lines[1]] = (unsigned char)lines[0];
}

/* compute_boundary, 3D branch (cell.cpp:266-341): grows the cavity boundary
 * cycle one removed vertex at a time, deferring vertices whose addition would
 * make the boundary non-simple. */
static void boundary_3d(cell_t *c) {
    for (int i = 0; i < OM_MAX_P; i++) c->bnext[i] = END_OF_LIST;
    c->first = END_OF_LIST;
    int nb_iter = 0;
    int t = c->nb_t;
    while (c->nb_r > 0) {
        if (nb_iter++ > 100) {
            c->status = OM_INCONSISTENT_BOUNDARY;
            return;
        }
        unsigned char *T = c->tri[t];
        int in_border[3], opp[3];
        for (int e = 0; e < 3; e++) in_border[e] = c->bnext[T[e]] != END_OF_LIST;
        for (int e = 0; e < 3; e++) opp[e] = c->bnext[T[(e + 1) % 3]] == T[e];
        int simple = 1;
        for (int e = 0; e < 3; e++)
            if (!opp[e] && !opp[(e + 1) % 3] && in_border[(e + 1) % 3]) simple = 0;
        if (!opp[0] && !opp[1] && !opp[2]) {
            if (c->first == END_OF_LIST) {
                for (int e = 0; e < 3; e++) c->bnext[T[e]] = T[(e + 1) % 3];
                c->first = T[0];
            } else {
                simple = 0;
            }
        }
        if (!simple) {
            t++;
            if (t == c->nb_t + c->nb_r) t = c->nb_t;
            continue;
        }
        for (int e = 0; e < 3; e++)
            if (!opp[e]) c->bnext[T[e]] = T[(e + 1) % 3];
        for (int e = 0; e < 3; e++) {
            if (opp[e] && opp[(e + 1) % 3]) {
                if (c->first == T[(e + 1) % 3]) c->first = c->bnext[T[(e + 1) % 3]];
                c->bnext[T[(e + 1) % 3]] = END_OF_LIST;
            }
        }
        unsigned char tmp[3];
        memcpy(tmp, c->tri[t], 3);
        memcpy(c->tri[t], c->tri[c->nb_t + c->nb_r - 1], 3);
        memcpy(c->tri[c->nb_t + c->nb_r - 1], tmp, 3);
        t = c->nb_t;
        c->nb_r--;
    }
}

/* Alternative cavity boundary used to cross-check the CUDA kernel's method
 * (not the reference's): the boundary is the set of directed edges x -> y of
 * removed vertices whose reverse edge belongs to no removed vertex; it must form
 * one cycle.  Selected by om_set_boundary_mode(1). */
int om_boundary_mode = 0;
void om_set_boundary_mode(int m) { om_boundary_mode = m; }

static void boundary_3d_set(cell_t *c) {
    unsigned long long em[OM_MAX_P];
    memset(em, 0, sizeof(em));
    for (int i = 0; i < OM_MAX_P; i++) c->bnext[i] = END_OF_LIST;
    c->first = END_OF_LIST;
    for (int r = 0; r < c->nb_r; r++) {
        unsigned char *T = c->tri[c->nb_t + r];
        for (int e = 0; e < 3; e++) em[T[e]] |= 1ull << T[(e + 1) % 3];
    }
    unsigned long long src = 0;
    int n = 0;
    for (int r = 0; r < c->nb_r; r++) {
        unsigned char *T = c->tri[c->nb_t + r];
        for (int e = 0; e < 3; e++) {
            int x = T[e], y = T[(e + 1) % 3];
            if (!((em[y] >> x) & 1ull)) {
                if ((src >> x) & 1ull) { c->status = OM_INCONSISTENT_BOUNDARY; return; }
                src |= 1ull << x;
                c->bnext[x] = (unsigned char)y;
                n++;
            }
        }
    }
    if (n < 3) { c->status = OM_INCONSISTENT_BOUNDARY; return; }
    int x0 = __builtin_ctzll(src), x = x0;
    for (int st = 1; st <= n; st++) {
        x = c->bnext[x];
        if (!((src >> x) & 1ull) || (x == x0 && st < n)) { c->status = OM_INCONSISTENT_BOUNDARY; return; }
    }
    if (x != x0) { c->status = OM_INCONSISTENT_BOUNDARY; return; }
    c->first = x0;
    c->nb_t += 0;
    c->nb_r = 0;
}

/* new_vertex (cell.cpp:346-364) */
static void new_vertex(cell_t *c, int i, int j, int k) {
    if (c->nb_t + 1 >= OM_MAX_T) {
        c->status = OM_TRIANGLE_OVERFLOW;
        return;
    }
    if (c->dim == 2) {
        double rw = det2(c->hp[i][0], c->hp[i][1], c->hp[j][0], c->hp[j][1]);
        if (rw > 0) {
            c->tri[c->nb_t][0] = (unsigned char)j;
            c->tri[c->nb_t][1] = (unsigned char)i;
        } else {
            c->tri[c->nb_t][0] = (unsigned char)i;
            c->tri[c->nb_t][1] = (unsigned char)j;
        }
        c->tri[c->nb_t][2] = 0;
    } else {
        c->tri[c->nb_t][0] = (unsigned char)i;
        c->tri[c->nb_t][1] = (unsigned char)j;
        c->tri[c->nb_t][2] = (unsigned char)k;
    }
    c->nb_t++;
    c->n_newv++;
}

/* clip_by_plane + new_halfplane (cell.cpp:110-172) */
static void clip(cell_t *c, long vid) {
    if (c->nb_v >= OM_MAX_P) {
        c->status = OM_VERTEX_OVERFLOW;
        return;
    }
    double B[4], dir[4], ave2[4];
    point4(c->pts + c->dim * vid, c->dim, B);
    for (int k = 0; k < 4; k++) dir[k] = c->seed[k] - B[k], ave2[k] = c->seed[k] + B[k];
    double dot = dot3(ave2, dir);
    int cur = c->nb_v;
    c->hp[cur][0] = dir[0];
    c->hp[cur][1] = dir[1];
    c->hp[cur][2] = dir[2];
    c->hp[cur][3] = -dot / 2.0;
    c->vid[cur] = (int)vid;
    c->nb_v++;

    const double *eqn = c->hp[cur];
    c->n_pred += c->nb_t;
    c->nb_r = 0;
    int i = 0;
    while (i < c->nb_t) {
        if (in_conflict(c, c->tri[i], eqn)) {
            c->nb_t--;
            unsigned char tmp[3];
            memcpy(tmp, c->tri[i], 3);
            memcpy(c->tri[i], c->tri[c->nb_t], 3);
            memcpy(c->tri[c->nb_t], tmp, 3);
            c->nb_r++;
        } else {
            i++;
        }
    }
    if (c->status == OM_NEEDS_EXACT_PREDICATES) return;
    if (c->nb_r == 0) {
        c->nb_v--;
        return;
    }
    if (c->dim == 2)
        boundary_2d(c);
    else if (om_boundary_mode == 1)
        boundary_3d_set(c);
    else
        boundary_3d(c);
    if (c->status != OM_SUCCESS) return;
    if (c->first == END_OF_LIST) return;
    int cir = c->first;
    do {
        new_vertex(c, cur, cir, c->dim == 3 ? c->bnext[cir] : 0);
        if (c->status != OM_SUCCESS) return;
        cir = c->bnext[cir];
    } while (cir != c->first);
}

/* ---- extraction (cell.cpp:416-669) ---- */

typedef struct {
    int nf;
    int neighbor[OM_MAX_P];
    double normal[OM_MAX_P][3];
    double area[OM_MAX_P];
    double volume;
    double centroid[3];
} cell_out_t;

static inline int refs_plane(const cell_t *c, int t, int p) {
    for (int d = 0; d < c->dim; d++)
        if (c->tri[t][d] == p) return 1;
    return 0;
}

static double g_sort_cx, g_sort_cy; /* used by the 2D angular sort below */
typedef struct {
    double ang;
    int idx;
} angle_key;
static int cmp_angle(const void *a, const void *b) {
    double x = ((const angle_key *)a)->ang, y = ((const angle_key *)b)->ang;
    return (x < y) ? -1 : (x > y ? 1 : 0);
}

/* compute_cell_area_2d (cell.cpp:475-498) plus the polygon centroid (extension) */
static double area_2d(const double (*v)[4], int n, double *cen) {
    double cx = 0, cy = 0;
    for (int i = 0; i < n; i++) cx += v[i][0], cy += v[i][1];
    cx /= n;
    cy /= n;
    angle_key keys[OM_MAX_T];
    for (int i = 0; i < n; i++) keys[i].ang = atan2(v[i][1] - cy, v[i][0] - cx), keys[i].idx = i;
    qsort(keys, n, sizeof(angle_key), cmp_angle);
    double a = 0, sx = 0, sy = 0;
    for (int i = 0; i < n; i++) {
        int j = (i + 1) % n;
        const double *p = v[keys[i].idx], *q = v[keys[j].idx];
        a += p[0] * q[1];
        a -= q[0] * p[1];
        double cr = (p[0] - cx) * (q[1] - cy) - (q[0] - cx) * (p[1] - cy);
        sx += (p[0] + q[0] - 2 * cx) * cr;
        sy += (p[1] + q[1] - 2 * cy) * cr;
    }
    double sa = 0;
    for (int i = 0; i < n; i++) {
        int j = (i + 1) % n;
        const double *p = v[keys[i].idx], *q = v[keys[j].idx];
        sa += (p[0] - cx) * (q[1] - cy) - (q[0] - cx) * (p[1] - cy);
    }
    cen[0] = cx + sx / (3.0 * sa);
    cen[1] = cy + sy / (3.0 * sa);
    cen[2] = 0;
    (void)g_sort_cx;
    (void)g_sort_cy;
    return fabs(a) / 2.0;
}

static void extract(const cell_t *c, cell_out_t *o) {
    const int dim = c->dim;
    double vert[OM_MAX_T][4];
    for (int i = 0; i < c->nb_t; i++) vertex_point(c, c->tri[i], vert[i]);
    double cell_volume = 0.0;
    double vc[3] = {0, 0, 0}; /* volume-weighted centroid offset (3D extension) */
    if (dim == 2) o->volume = area_2d((const double (*)[4])vert, c->nb_t, o->centroid);
    o->nf = 0;
    for (int p = 0; p < c->nb_v; p++) {
        int idx[OM_MAX_T] = {0}, cnt = 0;
        for (int i = 0; i < c->nb_t; i++)
            if (refs_plane(c, i, p)) idx[cnt++] = i;
        if (cnt < dim) continue;
        double fv[OM_MAX_T][4];
        int nfv = 0;
        if (dim == 2) {
            for (int k = 0; k < cnt; k++) memcpy(fv[nfv++], vert[idx[k]], sizeof(fv[0]));
        } else {
            /* collect_face_vertices: order by adjacency (cell.cpp:530-563) */
            int ordered[OM_MAX_T], no = 0, used[OM_MAX_T] = {0};
            ordered[no++] = idx[0];
            used[0] = 1;
            for (int step = 1; step < cnt; step++) {
                int last = ordered[no - 1];
                int others[2], oc = 0;
                for (int d = 0; d < 3; d++)
                    if (c->tri[last][d] != p) others[oc++] = c->tri[last][d];
                int found = 0;
                for (int j = 0; j < cnt && !found; j++) {
                    if (used[j]) continue;
                    for (int q = 0; q < 2; q++) {
                        if (refs_plane(c, idx[j], others[q])) {
                            ordered[no++] = idx[j];
                            used[j] = 1;
                            found = 1;
                            break;
                        }
                    }
                }
                if (!found) break;
            }
            if (no < dim) continue;
            for (int k = 0; k < no; k++) memcpy(fv[nfv++], vert[ordered[k]], sizeof(fv[0]));
        }
        /* compute_face_normal (cell.cpp:575-579) */
        const double *pe = c->hp[p];
        double nlen = sqrt(dot3(pe, pe));
        double measure = 0.0;
        if (dim == 2) {
            double dx = fv[1][0] - fv[0][0];
            double dy = fv[1][1] - fv[0][1];
            measure = sqrt(dx * dx + dy * dy);
        } else {
            /* compute_face_measure (cell.cpp:591-627) */
            double e1[4], e2[4], cr[3], cen[4] = {0, 0, 0, 0}, out[4];
            for (int k = 0; k < 4; k++) e1[k] = fv[1][k] - fv[0][k], e2[k] = fv[2][k] - fv[0][k];
            cr[0] = e1[1] * e2[2] - e1[2] * e2[1];
            cr[1] = e1[2] * e2[0] - e1[0] * e2[2];
            cr[2] = e1[0] * e2[1] - e1[1] * e2[0];
            for (int k = 0; k < nfv; k++) cen[0] += fv[k][0], cen[1] += fv[k][1], cen[2] += fv[k][2];
            cen[0] /= (double)nfv;
            cen[1] /= (double)nfv;
            cen[2] /= (double)nfv;
            for (int k = 0; k < 4; k++) out[k] = cen[k] - c->seed[k];
            if (dot3(cr, out) < 0) {
                for (int a = 0, b = nfv - 1; a < b; a++, b--) {
                    double t[4];
                    memcpy(t, fv[a], sizeof(t));
                    memcpy(fv[a], fv[b], sizeof(t));
                    memcpy(fv[b], t, sizeof(t));
                }
            }
            for (int i = 1; i + 1 < nfv; i++) {
                double a1[3], a2[3], x[3];
                for (int k = 0; k < 3; k++) a1[k] = fv[i][k] - fv[0][k], a2[k] = fv[i + 1][k] - fv[0][k];
                x[0] = a1[1] * a2[2] - a1[2] * a2[1];
                x[1] = a1[2] * a2[0] - a1[0] * a2[2];
                x[2] = a1[0] * a2[1] - a1[1] * a2[0];
                measure += 0.5 * sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
            }
            for (int i = 1; i + 1 < nfv; i++) {
                double a[3], b[3], cc[3], bxc[3];
                for (int k = 0; k < 3; k++)
                    a[k] = fv[0][k] - c->seed[k], b[k] = fv[i][k] - c->seed[k], cc[k] = fv[i + 1][k] - c->seed[k];
                bxc[0] = b[1] * cc[2] - b[2] * cc[1];
                bxc[1] = b[2] * cc[0] - b[0] * cc[2];
                bxc[2] = b[0] * cc[1] - b[1] * cc[0];
                double tv = dot3(a, bxc) / 6.0;
                cell_volume += tv;
                for (int k = 0; k < 3; k++) vc[k] += tv * (a[k] + b[k] + cc[k]) * 0.25;
            }
        }
        int f = o->nf++;
        o->neighbor[f] = c->vid[p];
        o->normal[f][0] = pe[0] / nlen;
        o->normal[f][1] = pe[1] / nlen;
        o->normal[f][2] = pe[2] / nlen;
        o->area[f] = measure;
    }
    if (dim == 3) {
        o->volume = fabs(cell_volume);
        for (int k = 0; k < 3; k++) o->centroid[k] = c->seed[k] + vc[k] / cell_volume;
    }
}

/* ---- cell loop (voronoi.cpp:115-155) ---- */
/* row: the cell's K neighbour ids (knn + K * i in a full list) */
static void one_cell(int dim, const double *ext, long i, const uint32_t *row, int K, cell_out_t *o, int *status,
                     int *cert_k) {
    cell_t c;
    cell_init(&c, dim, ext, i);
    c.n_pred = c.n_newv = 0;
    *cert_k = 0;
    for (int v = 0; v < K; v++) {
        uint32_t z = row[v];
        if (z == UINT32_MAX) break;
        clip(&c, z);
        double nb[4];
        point4(ext + dim * (long)z, dim, nb);
        if (security_reached(&c, nb)) {
            *cert_k = v + 1;
            break;
        }
        if (c.status != OM_SUCCESS) break;
    }
    uint32_t last = row[K - 1];
    if (last == UINT32_MAX) {
        c.status = OM_SECURITY_RADIUS_NOT_REACHED;
    } else {
        double nb[4];
        point4(ext + dim * (long)last, dim, nb);
        if (!security_reached(&c, nb)) c.status = OM_SECURITY_RADIUS_NOT_REACHED;
    }
    *status = c.status;
#pragma omp atomic
    om_counters_g[1] += c.n_pred;
#pragma omp atomic
    om_counters_g[2] += c.n_newv;
#pragma omp atomic
    om_counters_g[3] += 1;
    o->nf = 0;
    o->volume = 0;
    o->centroid[0] = o->centroid[1] = o->centroid[2] = 0;
    if (c.status == OM_SUCCESS) extract(&c, o);
}

int om_cells(int dim, const double *ext, long n_ext, long n_hydro, const uint32_t *knn, int K, long n_compute,
             om_mesh *m) {
    memset(m, 0, sizeof(*m));
    m->dim = dim;
    m->n_seeds = n_ext;
    m->n_hydro = n_hydro;
    m->seeds = (double *)calloc(n_ext * 3, sizeof(double));
    m->volumes = (double *)calloc(n_ext, sizeof(double));
    m->face_counts = (long *)calloc(n_ext, sizeof(long));
    m->face_ptr = (long *)calloc(n_ext, sizeof(long));
    m->status = (int *)calloc(n_ext, sizeof(int));
    m->cert_k = (int *)calloc(n_ext, sizeof(int));
    m->centroid = (double *)calloc(n_ext * 3, sizeof(double));
    long cap = n_ext * (dim == 2 ? 8 : 18) + 64, F = 0;
    m->neighbor = (int *)malloc(cap * sizeof(int));
    m->normal = (double *)malloc(cap * 3 * sizeof(double));
    m->area = (double *)malloc(cap * sizeof(double));

    const long CH = 8192;
    cell_out_t *outs = (cell_out_t *)malloc(CH * sizeof(cell_out_t));
    for (long c0 = 0; c0 < n_ext; c0 += CH) {
        long c1 = c0 + CH < n_ext ? c0 + CH : n_ext;
#pragma omp parallel for schedule(dynamic, 64)
        for (long i = c0; i < c1; i++) {
            cell_out_t *o = &outs[i - c0];
            if (i >= n_compute) {
                m->status[i] = OM_NOT_COMPUTED;
                o->nf = 0;
                o->volume = 0;
                continue;
            }
            one_cell(dim, ext, i, knn + (long)K * i, K, o, &m->status[i], &m->cert_k[i]);
            /* extract_cell_to_vmesh writes the seed only for extracted cells
               (cell.cpp:418-420); the others keep calloc's zeros */
            if (m->status[i] == OM_SUCCESS) {
                m->seeds[3 * i] = ext[dim * i];
                m->seeds[3 * i + 1] = ext[dim * i + 1];
                m->seeds[3 * i + 2] = dim == 3 ? ext[dim * i + 2] : 0.0;
            }
        }
        for (long i = c0; i < c1; i++) {
            const cell_out_t *o = &outs[i - c0];
            if (F + o->nf > cap) {
                cap = 2 * cap + o->nf;
                m->neighbor = (int *)realloc(m->neighbor, cap * sizeof(int));
                m->normal = (double *)realloc(m->normal, cap * 3 * sizeof(double));
                m->area = (double *)realloc(m->area, cap * sizeof(double));
            }
            m->face_ptr[i] = F;
            m->face_counts[i] = o->nf;
            m->volumes[i] = o->volume;
            if (i < n_compute && m->status[i] == OM_SUCCESS)
                for (int k = 0; k < 3; k++) m->centroid[3 * i + k] = o->centroid[k];
            for (int f = 0; f < o->nf; f++, F++) {
                m->neighbor[F] = o->neighbor[f];
                for (int k = 0; k < 3; k++) m->normal[3 * F + k] = o->normal[f][k];
                m->area[F] = o->area[f];
            }
        }
    }
    free(outs);
    m->num_faces = F;
    return 0;
}

void om_mesh_free(om_mesh *m) {
    free(m->seeds);
    free(m->volumes);
    free(m->face_counts);
    free(m->face_ptr);
    free(m->neighbor);
    free(m->normal);
    free(m->area);
    free(m->ghost_ids);
    free(m->ghost_code);
    free(m->status);
    free(m->cert_k);
    free(m->centroid);
    free(m->ext);
    memset(m, 0, sizeof(*m));
}

/* ---- listed cells (checker extension) ----
 * Cells ids[0, nq) of the extended point set clipped with their rows of `knn`
 * (nq x K, in list order) exactly as om_cells clips them; the result is a mesh
 * whose cell t is ids[t] (unit-box units, face neighbours are extended ids). */
int om_cells_list(int dim, const double *ext, long n_ext, const long *ids, long nq, const uint32_t *knn, int K,
                  om_mesh *m) {
    (void)n_ext;
    memset(m, 0, sizeof(*m));
    m->dim = dim;
    m->n_seeds = nq;
    m->n_hydro = nq;
    m->seeds = (double *)calloc(nq * 3 + 3, sizeof(double));
    m->volumes = (double *)calloc(nq + 1, sizeof(double));
    m->face_counts = (long *)calloc(nq + 1, sizeof(long));
    m->face_ptr = (long *)calloc(nq + 1, sizeof(long));
    m->status = (int *)calloc(nq + 1, sizeof(int));
    m->cert_k = (int *)calloc(nq + 1, sizeof(int));
    m->centroid = (double *)calloc(nq * 3 + 3, sizeof(double));
    cell_out_t *outs = (cell_out_t *)malloc((nq > 0 ? nq : 1) * sizeof(cell_out_t));
#pragma omp parallel for schedule(dynamic, 4)
    for (long t = 0; t < nq; t++) {
        one_cell(dim, ext, ids[t], knn + (long)K * t, K, &outs[t], &m->status[t], &m->cert_k[t]);
        if (m->status[t] == OM_SUCCESS)
            for (int k = 0; k < dim; k++) m->seeds[3 * t + k] = ext[dim * ids[t] + k];
    }
    long F = 0;
    for (long t = 0; t < nq; t++) F += outs[t].nf;
    m->neighbor = (int *)malloc((F + 1) * sizeof(int));
    m->normal = (double *)malloc((F + 1) * 3 * sizeof(double));
    m->area = (double *)malloc((F + 1) * sizeof(double));
    F = 0;
    for (long t = 0; t < nq; t++) {
        const cell_out_t *o = &outs[t];
        m->face_ptr[t] = F;
        m->face_counts[t] = o->nf;
        m->volumes[t] = o->volume;
        if (m->status[t] == OM_SUCCESS)
            for (int k = 0; k < 3; k++) m->centroid[3 * t + k] = o->centroid[k];
        for (int f = 0; f < o->nf; f++, F++) {
            m->neighbor[F] = o->neighbor[f];
            for (int k = 0; k < 3; k++) m->normal[3 * F + k] = o->normal[f][k];
            m->area[F] = o->area[f];
        }
    }
    m->num_faces = F;
    free(outs);
    return 0;
}

/* m <- per cell i: b's cell sel[i] where sel[i] >= 0, else m's own */
static void merge_cells(om_mesh *m, const om_mesh *b, const long *sel) {
    long F = 0;
    for (long i = 0; i < m->n_seeds; i++) F += sel[i] >= 0 ? b->face_counts[sel[i]] : m->face_counts[i];
    int *nb = (int *)malloc((F + 1) * sizeof(int));
    double *nr = (double *)malloc((F + 1) * 3 * sizeof(double));
    double *ar = (double *)malloc((F + 1) * sizeof(double));
    long *fp = (long *)malloc((m->n_seeds + 1) * sizeof(long));
    long *fc = (long *)malloc((m->n_seeds + 1) * sizeof(long));
    long f = 0;
    for (long i = 0; i < m->n_seeds; i++) {
        const om_mesh *s = sel[i] >= 0 ? b : m;
        const long j = sel[i] >= 0 ? sel[i] : i;
        fp[i] = f;
        fc[i] = s->face_counts[j];
        for (long q = 0; q < s->face_counts[j]; q++, f++) {
            long g = s->face_ptr[j] + q;
            nb[f] = s->neighbor[g];
            for (int k = 0; k < 3; k++) nr[3 * f + k] = s->normal[3 * g + k];
            ar[f] = s->area[g];
        }
        if (sel[i] >= 0) {
            m->volumes[i] = b->volumes[j];
            m->status[i] = b->status[j];
            m->cert_k[i] = b->cert_k[j];
            for (int k = 0; k < 3; k++) m->centroid[3 * i + k] = b->centroid[3 * j + k], m->seeds[3 * i + k] = b->seeds[3 * j + k];
        }
    }
    free(m->neighbor);
    free(m->normal);
    free(m->area);
    free(m->face_ptr);
    free(m->face_counts);
    m->neighbor = nb;
    m->normal = nr;
    m->area = ar;
    m->face_ptr = fp;
    m->face_counts = fc;
    m->num_faces = F;
}

/* Listed cells clipped by the reference's algorithm with a budget large enough
 * to certify them: first K0 neighbours; every cell whose certificate did not
 * close (SECURITY_RADIUS_NOT_REACHED) is clipped again from scratch with 4x the
 * budget, up to k_max.  Since the clipping loop stops at the neighbour that
 * closes the certificate (voronoi.cpp:138), a certified result is the one the
 * reference gives with any _K_ at or beyond that neighbour.  k_used[t] (may be
 * NULL) receives the budget of the final attempt. */
int om_cells_certified(const om_grid *g, const double *ext, long n_ext, const long *ids, long nq, int K0,
                       int k_max, om_mesh *m, int *k_used) {
    const int dim = om_grid_dim(g);
    uint32_t *kl = (uint32_t *)malloc(((size_t)nq * K0 + 1) * sizeof(uint32_t));
    om_grid_knn(g, ids, nq, K0, kl);
    om_cells_list(dim, ext, n_ext, ids, nq, kl, K0, m);
    free(kl);
    if (k_used)
        for (long t = 0; t < nq; t++) k_used[t] = K0;
    int K = K0;
    long *sel = (long *)malloc((nq + 1) * sizeof(long));
    long *sub = (long *)malloc((nq + 1) * sizeof(long));
    long *pos = (long *)malloc((nq + 1) * sizeof(long));
    while (K < k_max) {
        long ns = 0;
        for (long t = 0; t < nq; t++)
            if (m->status[t] == OM_SECURITY_RADIUS_NOT_REACHED) sub[ns] = ids[t], pos[ns] = t, ns++;
        if (!ns) break;
        K = 4 * K < k_max ? 4 * K : k_max;
        uint32_t *k2 = (uint32_t *)malloc(((size_t)ns * K + 1) * sizeof(uint32_t));
        om_grid_knn(g, sub, ns, K, k2);
        om_mesh b;
        om_cells_list(dim, ext, n_ext, sub, ns, k2, K, &b);
        free(k2);
        for (long t = 0; t < nq; t++) sel[t] = -1;
        for (long s = 0; s < ns; s++) {
            sel[pos[s]] = s;
            if (k_used) k_used[pos[s]] = K;
        }
        merge_cells(m, &b, sel);
        om_mesh_free(&b);
    }
    free(sel);
    free(sub);
    free(pos);
    return 0;
}

int om_fallback_k = 0;
void om_set_fallback_k(int k) { om_fallback_k = k; }
int om_expand_k_max = 0;
void om_set_expand_k(int k_max) { om_expand_k_max = k_max; }

/* m <- per cell: b's result where m's hydro cell was SECURITY_RADIUS_NOT_REACHED, else m's */
static void merge_refit(om_mesh *m, const om_mesh *b, long n_hydro) {
    long F = 0;
    for (long i = 0; i < m->n_seeds; i++) {
        const om_mesh *s = (i < n_hydro && m->status[i] == OM_SECURITY_RADIUS_NOT_REACHED) ? b : m;
        F += s->face_counts[i];
    }
    int *nb = (int *)malloc((F + 1) * sizeof(int));
    double *nr = (double *)malloc((F + 1) * 3 * sizeof(double));
    double *ar = (double *)malloc((F + 1) * sizeof(double));
    long *fp = (long *)malloc((m->n_seeds + 1) * sizeof(long));
    long *fc = (long *)malloc((m->n_seeds + 1) * sizeof(long));
    long f = 0;
    for (long i = 0; i < m->n_seeds; i++) {
        const int use_b = i < n_hydro && m->status[i] == OM_SECURITY_RADIUS_NOT_REACHED;
        const om_mesh *s = use_b ? b : m;
        fp[i] = f;
        fc[i] = s->face_counts[i];
        for (long q = 0; q < s->face_counts[i]; q++, f++) {
            long g = s->face_ptr[i] + q;
            nb[f] = s->neighbor[g];
            for (int k = 0; k < 3; k++) nr[3 * f + k] = s->normal[3 * g + k];
            ar[f] = s->area[g];
        }
        if (use_b) {
            m->volumes[i] = b->volumes[i];
            m->status[i] = b->status[i];
            m->cert_k[i] = b->cert_k[i];
            for (int k = 0; k < 3; k++) m->centroid[3 * i + k] = b->centroid[3 * i + k], m->seeds[3 * i + k] = b->seeds[3 * i + k];
        }
    }
    free(m->neighbor);
    free(m->normal);
    free(m->area);
    free(m->face_ptr);
    free(m->face_counts);
    m->neighbor = nb;
    m->normal = nr;
    m->area = ar;
    m->face_ptr = fp;
    m->face_counts = fc;
    m->num_faces = F;
}

int om_build_mesh(int dim, int boundary, double buff, int K, const double *pts, long n, int hydro_only,
                  om_mesh *m) {
    const int nreg = om_num_regions(dim);
    double *ext = (double *)malloc((size_t)(nreg + 1) * (n > 0 ? n : 1) * dim * sizeof(double));
    long *gsrc = (long *)malloc((size_t)nreg * (n > 0 ? n : 1) * sizeof(long));
    int *gcode = (int *)malloc((size_t)nreg * (n > 0 ? n : 1) * sizeof(int));
    long ntot = om_ghosts(dim, boundary, buff, pts, n, ext, gsrc, gcode);
    uint32_t *knn = (uint32_t *)malloc(((size_t)ntot * K + 1) * sizeof(uint32_t));
    om_grid *grid = NULL;
    if (hydro_only) {
        /* only the hydro cells are clipped: only their rows are searched (the
           same lists as om_knn's first n rows) */
        grid = om_grid_new(dim, ext, ntot);
        long *q = (long *)malloc((n + 1) * sizeof(long));
        for (long i = 0; i < n; i++) q[i] = i;
        om_grid_knn(grid, q, n, K, knn);
        free(q);
    } else {
        om_knn(dim, ext, ntot, K, knn);
    }
    om_cells(dim, ext, ntot, n, knn, K, hydro_only ? n : ntot, m);
    free(knn);
    if (hydro_only && om_expand_k_max > K) {
        /* extension: hydro cells whose certificate did not close within K are
           clipped again with growing budgets up to om_expand_k_max */
        long nunc = 0;
        for (long i = 0; i < n; i++) nunc += m->status[i] == OM_SECURITY_RADIUS_NOT_REACHED;
        if (nunc) {
            long *ids = (long *)malloc(nunc * sizeof(long));
            long *sel = (long *)malloc((ntot + 1) * sizeof(long));
            nunc = 0;
            for (long i = 0; i < ntot; i++) {
                sel[i] = -1;
                if (i < n && m->status[i] == OM_SECURITY_RADIUS_NOT_REACHED) sel[i] = nunc, ids[nunc++] = i;
            }
            om_mesh b;
            om_cells_certified(grid, ext, ntot, ids, nunc, 4 * K, om_expand_k_max, &b, NULL);
            merge_cells(m, &b, sel);
            om_mesh_free(&b);
            free(ids);
            free(sel);
        }
    }
    om_grid_free(grid);
    if (hydro_only && om_fallback_k > K) {
        /* extension: hydro cells whose certificate did not close within K are
           recomputed with the fallback budget (the other cells keep their K result) */
        long nunc = 0;
        for (long i = 0; i < n; i++) nunc += m->status[i] == OM_SECURITY_RADIUS_NOT_REACHED;
        if (nunc) {
            const int K2 = om_fallback_k;
            uint32_t *knn2 = (uint32_t *)malloc((size_t)ntot * K2 * sizeof(uint32_t));
            om_knn(dim, ext, ntot, K2, knn2);
            om_mesh b;
            om_cells(dim, ext, ntot, n, knn2, K2, n, &b);
            free(knn2);
            merge_refit(m, &b, n);
            om_mesh_free(&b);
        }
    }
    /* kept: the second-order step measures generator offsets in the unit box */
    m->ext = (double *)realloc(ext, (size_t)(ntot > 0 ? ntot : 1) * dim * sizeof(double));
    m->ghost_ids = (long *)malloc((ntot - n + 1) * sizeof(long));
    m->ghost_code = (int *)malloc((ntot - n + 1) * sizeof(int));
    memcpy(m->ghost_ids, gsrc, (ntot - n) * sizeof(long));
    memcpy(m->ghost_code, gcode, (ntot - n) * sizeof(int));
    free(gsrc);
    free(gcode);

    /* scale back (periodic_mesh.cpp:146-166) */
    const double scale = 1. + (2 * buff);
    m->unit_scale = scale;
    const double vscale = dim == 2 ? scale * scale : scale * scale * scale;
    const double ascale = dim == 2 ? scale : scale * scale;
    for (long i = 0; i < ntot; i++) {
        for (int k = 0; k < dim; k++) {
            m->seeds[3 * i + k] = (m->seeds[3 * i + k] - 0.5) * scale + 0.5;
            if (m->status[i] == OM_SUCCESS) m->centroid[3 * i + k] = (m->centroid[3 * i + k] - 0.5) * scale + 0.5;
        }
        m->volumes[i] = vscale * m->volumes[i];
    }
    for (long f = 0; f < m->num_faces; f++) m->area[f] = ascale * m->area[f];
    return 0;
}
