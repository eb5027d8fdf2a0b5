/*
 * Ghost layer and unit-box scaling (test-infrastructure oracle).
 *
 * Restates voronoi::compute_periodic_mesh's ghost selection and scaling
 * (src/voronoi/periodic_mesh.cpp:16-41 is_in/add_ghost, :63-126 regions and
 * scale).  The 8 (2D) / 26 (3D) regions are visited per point in the
 * reference's order, because that order numbers the ghosts and the ghost ids
 * appear as face neighbours.  A region is described by its shift vector: a
 * shift of +1 on an axis selects coordinates in the open interval (0, buff),
 * -1 selects (1-buff, 1) and 0 selects (0, 1), exactly the intervals the
 * reference's is_in() tests with strict comparisons.
 *
 * Reflective (mirror) ghosts are an extension: same regions, but the copy is
 * mirrored across the wall(s) instead of shifted (x -> -x at the low wall,
 * x -> 2 - x at the high wall).
 */
#include "om.h"

#include <stdlib.h>

/* Shift vectors in the order of periodic_mesh.cpp:71-79 (2D) and :83-110 (3D). */
static const int k_regions_2d[8][2] = {
    {1, 0}, {0, -1}, {-1, 0}, {0, 1}, {1, 1}, {1, -1}, {-1, -1}, {-1, 1}};

static const int k_regions_3d[26][3] = {
    /* faces */
    {0, 0, 1}, {1, 0, 0}, {0, -1, 0}, {-1, 0, 0}, {0, 1, 0}, {0, 0, -1},
    /* edges */
    {0, 1, 1}, {1, 0, 1}, {0, -1, 1}, {-1, 0, 1}, {1, 1, 0}, {1, -1, 0},
    {-1, -1, 0}, {-1, 1, 0}, {1, 0, -1}, {0, -1, -1}, {-1, 0, -1}, {0, 1, -1},
    /* corners */
    {1, 1, 1}, {1, -1, 1}, {-1, -1, 1}, {-1, 1, 1}, {1, 1, -1}, {1, -1, -1},
    {-1, -1, -1}, {-1, 1, -1}};

int om_num_regions(int dim) { return dim == 2 ? 8 : 26; }

void om_region_shift(int dim, int r, int *shift3) {
    shift3[2] = 0;
    if (dim == 2) {
        shift3[0] = k_regions_2d[r][0];
        shift3[1] = k_regions_2d[r][1];
    } else {
        shift3[0] = k_regions_3d[r][0];
        shift3[1] = k_regions_3d[r][1];
        shift3[2] = k_regions_3d[r][2];
    }
}

int om_image_code(const int *shift, int dim) {
    int code = 0, mul = 1;
    for (int a = 0; a < dim; a++) {
        int d = shift[a] == 0 ? 0 : (shift[a] > 0 ? 1 : 2);
        code += d * mul;
        mul *= 3;
    }
    return code;
}

/* is_in(): strict open intervals per axis (periodic_mesh.cpp:16-24). */
static int in_region(const double *p, const int *shift, int dim, double buff) {
    for (int a = 0; a < dim; a++) {
        double lo, hi;
        if (shift[a] > 0) {
            lo = 0.;
            hi = 0. + buff;
        } else if (shift[a] < 0) {
            lo = 1. - buff;
            hi = 1.;
        } else {
            lo = 0.;
            hi = 1.;
        }
        if (!(p[a] > lo && p[a] < hi)) return 0;
    }
    return 1;
}

long om_ghosts(int dim, int boundary, double buff, const double *pts, long n, double *ext,
               long *ghost_src, int *ghost_code) {
    const int nreg = om_num_regions(dim);
    long ng = 0;
    for (long i = 0; i < n; i++) ext[i * dim + 0] = pts[i * dim + 0], ext[i * dim + 1] = pts[i * dim + 1];
    if (dim == 3)
        for (long i = 0; i < n; i++) ext[i * 3 + 2] = pts[i * 3 + 2];
    for (long i = 0; i < n; i++) {
        const double *p = pts + i * dim;
        for (int r = 0; r < nreg; r++) {
            int s[3];
            om_region_shift(dim, r, s);
            if (!in_region(p, s, dim, buff)) continue;
            double *g = ext + (n + ng) * dim;
            for (int a = 0; a < dim; a++) {
                if (boundary == OM_PERIODIC) {
                    /* add_ghost: pts[index].x + shift_x (periodic_mesh.cpp:28-33) */
                    g[a] = p[a] + (double)s[a];
                } else {
                    g[a] = s[a] > 0 ? -p[a] : (s[a] < 0 ? 2.0 - p[a] : p[a]);
                }
            }
            ghost_src[ng] = i;
            ghost_code[ng] = om_image_code(s, dim);
            ng++;
        }
    }
    /* scale into [0,1]^dim (periodic_mesh.cpp:119-126) */
    const double scale = 1. / (1. + (2 * buff));
    const long ntot = n + ng;
    for (long i = 0; i < ntot * dim; i++) ext[i] = scale * (ext[i] - 0.5) + 0.5;
    return ntot;
}
