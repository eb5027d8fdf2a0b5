#define _GNU_SOURCE
/*
 * Exact K nearest neighbours (test-infrastructure oracle).
 *
 * Restates knn::init / sort_points_into_grid / cpu_knearest
 * (src/knn/knn.cpp:16-315): points are binned into an N_grid^D uniform grid
 * (N_grid from the same expression, knn.cpp:22), and each query scans
 * Chebyshev rings of bins outwards, stopping before ring r once its K-th best
 * squared distance is below ((r-1)/N_grid)^2 (knn.cpp:267-273).  The squared
 * distance is dist2_point's dx*dx + dy*dy (+ dz*dz) (knn.h:64-75); the query
 * itself is skipped (knn.cpp:285).
 *
 * Differences, all of which leave the result equal to the reference's whenever
 * squared distances are distinct:
 *   - neighbours are ordered by (squared distance, index) instead of the
 *     heap's unspecified order among equal distances;
 *   - bins are addressed by (i, j, k) and rings clipped to the grid, so no bin
 *     is visited twice (the reference's linear offsets alias across rows,
 *     knn.cpp:58,77, which only adds candidates);
 *   - the ring count is not capped at 15 and grids below 16^D are allowed.
 */
#include "om.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

long om_counters_g[4];  /* see om_get_counters */

void om_reset_counters(void) {
    for (int i = 0; i < 4; i++) om_counters_g[i] = 0;
}

void om_get_counters(long *out4) {
    for (int i = 0; i < 4; i++) out4[i] = om_counters_g[i];
}

static int n_grid_for(long n, int dim) {
    int g = (int)round(pow((double)(n / 3.1f), (double)(1.0f / (float)dim)));
    return g < 1 ? 1 : g;
}

static int bin_coord(double x, int G) {
    int i = (int)floor(x * (double)G);
    if (i < 0) i = 0;
    if (i > G - 1) i = G - 1;
    return i;
}

static double dist2(const double *a, const double *b, int dim) {
    double dx = a[0] - b[0];
    double dy = a[1] - b[1];
    if (dim == 2) return dx * dx + dy * dy;
    double dz = a[2] - b[2];
    return dx * dx + dy * dy + dz * dz;
}

/* insert (d, id) into the ascending list of length *cnt (capacity K) */
static void topk_insert(double *bd, uint32_t *bi, int *cnt, int K, double d, uint32_t id) {
    int c = *cnt;
    if (c == K) {
        if (d > bd[K - 1] || (d == bd[K - 1] && id >= bi[K - 1])) return;
        c = K - 1;
    }
    int pos = c;
    while (pos > 0 && (bd[pos - 1] > d || (bd[pos - 1] == d && bi[pos - 1] > id))) {
        bd[pos] = bd[pos - 1];
        bi[pos] = bi[pos - 1];
        pos--;
    }
    bd[pos] = d;
    bi[pos] = id;
    if (*cnt < K) (*cnt)++;
}

int om_knn(int dim, const double *pts, long n, int K, uint32_t *out) {
    const int G = n_grid_for(n, dim);
    const long nb = dim == 2 ? (long)G * G : (long)G * G * G;
    long *start = (long *)calloc(nb + 1, sizeof(long));
    long *order = (long *)malloc((n > 0 ? n : 1) * sizeof(long));
    int *bin = (int *)malloc((n > 0 ? n : 1) * sizeof(int));
    for (long i = 0; i < n; i++) {
        const double *p = pts + i * dim;
        int b = bin_coord(p[0], G) + G * bin_coord(p[1], G);
        if (dim == 3) b += G * G * bin_coord(p[2], G);
        bin[i] = b;
        start[b + 1]++;
    }
    for (long b = 0; b < nb; b++) start[b + 1] += start[b];
    {
        long *fill = (long *)calloc(nb, sizeof(long));
        for (long i = 0; i < n; i++) order[start[bin[i]] + fill[bin[i]]++] = i;
        free(fill);
    }

    long total_cand = 0;
#pragma omp parallel reduction(+ : total_cand)
    {
        double *bd = (double *)malloc(K * sizeof(double));
        uint32_t *bi = (uint32_t *)malloc(K * sizeof(uint32_t));
#pragma omp for schedule(dynamic, 256)
        for (long q = 0; q < n; q++) {
            const double *p = pts + q * dim;
            int c[3] = {bin_coord(p[0], G), bin_coord(p[1], G), dim == 3 ? bin_coord(p[2], G) : 0};
            int cnt = 0;
            for (int r = 0; r <= G; r++) {
                if (r >= 1 && cnt == K) {
                    double md = (double)(r - 1) / (double)G;
                    if (bd[K - 1] < md * md) break;
                }
                int zlo = dim == 3 ? -r : 0, zhi = dim == 3 ? r : 0;
                for (int dz = zlo; dz <= zhi; dz++) {
                    int z = c[2] + dz;
                    if (dim == 3 && (z < 0 || z >= G)) continue;
                    for (int dy = -r; dy <= r; dy++) {
                        int y = c[1] + dy;
                        if (y < 0 || y >= G) continue;
                        for (int dx = -r; dx <= r; dx++) {
                            int ar = abs(dx);
                            if (abs(dy) > ar) ar = abs(dy);
                            if (abs(dz) > ar) ar = abs(dz);
                            if (ar != r) continue;
                            int x = c[0] + dx;
                            if (x < 0 || x >= G) continue;
                            long b = x + (long)G * y + (long)G * G * z;
                            for (long s = start[b]; s < start[b + 1]; s++) {
                                long j = order[s];
                                if (j == q) continue;
                                total_cand++;
                                topk_insert(bd, bi, &cnt, K, dist2(p, pts + j * dim, dim), (uint32_t)j);
                            }
                        }
                    }
                }
            }
            for (int t = 0; t < K; t++) out[q * K + t] = t < cnt ? bi[t] : UINT32_MAX;
        }
        free(bd);
        free(bi);
    }
    om_counters_g[0] += total_cand;
    free(start);
    free(order);
    free(bin);
    return 0;
}

/* ---- exact K nearest neighbours of listed queries (checker extension) ----
 * The same grid (N_grid from knn.cpp:22), the same Chebyshev-ring order and the
 * same stopping rule as om_knn, so a query's list is identical to its om_knn
 * row; only the listed queries are searched, and the best K are kept by
 * selection over a candidate buffer instead of insertion, so that budgets of
 * thousands of neighbours stay cheap.  The grid is built once per point set. */
struct om_grid {
    int dim, G;
    long n;
    const double *pts;
    long *start, *order;
};

om_grid *om_grid_new(int dim, const double *pts, long n) {
    om_grid *g = (om_grid *)calloc(1, sizeof(om_grid));
    g->dim = dim;
    g->n = n;
    g->pts = pts;
    g->G = n_grid_for(n, dim);
    const int G = g->G;
    const long nb = dim == 2 ? (long)G * G : (long)G * G * G;
    g->start = (long *)calloc(nb + 1, sizeof(long));
    g->order = (long *)malloc((n > 0 ? n : 1) * sizeof(long));
    int *bin = (int *)malloc((n > 0 ? n : 1) * sizeof(int));
    for (long i = 0; i < n; i++) {
        const double *p = pts + i * dim;
        int b = bin_coord(p[0], G) + G * bin_coord(p[1], G);
        if (dim == 3) b += G * G * bin_coord(p[2], G);
        bin[i] = b;
        g->start[b + 1]++;
    }
    for (long b = 0; b < nb; b++) g->start[b + 1] += g->start[b];
    long *fill = (long *)calloc(nb, sizeof(long));
    for (long i = 0; i < n; i++) g->order[g->start[bin[i]] + fill[bin[i]]++] = i;
    free(fill);
    free(bin);
    return g;
}

int om_grid_dim(const om_grid *g) { return g->dim; }

void om_grid_free(om_grid *g) {
    if (!g) return;
    free(g->start);
    free(g->order);
    free(g);
}

typedef struct {
    double d;
    uint32_t i;
} om_cand;

static int cmp_cand(const void *a, const void *b) {
    const om_cand *x = (const om_cand *)a, *y = (const om_cand *)b;
    if (x->d < y->d) return -1;
    if (x->d > y->d) return 1;
    return (x->i > y->i) - (x->i < y->i);
}

int om_grid_knn(const om_grid *g, const long *queries, long nq, int K, uint32_t *out) {
    const int dim = g->dim, G = g->G;
    const double *pts = g->pts;
#pragma omp parallel
    {
        long cap = 4096;
        om_cand *buf = (om_cand *)malloc(cap * sizeof(om_cand));
#pragma omp for schedule(dynamic, 16)
        for (long t = 0; t < nq; t++) {
            const long q = queries[t];
            const double *p = pts + q * dim;
            int c[3] = {bin_coord(p[0], G), bin_coord(p[1], G), dim == 3 ? bin_coord(p[2], G) : 0};
            long cnt = 0;
            int have = 0;
            double kth = 0.0;
            for (int r = 0; r <= G; r++) {
                if (r >= 1 && have) {
                    double md = (double)(r - 1) / (double)G;
                    if (kth < md * md) break;
                }
                int zlo = dim == 3 ? -r : 0, zhi = dim == 3 ? r : 0;
                for (int dz = zlo; dz <= zhi; dz++) {
                    int z = c[2] + dz;
                    if (dim == 3 && (z < 0 || z >= G)) continue;
                    for (int dy = -r; dy <= r; dy++) {
                        int y = c[1] + dy;
                        if (y < 0 || y >= G) continue;
                        for (int dx = -r; dx <= r; dx++) {
                            int ar = abs(dx);
                            if (abs(dy) > ar) ar = abs(dy);
                            if (abs(dz) > ar) ar = abs(dz);
                            if (ar != r) continue;
                            int x = c[0] + dx;
                            if (x < 0 || x >= G) continue;
                            long b = x + (long)G * y + (long)G * G * z;
                            for (long s = g->start[b]; s < g->start[b + 1]; s++) {
                                long j = g->order[s];
                                if (j == q) continue;
                                double d = dist2(p, pts + j * dim, dim);
                                if (have && d > kth) continue;
                                if (cnt == cap) {
                                    cap *= 2;
                                    buf = (om_cand *)realloc(buf, cap * sizeof(om_cand));
                                }
                                buf[cnt].d = d;
                                buf[cnt].i = (uint32_t)j;
                                cnt++;
                            }
                        }
                    }
                }
                if (cnt >= K) {
                    qsort(buf, cnt, sizeof(om_cand), cmp_cand);
                    cnt = K;
                    kth = buf[K - 1].d;
                    have = 1;
                }
            }
            if (!have) qsort(buf, cnt, sizeof(om_cand), cmp_cand);
            for (int k = 0; k < K; k++) out[t * K + k] = k < cnt ? buf[k].i : UINT32_MAX;
        }
        free(buf);
    }
    return 0;
}
