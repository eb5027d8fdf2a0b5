/*
 * om.h -- CPU restatement of ProteusGPU's per-timestep mesh-and-flux path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the oracle that the CUDA path is
 * checked against (and the "port" CPU baseline); the product never links it.
 *
 * It restates, in plain C with runtime dimension and K, the reference's
 *   - periodic ghost layer + unit-box scaling   (src/voronoi/periodic_mesh.cpp:16-184)
 *   - exact K nearest neighbours               (src/knn/knn.cpp:16-347)
 *   - Ray et al. half-space clipping + security-radius certificate
 *                                              (src/voronoi/cell.cpp:42-411,
 *                                               src/voronoi/voronoi.cpp:115-155)
 *   - cell -> mesh extraction                  (src/voronoi/cell.cpp:416-669)
 *   - CFL time step and HLL flux update        (src/hydro/finite_volume_solver.cpp:43-186,
 *                                               src/hydro/riemann.cpp:7-124)
 * with the same FP64 operation sequence (build with -ffp-contract=off), so that
 * its results are bit-identical to the reference build in oracle/_ref.
 *
 * It also defines the semantics of what the reference does not have and the
 * moving-mesh workloads need: reflective (mirror) ghosts, mesh-point drift,
 * conserved-variable carry across re-meshing, face-pair-symmetric areas, the
 * outward-normal ("physical") flux sign, the certified-K record and cell
 * centroids.  Each such function says so.
 */
#ifndef PGPU_ORACLE_OM_H
#define PGPU_ORACLE_OM_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Cell status codes, same values as the reference's `Status` (allvars.h:13-20). */
enum {
    OM_TRIANGLE_OVERFLOW = 0,
    OM_VERTEX_OVERFLOW = 1,
    OM_INCONSISTENT_BOUNDARY = 2,
    OM_SECURITY_RADIUS_NOT_REACHED = 3,
    OM_SUCCESS = 4,
    OM_NEEDS_EXACT_PREDICATES = 5,
    OM_NOT_COMPUTED = 6 /* ghost cell skipped by a hydro-only build */
};

enum { OM_PERIODIC = 0, OM_REFLECTIVE = 1 };

/* Clipping pool limits, the reference's defaults (Config.sh:37-38). */
#define OM_MAX_P 64
#define OM_MAX_T 96

typedef struct {
    int dim;
    long n_seeds;   /* hydro + ghost cells */
    long n_hydro;
    long num_faces;
    double *seeds;      /* n_seeds * 3, physical coordinates (z = 0 in 2D) */
    double *volumes;    /* n_seeds */
    long *face_counts;  /* n_seeds */
    long *face_ptr;     /* n_seeds, CSR start in the face arrays */
    int *neighbor;      /* num_faces; input/ghost id of the other cell, -1 = box face */
    double *normal;     /* num_faces * 3; unit plane normal, pointing into the cell (reference convention) */
    double *area;       /* num_faces; edge length (2D) or face area (3D), physical units */
    long *ghost_ids;    /* n_seeds - n_hydro; hydro id each ghost copies */
    int *ghost_code;    /* n_seeds - n_hydro; image code, see om_image_code() */
    int *status;        /* n_seeds */
    int *cert_k;        /* n_seeds; 1-based neighbour index where the certificate closed, 0 if never */
    double *centroid;   /* n_seeds * 3, physical coordinates */
    double *ext;        /* n_seeds * dim: the unit-box points the mesh was built on (om_build_mesh
                           only; NULL otherwise) */
    double unit_scale;  /* 1 + 2 buff: unit box -> physical (om_build_mesh only) */
} om_mesh;

/* ---- ghosts -------------------------------------------------------------- */

/* Image code of a ghost: per axis a in 0..dim-1 a base-3 digit d_a, with
 * d_a = 0 for no change, 1 for the image across the low wall (periodic shift
 * +1 or mirror x -> -x), 2 for the image across the high wall (shift -1 or
 * mirror x -> 2 - x).  code = d_0 + 3 d_1 + 9 d_2. */
int om_image_code(const int *shift, int dim);

/* Number of ghost regions (8 in 2D, 26 in 3D) and their shift vectors in the
 * reference's order (periodic_mesh.cpp:71-110). */
int om_num_regions(int dim);
void om_region_shift(int dim, int r, int *shift3);

/* Builds the extended point set (hydro points first, then ghosts in the
 * reference's order) scaled into the unit box as the reference does
 * (periodic_mesh.cpp:63-126).  `ext` needs capacity (1 + num_regions) * n * dim.
 * Returns the number of extended points. */
long om_ghosts(int dim, int boundary, double buff, const double *pts, long n,
               double *ext, long *ghost_src, int *ghost_code);

/* ---- work counters (instrumentation for the roofline's algorithmic counts) ----
 * [0] KNN candidate distance evaluations, [1] clip plane-vertex predicates,
 * [2] vertices created, [3] cells clipped. */
void om_reset_counters(void);
void om_get_counters(long *out4);

/* ---- KNN --------------------------------------------------------------- */

/* Exact K nearest neighbours of every point of `pts` (n x dim, unit box),
 * excluding itself, ascending by (squared distance, index).  Unfilled slots are
 * UINT32_MAX.  Uses a uniform grid with Chebyshev-ring search as in
 * knn.cpp:16-315.  Returns 0. */
int om_knn(int dim, const double *pts, long n, int K, uint32_t *out);

/* Exact K nearest neighbours of listed queries (checker extension): the grid
 * of om_knn built once for a point set (which must outlive it), and per query
 * the same ring order and stopping rule, hence the same row as om_knn gives
 * that point; the best K are selected from a candidate buffer, so large K
 * (thousands) stays cheap.  out is nq x K. */
typedef struct om_grid om_grid;
om_grid *om_grid_new(int dim, const double *pts, long n);
void om_grid_free(om_grid *g);
int om_grid_dim(const om_grid *g);
int om_grid_knn(const om_grid *g, const long *queries, long nq, int K, uint32_t *out);

/* ---- cells ------------------------------------------------------------- */

/* Clips and extracts cells [0, n_cells) of the extended unit-box point set
 * (cells >= n_compute are skipped and get OM_NOT_COMPUTED), producing a mesh
 * in unit-box units.  knn is n_ext x K in extended ids. */
int om_cells(int dim, const double *ext, long n_ext, long n_hydro, const uint32_t *knn, int K,
             long n_compute, om_mesh *mesh);

/* The whole mesh build: ghosts (periodic or reflective within `buff`), unit-box
 * scaling, KNN, clipping, extraction and the rescale back
 * (periodic_mesh.cpp:44-184).  hydro_only skips the ghost cells. */
int om_build_mesh(int dim, int boundary, double buff, int K, const double *pts, long n,
                  int hydro_only, om_mesh *mesh);

void om_mesh_free(om_mesh *mesh);

/* Checker extensions.  om_cells_list clips the listed cells ids[0, nq) with
 * their neighbour rows knn (nq x K) as om_cells does; the result's cell t is
 * ids[t] (n_seeds = nq, unit-box units, extended ids as face neighbours).
 * om_cells_certified clips them with K0 neighbours and again with 4x budgets,
 * up to k_max, while their certificate does not close: the reference's
 * algorithm with a _K_ large enough for each cell.  k_used may be NULL. */
int om_cells_list(int dim, const double *ext, long n_ext, const long *ids, long nq, const uint32_t *knn, int K,
                  om_mesh *mesh);
int om_cells_certified(const om_grid *g, const double *ext, long n_ext, const long *ids, long nq, int K0,
                       int k_max, om_mesh *mesh, int *k_used);

/* Test hook: 0 = the reference's boundary walk (default), 1 = the set-based
 * cavity boundary that the CUDA kernel uses. */
void om_set_boundary_mode(int mode);

/* Extensions used by the moving-mesh workloads (both default to the reference's
 * behaviour, 0):
 *   predicate mode 1 keeps a vertex whose plane predicate is within the
 *   reference's error bound of zero instead of failing the cell;
 *   fallback K > K recomputes, in hydro-only builds, the hydro cells whose
 *   certificate did not close within K with the larger budget. */
void om_set_predicate_mode(int mode);
void om_set_fallback_k(int k);
/* Extension (default 0 = off): in hydro-only builds, hydro cells whose
 * certificate did not close within K are clipped again by om_cells_certified
 * with budgets from 4K up to k_max (the cells the CUDA path certifies by its
 * grid walk). */
void om_set_expand_k(int k_max);

/* ---- hydro ------------------------------------------------------------- */

/* hydro::dt_CFL (finite_volume_solver.cpp:151-186). v is n_hydro x dim. */
double om_dt_cfl(const om_mesh *mesh, double cfl, double gamma, const double *rho,
                 const double *v, const double *E);

/* hydro::hydro_step (finite_volume_solver.cpp:43-123) in place, reference
 * arithmetic: inward stored normal, each side's own face area. Returns the
 * number of faces whose neighbour is a box face (the reference would crash). */
long om_hydro_step_ref(const om_mesh *mesh, double dt, double gamma, double *rho, double *v, double *E);

/* Extension.  One moving-mesh step on conserved variables:
 *   W = (m/V, p/m, e/V); dt = CFL min (reference formula);
 *   Q_i -= dt * sum_faces HLL(W_i, W_j, n_out) A_sym;  x_i += v_i dt (v at step start),
 * then wrap (periodic) or reflect (reflective) into [0,1)^dim.
 * n_out is the outward normal (the negated stored one); A_sym is the area computed
 * by the lower hydro id of the face pair, so the update is antisymmetric.
 * mirror ghosts flip the velocity components normal to their walls.
 * If fixed_dt > 0 it is used instead of the CFL step.  Returns dt. */
double om_step_moving(const om_mesh *mesh, double cfl, double fixed_dt, double gamma, int boundary,
                      double *x, double *mass, double *mom, double *energy, long *n_unpaired);

/* Extension: one moving-mesh step with moving faces (the faces move with the
 * generators, so the Riemann problem is solved in the face's frame), first or
 * second order, on conserved variables, for periodic boxes (the mesh from
 * om_build_mesh, which keeps its unit-box points).  order 1: the cells'
 * primitives as face states (no gradients, no prediction); order 2:
 * MUSCL-Hancock on the moving Voronoi mesh (Springel 2010, MNRAS 401, 791,
 * sections 3.2-3.3), with the least-squares gradients of Pakmor et al. 2016
 * (MNRAS 455, 1134) and the moving-face flux of Pakmor et al. 2011:
 *   primitives W = (rho, v, P) per cell; dt = CFL min (reference formula);
 *   gradients: per variable, min_g sum_faces (A/|d|^2) (W_j - W_i - g.d)^2 with
 *     d = x_j - x_i (the neighbour's image), solved by the 2x2 / 3x3 normal
 *     equations, then limited by alpha = min(1, min_faces psi), psi = (W_max -
 *     W_i) / (g.d/2) or (W_min - W_i) / (g.d/2) by the sign of g.d (W_max, W_min
 *     over the cell and its neighbours);
 *   half-step prediction in the frame of the cell (which moves with v):
 *     rho' = rho - dt/2 rho div v, v' = v - dt/2 grad P / rho, P' = P - dt/2 gamma P div v;
 *   face states at the midpoint of the generators: W_L = W'_i + g_i.d/2,
 *     W_R = W'_j - g_j.d/2 (first order, W' alone, when either has rho or P <= 0);
 *   the face moves with w = (v_i + v_j)/2: HLL on the states boosted by -w along
 *     the outward normal, then back to the lab frame: F_rho, F_m + w F_rho,
 *     F_E + w.F_m + |w|^2 F_rho / 2;
 *   Q_i -= dt sum F A_sym;  x_i += v_i dt, wrapped.
 * For a face whose other cell has the lower hydro id, d and the area are those
 * the lower id computes for the same face (negated), so both cells evaluate the
 * same face states and every face flux cancels exactly between them.
 * Returns dt, or -1 when the mesh has no unit-box points or is not periodic. */
double om_step_ale(const om_mesh *mesh, int order, double cfl, double fixed_dt, double gamma, double *x,
                   double *mass, double *mom, double *energy, long *n_unpaired);

/* Face-pair symmetric areas (extension): out[f] = area of the same face as seen from
 * the lower hydro id.  Returns the number of faces with no partner found. */
long om_symmetric_area(const om_mesh *mesh, double *out);

#ifdef __cplusplus
}
#endif
#endif
