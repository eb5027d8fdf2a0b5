/*
 * proteus_gpu.h -- C ABI of the B200 (sm_100a) mesh-and-flux path.
 *
 * Plain pointers and sizes only.  One context owns one CUDA stream and all
 * device buffers of one simulation; calls on one context are not reentrant,
 * different contexts are independent.  Every entry point returns 0 on success
 * or a negative PGPU_E* code; pgpu_last_error() gives the message.
 *
 * Which reference interface each entry point replaces is cited beside it
 * (paths relative to the reference project's root).  The reference's C++
 * signatures themselves are kept by the drop-in translation units in
 * proteusgpu_b200/dropin/, which forward to this ABI.
 *
 * Layouts follow the reference's VMesh (src/voronoi/voronoi.h:22-41):
 *   cells  : seeds double[3] (z = 0 in 2D), volumes, face_counts, face_ptr (u64)
 *   faces  : neighbor_cell int32 (-1 = bounding-box face), face_normal double[3]
 *            (unit, pointing from the neighbour into the cell), face_area
 *   ghosts : ghost_ids u64, the hydro id each ghost cell copies
 * and primitives follow primvars (src/global/allvars.h:203-207): rho, v
 * (dim doubles per cell), E (total energy per unit volume).
 */
#ifndef PROTEUS_GPU_H
#define PROTEUS_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PGPU_ABI_VERSION 1

/* error codes */
#define PGPU_OK 0
#define PGPU_EINVAL (-1)   /* bad argument */
#define PGPU_ECUDA (-2)    /* CUDA runtime error */
#define PGPU_ESTATE (-3)   /* call out of order (e.g. no mesh yet) */
#define PGPU_ECAPACITY (-4) /* a size exceeds a fixed limit */
#define PGPU_EMESH (-5)    /* mesh unusable for the requested step (failed cells, box faces) */

/* boundary handling of the ghost layer */
#define PGPU_PERIODIC 0   /* shifted copies, src/voronoi/periodic_mesh.cpp:63-112 */
#define PGPU_REFLECTIVE 1 /* mirrored copies (extension) */

/* flux conventions */
#define PGPU_FLUX_REFERENCE 0 /* stored (inward) normal, each cell's own face area: riemann.cpp:7-45 as is */
#define PGPU_FLUX_PHYSICAL 1  /* outward normal, face-pair-symmetric area: conservative to round-off */
/* Moving-mesh steps only (extension), periodic boxes: the faces move with the
 * generators (velocity (v_i + v_j)/2) and the Riemann problem is solved in the
 * face's frame; outward normal, pair-symmetric area, exactly conservative.
 * ALE1: first order; ALE2: second order (MUSCL-Hancock: least-squares
 * gradients, slope limiter, half-step prediction, face states at the
 * generators' midpoint).  pgpu_hydro_step (the reference's static step)
 * treats them as PGPU_FLUX_PHYSICAL. */
#define PGPU_FLUX_ALE1 2
#define PGPU_FLUX_ALE2 3

/* plane-vertex predicate near zero (|det| below the reference's error bound, cell.cpp:187-218) */
#define PGPU_PRED_REFERENCE 0 /* as the reference: the cell fails with NEEDS_EXACT_PREDICATES */
#define PGPU_PRED_ROBUST 1    /* the vertex is kept (treated as not cut); needed for mirror walls,
                                 whose symmetric point sets make exact degeneracies */

/* clipping precision (extension): FP32 clips in a frame centred on each seed with an
 * error-bounded predicate, hands undecided cells to the FP64 kernel, and extracts
 * certified cells in FP64 -- same topology, statuses and geometry as FP64 */
#define PGPU_CLIP_FP64 0
#define PGPU_CLIP_FP32 1

/* cell status codes: the reference's Status enum, src/global/allvars.h:13-20 */
#define PGPU_TRIANGLE_OVERFLOW 0
#define PGPU_VERTEX_OVERFLOW 1
#define PGPU_INCONSISTENT_BOUNDARY 2
#define PGPU_SECURITY_RADIUS_NOT_REACHED 3
#define PGPU_SUCCESS 4
#define PGPU_NEEDS_EXACT_PREDICATES 5
#define PGPU_NOT_COMPUTED 6 /* ghost cell, skipped by the per-step path */

typedef struct pgpu_ctx pgpu_ctx;

typedef struct {
    int dim;          /* 2 or 3 (the reference's dim_2D / dim_3D) */
    int k;            /* neighbour budget, the reference's _K_ (Config.sh:34); 1..256 */
    int boundary;     /* PGPU_PERIODIC or PGPU_REFLECTIVE */
    int flux_mode;    /* PGPU_FLUX_REFERENCE or PGPU_FLUX_PHYSICAL */
    double buff;      /* ghost layer width, the reference's global `buff` (allvars.cpp:13) */
    double gamma;     /* adiabatic index, the reference's global `_gamma_` (allvars.cpp:14) */
    int device;       /* CUDA device ordinal */
    int verbose;      /* 0 = silent */
    int predicates;   /* PGPU_PRED_REFERENCE or PGPU_PRED_ROBUST */
    int k_fallback;   /* moving-mesh steps only: hydro cells whose certificate does not close
                         within k neighbours are recomputed with this budget (0 = off; k < k_fallback <= 256) */
    int precision;    /* PGPU_CLIP_FP64 or PGPU_CLIP_FP32 */
} pgpu_params;

/* Fills p with the reference's defaults: dim 3, K 190, periodic, reference flux,
 * buff 0.04, gamma 5/3, device 0. */
void pgpu_default_params(pgpu_params *p);

int pgpu_create(const pgpu_params *p, pgpu_ctx **out);
void pgpu_destroy(pgpu_ctx *ctx);
const char *pgpu_last_error(const pgpu_ctx *ctx);
int pgpu_abi_version(void);

/* ---------------------------------------------------------------- KNN ---
 * knn::init + knn::solve + knn::get_knearest + knn::get_permutation
 * (src/knn/knn.h:36-57, src/knn/knn.cpp:16-234).  pts: n x dim doubles in the
 * unit box, host memory.  out: n x k neighbour ids (input ids, ascending by
 * squared distance then id; UINT32_MAX where fewer than k exist).  The sorted
 * order is internal; it is returned by pgpu_knn_sorted for the drop-in's
 * knn_problem. */
int pgpu_knn(pgpu_ctx *ctx, const double *pts, int64_t n, uint32_t *out);

/* After pgpu_knn: the internal grid order (knn::get_points / get_permutation,
 * src/knn/knn.cpp:445-455): sorted points (n x dim) and perm[sorted] = input id;
 * and the grid resolution.  Any pointer may be NULL. */
int pgpu_knn_sorted(pgpu_ctx *ctx, double *sorted_pts, uint32_t *perm, int *n_grid);

/* ---------------------------------------------------------------- mesh ---
 * voronoi::compute_periodic_mesh (src/voronoi/periodic_mesh.cpp:44-184):
 * ghosts within buff (periodic or mirrored), unit-box scaling, KNN, clipping
 * with the security-radius certificate, extraction and rescale.  All cells,
 * hydro and ghost, are computed, as in the reference.  The mesh stays on the
 * device; sizes are returned. */
int pgpu_periodic_mesh(pgpu_ctx *ctx, const double *pts, int64_t n, int64_t *n_seeds, int64_t *num_faces);

/* voronoi::compute_mesh (src/voronoi/voronoi.cpp:17-64) on n points already
 * in the unit box: no ghosts, no scaling; n_hydro = n. */
int pgpu_compute_mesh(pgpu_ctx *ctx, const double *pts, int64_t n, int64_t *num_faces);

/* Copies the current mesh to host arrays in the reference's VMesh layout,
 * cells in input order with faces contiguous per cell
 * (src/voronoi/voronoi.cpp:212-333 unpermute_vmesh).  Any pointer may be NULL.
 * status and cert_k are per cell; cert_k is the 1-based neighbour index at which
 * the certificate closed (0 if it did not); centroid is an extension. */
int pgpu_download_mesh(pgpu_ctx *ctx, double *seeds, double *volumes, uint64_t *face_counts,
                       uint64_t *face_ptr, int32_t *neighbor, double *normal, double *area,
                       uint64_t *ghost_ids, int32_t *status, int32_t *cert_k, double *centroid);

/* ------------------------------------------------------ mesh checkers ---
 * Diagnostics with no reference counterpart: read parts of the current mesh
 * back without downloading all of it, so that a checker can recompute sampled
 * cells of a full-size mesh on the host.  They allocate and free staging
 * memory and synchronise the stream.
 *
 * pgpu_download_points: the extended point set the mesh was built on, hydro
 * points then ghosts (extended ids), in the unit box (n_seeds x dim doubles),
 * exactly the coordinates the KNN and the clipping used. */
int pgpu_download_points(pgpu_ctx *ctx, double *ext_unit);

/* The query slots of the hydro cells that the last mesh build certified by the
 * grid walk (cells whose security sphere reaches past every neighbour budget):
 * *count receives their number; out (capacity cap) may be NULL. */
int pgpu_walked_slots(pgpu_ctx *ctx, uint32_t *out, int64_t cap, int64_t *count);

/* n sampled query slots (0 <= slot < number of cells the last build computed;
 * slot order is the mesh's internal spatial order): per slot its extended id,
 * the neighbour row the main clipping pass used (lists: n x k extended ids;
 * list_len = the budget it had, k or the cell's learned budget, the rest of
 * the row UINT32_MAX), status, cert_k,
 * volume and centroid (physical units, as pgpu_download_mesh), and the
 * cell's faces in stored order: face_ptr (n + 1 entries, always filled),
 * neighbor / normal (x 3) / area (physical units) of capacity face_cap, or all
 * three NULL to get face_ptr only.  PGPU_ECAPACITY if face_ptr[n] > face_cap. */
int pgpu_sample_cells(pgpu_ctx *ctx, const uint32_t *slots, int64_t n, uint32_t *ext_id, uint16_t *list_len,
                      uint32_t *lists, int32_t *status, int32_t *cert_k, double *volumes, double *centroid,
                      uint64_t *face_ptr, int32_t *neighbor, double *normal, double *area, int64_t face_cap);

/* Mesh sizes: cells (hydro + ghost), hydro cells, faces. */
int pgpu_mesh_sizes(pgpu_ctx *ctx, int64_t *n_seeds, int64_t *n_hydro, int64_t *num_faces);

/* Replaces the device mesh by a host VMesh (for the drop-in hydro:: calls on a
 * mesh built elsewhere).  normal is num_faces x 3. */
int pgpu_upload_mesh(pgpu_ctx *ctx, int64_t n_seeds, int64_t n_hydro, int64_t num_faces, const double *volumes,
                     const uint64_t *face_counts, const uint64_t *face_ptr, const int32_t *neighbor,
                     const double *normal, const double *area, const uint64_t *ghost_ids);

/* --------------------------------------------------------------- hydro ---
 * Primitive state of the n_hydro cells (hydro::init, finite_volume_solver.cpp:8-31). */
int pgpu_set_prim(pgpu_ctx *ctx, const double *rho, const double *v, const double *E, int64_t n);
int pgpu_get_prim(pgpu_ctx *ctx, double *rho, double *v, double *E);

/* hydro::dt_CFL (src/hydro/finite_volume_solver.cpp:151-186) on the current mesh. */
int pgpu_dt_cfl(pgpu_ctx *ctx, double cfl, double *dt);

/* hydro::hydro_step (src/hydro/finite_volume_solver.cpp:43-123) on the current
 * mesh and primitives, in the context's flux_mode. */
int pgpu_hydro_step(pgpu_ctx *ctx, double dt);

/* No counterpart in the reference.  The CFL step of pgpu_dt_cfl (the same
 * per-cell formula and minimum, starting from 1e100) computed from the
 * caller's own DEVICE arrays -- rho[n], v[n * dim], E[n], volumes[n] of the n
 * hydro cells -- without a context and without allocating anything: no
 * cudaMalloc/cudaFree, no allocating library.  It is for callers that keep
 * their cell data in device memory they manage themselves and cannot let a
 * library allocate: a code whose device memory is reserved up front by its own
 * pool (a further cudaMalloc would fail or fragment it), or one whose time loop
 * cannot afford the device-wide synchronisation of cudaFree.
 *   Scratch: a fixed 128 KiB array in the library's device image, one partial
 * minimum per 1024 cells, hence n <= PGPU_DT_STATIC_MAX_CELLS; a larger n (or a
 * device ordinal >= PGPU_DT_STATIC_MAX_DEVICES) returns PGPU_ECAPACITY before
 * any device work.  Nothing in the scratch has to start at zero.  The first
 * call on each device looks up the scratch's address (cudaGetSymbolAddress)
 * with that device current; make that first call before capturing work on a
 * stream.  The address is kept per device ordinal for the life of the process
 * and belongs to that device's primary context (the runtime's): a caller that
 * drives the device through a context of its own, or that resets the device
 * after the first call, must not use this entry point.  Calls that overlap on
 * one device (other threads, other streams) share the scratch and race: order
 * them.
 *   Runs on the current device, on `stream` (a cudaStream_t; NULL = the legacy
 * default stream), and waits for it before writing *dt on the host. */
#define PGPU_DT_STATIC_MAX_CELLS 16777216
#define PGPU_DT_STATIC_MAX_DEVICES 64
int pgpu_dt_cfl_static(int dim, double gamma, double cfl, const double *rho, const double *v, const double *E,
                       const double *volumes, int64_t n, void *stream, double *dt);

/* -------------------------------------------------- initial conditions ---
 * Extension (the reference reads its initial conditions from HDF5 files written
 * by its create*.py scripts, src/io/input.cpp:121-309).  The benchmark
 * workloads' initial conditions generated on the device from a seed, bit for
 * bit the ones proteusgpu_b200/ics.py builds on the host (a counter-based
 * generator and fixed operation sequences for ln, exp, sin, cos and the
 * normals, so both sides compute the same doubles):
 *   PGPU_IC_SOD        2D Sod tube on a jittered n_side^2 lattice (rho 1 / 0.125,
 *                      P 1 / 0.1), split along the line through the centre with
 *                      normal (split_cos, split_sin);
 *   PGPU_IC_SEDOV      uniform points (dim 2 or 3), rho 1, P p0, and a blast of
 *                      e_blast over the 32 points nearest the centre;
 *   PGPU_IC_KH         2D Kelvin-Helmholtz shear on a jittered n_side^2 lattice
 *                      (density ratio rho_ratio, vx +-0.5, P 2.5, seeded vy);
 *   PGPU_IC_CLUSTERED  3D: a fraction frac_clumped of n points in n_clumps
 *                      Gaussian clumps (widths log-uniform in [0.005, 0.05]),
 *                      the rest uniform, and the blast as PGPU_IC_SEDOV. */
#define PGPU_IC_SOD 0
#define PGPU_IC_SEDOV 1
#define PGPU_IC_KH 2
#define PGPU_IC_CLUSTERED 3
typedef struct {
    int32_t kind;       /* PGPU_IC_* */
    int32_t dim;        /* 2, or 3 for PGPU_IC_SEDOV / PGPU_IC_CLUSTERED */
    int64_t n;          /* points (PGPU_IC_SEDOV, PGPU_IC_CLUSTERED) */
    int32_t n_side;     /* lattice side (PGPU_IC_SOD, PGPU_IC_KH): n_side^2 points */
    int32_t n_clumps;   /* PGPU_IC_CLUSTERED */
    uint64_t seed;
    double gamma, jitter, split_cos, split_sin, p0, e_blast, rho_ratio, frac_clumped;
} pgpu_ic_spec;

/* The initial condition of spec in host arrays (pos n x dim, rho, v n x dim, E,
 * deposit: energy per cell of the blast, zero elsewhere); any may be NULL. */
int pgpu_ic_generate(pgpu_ctx *ctx, const pgpu_ic_spec *spec, double *pos, double *rho, double *v, double *E,
                     double *deposit);
/* pgpu_sim_init from the initial condition of spec generated on the device: no
 * host arrays; the spec's dim must be the context's. */
int pgpu_sim_init_ic(pgpu_ctx *ctx, const pgpu_ic_spec *spec);
/* pgpu_batch_init from n_inst specs (gamma from each spec), each generated on the
 * device; buff and boundary per instance as pgpu_batch_init takes them. */
int pgpu_batch_init_ic(pgpu_ctx *ctx, int n_inst, const pgpu_ic_spec *specs, const double *buff,
                       const int *boundary);

/* -------------------------------------------------- moving-mesh stepping ---
 * Extension (the reference's time loop, src/main.cpp:50-63, keeps its mesh
 * fixed).  The simulation state is conserved mass, momentum and energy per
 * cell plus the generating points.  pgpu_sim_init builds the first mesh,
 * converts the primitives (and an optional per-cell energy deposit, e.g. a
 * Sedov blast) to conserved variables.  Host arrays: pos n x dim, v n x dim. */
int pgpu_sim_init(pgpu_ctx *ctx, const double *pos, const double *rho, const double *v, const double *E,
                  const double *deposit, int64_t n);

/* One full step on the device: ghosts, sort, KNN, clip + certificate,
 * extraction (hydro cells only), CFL dt (unless fixed_dt > 0), HLL fluxes with
 * the conserved update, and drift of the points with their cells' velocity.
 * dt_out (host, may be NULL) receives the step's dt; passing NULL keeps the
 * step free of device-to-host synchronisation. */
int pgpu_sim_step(pgpu_ctx *ctx, double cfl, double fixed_dt, double *dt_out);

/* Same step with the inputs given in, and the results read back to, host
 * memory: positions and conserved state are copied to the device before the
 * step and back after it (the end-to-end form of the call). */
int pgpu_sim_step_host(pgpu_ctx *ctx, double cfl, double fixed_dt, double *pos, double *mass, double *mom,
                       double *energy, double *dt_out);

/* Current simulation state (host arrays; any may be NULL). */
int pgpu_sim_get(pgpu_ctx *ctx, double *pos, double *mass, double *mom, double *energy);
int pgpu_sim_set(pgpu_ctx *ctx, const double *pos, const double *mass, const double *mom, const double *energy);

typedef struct {
    int64_t n_hydro, n_ext, num_faces;
    int64_t failed_cells;       /* hydro cells whose status is not SUCCESS */
    int64_t box_faces;          /* hydro faces on the bounding box (ghost layer too thin) */
    int64_t unpaired_faces;     /* faces whose reverse face was not found */
    int64_t knn_candidates;     /* distance evaluations in the last KNN (if counted) */
    double last_dt;
    double total_mass, total_energy, total_mom[3]; /* deterministic sums over hydro cells */
    int32_t cert_k_max;
    int32_t n_grid;
    int64_t refit_cells;        /* cells recomputed with k_fallback in the last step */
    int64_t uncertified_cells;  /* hydro cells still without a certificate after it */
    int64_t reclip_cells;       /* cells the FP32 clip handed to the FP64 clip in the last step */
    int64_t pruned_cells;       /* moving-mesh steps: hydro cells whose certificate needed more than the
                                   neighbour budget(s), clipped by walking the grid instead (extension) */
    int64_t walk_points, walk_boxes; /* that walk's work: points clipped, grid boxes visited */
    float clip_split_ms[3];     /* with timing on: the last build's clip stage as main clip (with the
                                   FP64 re-clip), fallback KNN + clip, grid walk */
    int32_t knn_redone;         /* queries of the last KNN stage searched a second time with exact keys
                                   (a tie of FP32-rounded distances in the packed-key search) */
} pgpu_stats;

/* Statistics of the last step (synchronises the stream). */
int pgpu_sim_stats(pgpu_ctx *ctx, pgpu_stats *out);

/* ---------------------------------------------------------- batches ---
 * Extension (the reference runs one simulation per process).  n_inst
 * independent moving-mesh simulations of uneven sizes advanced together: their
 * points are concatenated (instance b owns hydro ids [sum counts[<b], +counts[b])
 * of pos/rho/v/E/deposit, each in its own unit box) and every stage of a step is
 * one launch over all of them.  Each instance keeps its own ghost layer (buff),
 * gamma, boundary (PGPU_PERIODIC / PGPU_REFLECTIVE), grid and CFL time step, so
 * its mesh and state are the ones it gets when run alone.  Faces and neighbour
 * ids refer to the concatenated ids.  Needs flux_mode PGPU_FLUX_PHYSICAL; then
 * pgpu_sim_step / sim_get / sim_set / download_mesh work on the whole batch
 * (the step's dt_out is the smallest instance dt; pgpu_batch_dt gives each). */
int pgpu_batch_init(pgpu_ctx *ctx, int n_inst, const int64_t *counts, const double *buff, const double *gamma,
                    const int *boundary, const double *pos, const double *rho, const double *v, const double *E,
                    const double *deposit);
int pgpu_batch_dt(pgpu_ctx *ctx, double *dt_per_instance);

/* -------------------------------------------------------- autotuner ---
 * Extension.  Times mesh builds of the current simulation state (nothing
 * advances) and picks the coarse grid's mean points per bin (1.5, 2, 3, 4), the
 * KNN block size (1, 2, 4, 8 queries; or one thread per query for the queries whose
 * K is at most 32 or 64) and the clipping block size (1, 2, 4 cells; in 2D
 * also one thread per cell instead of one warp), one
 * after the other; the choice is cached for the process by (dim, log2 n, batch,
 * precision, learned K, k) and reused without timing.  The block sizes and the
 * thread-or-warp choices change no result.  The grid bin size changes nothing
 * either except in cells certified by the grid walk (beside dense clumps), whose
 * clipping order follows the grid: their areas and volumes move at rounding
 * level.  So the bin size is chosen once per (dim, log2 n, batch, k) and shared
 * by every form (plain or learned K, FP64 or FP32), which therefore build the
 * same meshes bit for bit. */
typedef struct {
    double ppb;
    int32_t knn_warps, clip_warps;
    int32_t clip_thread;         /* 2D: one thread per cell chosen over one warp per cell */
    int32_t knn_thread;          /* 0, 32 or 64: queries with K <= this are searched one per thread */
    float ms_default, ms_tuned;  /* ghosts + sort + KNN + clip of one build, before and after */
    int32_t from_cache;
} pgpu_tuning;
int pgpu_autotune(pgpu_ctx *ctx, pgpu_tuning *out);
/* Sets the launch shapes directly (ppb in [0.5, 64], knn_warps 1/2/4/8, clip_warps 1/2/4,
 * clip_thread 0/1, knn_thread 0/32/64; the timing fields are ignored). */
int pgpu_set_tuning(pgpu_ctx *ctx, const pgpu_tuning *t);

/* ------------------------------------------- learned neighbour budget ---
 * Extension (the reference uses one compile-time _K_ for every cell, Config.sh,
 * src/knn/knn.cpp:225-315).  When enabled, every mesh build of a moving-mesh
 * step gives each hydro cell its own K: an MLP (8 features -> 32 -> 32 -> 6,
 * GELU; BF16 weights, FP32 accumulation on the tensor cores) picks one of six
 * classes, {12,16,20,24,32,48} in 2D and {32,40,48,64,96,128} in 3D (capped at
 * the context's k).  A cell that does not certify within its K is computed
 * again at max(k, k_fallback), so the mesh equals the plain method's.  The
 * first train_steps steps run the plain method and train the MLP on the K its
 * certificate records (iters_per_step Adam iterations on 16384-cell batches);
 * the proposal is the smallest class whose predicted cumulative probability
 * reaches `quantile`.  train_steps 0 uses the current weights at once. */
int pgpu_kbudget_enable(pgpu_ctx *ctx, int train_steps, int iters_per_step, double quantile, uint64_t seed);
int pgpu_kbudget_classes(int dim, int *k_out6);

typedef struct {
    int32_t active;          /* proposals in use */
    int64_t steps_trained;
    double last_loss;        /* mean cross-entropy of the last training iteration */
    int64_t cells;           /* last step: cells that got a proposal */
    int64_t misses;          /* last step: proposals the certificate rejected */
    double mean_k;           /* last step: mean proposed K */
} pgpu_kbudget_info;
int pgpu_kbudget_stats(pgpu_ctx *ctx, pgpu_kbudget_info *out);

/* The MLP's FP32 master parameters, 1542 floats: W1[32][8], b1[32], W2[32][32],
 * b2[32], W3[6][32], b3[6] (row-major, out x in); get and/or set (NULL skips). */
int pgpu_kbudget_weights(pgpu_ctx *ctx, float *get, const float *set);

/* The device MLP on host arrays: feat n x 8 -> logits n x 6 and the proposed K
 * per row (either output may be NULL). */
int pgpu_mlp_forward(pgpu_ctx *ctx, const float *feat, int64_t n, float *logits, uint16_t *kq);

/* Gradient of the mean cross-entropy over n rows (labels = class indices 0-5)
 * at the current weights, in the parameter layout above, and the loss. */
int pgpu_mlp_grad(pgpu_ctx *ctx, const float *feat, const int32_t *labels, int64_t n, float *grad, float *loss);

/* Per-stage device times of the last step in milliseconds, measured with CUDA
 * events when timing is enabled: ghosts, sort, knn, clip, hydro. */
int pgpu_enable_timing(pgpu_ctx *ctx, int on);
int pgpu_stage_times(pgpu_ctx *ctx, float *ms5);

/* The CUDA stream of the context (a cudaStream_t), for callers that time or
 * order work around it. */
void *pgpu_stream(pgpu_ctx *ctx);

/* hydro::riemann_hll (src/hydro/riemann.cpp:7-45) for one face, on the host,
 * with the same arithmetic as the device kernels: L and R are (rho, vx, vy, vz, E)
 * (vz ignored in 2D), normal is the face normal as stored (3 doubles), flux
 * receives (rho, mx, my, mz, E) in the lab frame. */
int pgpu_riemann_hll(int dim, double gamma, const double *L, const double *R, const double *normal, double *flux);

/* Number of kernels launched by this library in this process so far (diagnostics). */
int64_t pgpu_launch_count(void);

/* Diagnostics, no reference counterpart: runs a dependent-chain FP64 FMA
 * kernel on the device for about `ms` milliseconds and returns the achieved
 * FP64 rate in TFLOP/s (the FP64 pipe peak that the KNN and clipping kernels
 * are measured against). */
int pgpu_fp64_peak(int device, float ms, double *tflops);
/* The same with FP32 FMAs (the FP32 pipe peak of the FP32 clipping kernel). */
int pgpu_fp32_peak(int device, float ms, double *tflops);

#ifdef __cplusplus
}
#endif
#endif /* PROTEUS_GPU_H */
