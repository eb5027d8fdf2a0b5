// Test-infrastructure driver for the reference build (oracle/_ref).
//
// This file is ours; it is compiled together with the reference's own
// translation units (src/global/allvars.cpp, src/knn/knn.cpp,
// src/voronoi/{voronoi,cell,periodic_mesh}.cpp,
// src/hydro/{finite_volume_solver,riemann}.cpp), read in place from the
// reference tree by oracle/Makefile.  It exposes a small extern "C" surface so
// that the Python tests can run the reference's mesh-and-flux path on seeded
// inputs held in memory (the reference itself only reads HDF5 files).
//
// Nothing here re-implements reference behaviour: every entry point forwards to
// the reference's own functions.  The one exception is ref_compute_mesh, which
// repeats the call sequence of voronoi::compute_mesh (voronoi.cpp:17-64) so
// that the per-cell Status vector it builds can be returned to the caller.
//
// The product never links this: only tests, smoke() and bench.py's CPU arms do.

#include "global/allvars.h"
#include "io/input.h"
#include "io/output.h"
#include "knn/knn.h"
#include "voronoi/voronoi.h"
#include "voronoi/periodic_mesh.h"
#include "hydro/finite_volume_solver.h"

#include <climits>
#include <cmath>
#include <cstdio>
#include <fcntl.h>
#include <iostream>
#include <unistd.h>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

// The reference defines these constructors in io/input.cpp and io/output.cpp,
// which need libhdf5; the hot path never calls any other member.
InputHandler::InputHandler(const std::string& filename) : paramFilePath(filename) {}
OutputHandler::OutputHandler(const std::string& outputDir) : outputDirectory(outputDir) {}

#define REF_API extern "C" __attribute__((visibility("default")))

namespace {

int g_quiet = 1;

// Silences the reference's progress printing on stdout for one call.
struct QuietStdout {
    int saved = -1;
    QuietStdout() {
        if (!g_quiet) return;
        std::cout.flush();
        fflush(stdout);
        saved = dup(1);
        int fd = open("/dev/null", O_WRONLY);
        if (fd >= 0) {
            dup2(fd, 1);
            close(fd);
        }
    }
    ~QuietStdout() {
        if (saved < 0) return;
        std::cout.flush();
        fflush(stdout);
        dup2(saved, 1);
        close(saved);
    }
};

// Same expression as knn::init (knn.cpp:22).
int n_grid_for(long n) {
    return std::max(1, (int)round(pow(n / 3.1f, 1.0f / (float)DIMENSION)));
}

}  // namespace

REF_API int ref_dim(void) { return DIMENSION; }
REF_API int ref_k(void) { return _K_; }
REF_API int ref_max_p(void) { return _MAX_P_; }
REF_API int ref_max_t(void) { return _MAX_T_; }

// Sets the reference's globals `buff` and `_gamma_` (allvars.cpp:13-14), the
// stdout silencing and the OpenMP thread count (0 keeps the default).
REF_API void ref_set_params(double buffer, double gamma, int quiet, int nthreads) {
    buff = buffer;
    _gamma_ = gamma;
    g_quiet = quiet;
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
}

REF_API int ref_n_grid(long n) { return n_grid_for(n); }

REF_API int ref_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

// voronoi::compute_periodic_mesh (periodic_mesh.cpp:44-184) on n points in
// [0,1]^D.  Returns the VMesh (all hydro + ghost cells, input order) or NULL
// when the reference would exit because its KNN grid is below 16^D
// (knn.cpp:32-36).
REF_API void* ref_periodic_mesh(const double* pts, long n) {
    if (n_grid_for(n) < 16) return nullptr;
    QuietStdout q;
    return voronoi::compute_periodic_mesh((POINT_TYPE*)pts, (hsize_t)n);
}

// The call sequence of voronoi::compute_mesh (voronoi.cpp:17-64) on n points
// already in [0,1]^D, additionally returning each cell's Status in input
// order.  NULL when the grid would be below 16^D.
REF_API void* ref_compute_mesh(const double* pts, long n, int* status_out) {
    if (n_grid_for(n) < 16) return nullptr;
    QuietStdout q;
    knn_problem* knn = knn::init((POINT_TYPE*)pts, (int)n);
    knn::solve(knn);
    std::vector<Status> stat(n, security_radius_not_reached);
    VMesh* mesh = voronoi::allocate_vmesh((hsize_t)n, (hsize_t)n * 16);
    voronoi::compute_cells((int)n, knn, stat, mesh);
    unsigned int* perm = knn::get_permutation(knn);
    voronoi::unpermute_vmesh(mesh, perm);
    if (status_out)
        for (long s = 0; s < n; s++) status_out[perm[s]] = (int)stat[s];
    free(perm);
    knn::knn_free(&knn);
    return mesh;
}

REF_API void ref_mesh_sizes(void* m, long* n_seeds, long* n_hydro, long* num_faces) {
    VMesh* mesh = (VMesh*)m;
    *n_seeds = (long)mesh->n_seeds;
    *n_hydro = (long)mesh->n_hydro;
    *num_faces = (long)mesh->num_faces;
}

// Copies the VMesh arrays out (voronoi.h:22-41).  seeds and normals are
// double3 even in 2D; any output pointer may be NULL.
REF_API void ref_mesh_copy(void* m, double* seeds, double* volumes, long* face_counts,
                           long* face_ptr, int* neighbor, double* normal, double* area,
                           long* ghost_ids) {
    VMesh* mesh = (VMesh*)m;
    const long n = (long)mesh->n_seeds, F = (long)mesh->num_faces;
    for (long i = 0; i < n; i++) {
        if (seeds) {
            seeds[3 * i] = mesh->seeds[i].x;
            seeds[3 * i + 1] = mesh->seeds[i].y;
            seeds[3 * i + 2] = mesh->seeds[i].z;
        }
        if (volumes) volumes[i] = mesh->volumes[i];
        if (face_counts) face_counts[i] = (long)mesh->face_counts[i];
        if (face_ptr) face_ptr[i] = (long)mesh->face_ptr[i];
    }
    for (long f = 0; f < F; f++) {
        if (neighbor) neighbor[f] = mesh->neighbor_cell[f];
        if (normal) {
            normal[3 * f] = mesh->face_normal[f].x;
            normal[3 * f + 1] = mesh->face_normal[f].y;
            normal[3 * f + 2] = mesh->face_normal[f].z;
        }
        if (area) area[f] = mesh->face_area[f];
    }
    if (ghost_ids && mesh->ghost_ids) {
        long ng = n - (long)mesh->n_hydro;
        for (long g = 0; g < ng; g++) ghost_ids[g] = (long)mesh->ghost_ids[g];
    }
}

// Builds a VMesh from caller arrays (for running the reference hydro on a mesh
// produced elsewhere).  Arrays are copied; free with ref_mesh_free.
REF_API void* ref_mesh_wrap(long n_seeds, long n_hydro, long num_faces, const double* volumes,
                            const long* face_counts, const long* face_ptr, const int* neighbor,
                            const double* normal, const double* area, const long* ghost_ids) {
    VMesh* mesh = voronoi::allocate_vmesh((hsize_t)n_seeds, (hsize_t)(num_faces > 0 ? num_faces : 1));
    mesh->num_faces = (hsize_t)num_faces;
    mesh->n_hydro = (hsize_t)n_hydro;
    for (long i = 0; i < n_seeds; i++) {
        mesh->cell_ids[i] = (hsize_t)i;
        mesh->volumes[i] = volumes[i];
        mesh->face_counts[i] = (hsize_t)face_counts[i];
        mesh->face_ptr[i] = (hsize_t)face_ptr[i];
    }
    for (long f = 0; f < num_faces; f++) {
        mesh->neighbor_cell[f] = neighbor[f];
        mesh->face_normal[f].x = normal[3 * f];
        mesh->face_normal[f].y = normal[3 * f + 1];
        mesh->face_normal[f].z = normal[3 * f + 2];
        mesh->face_area[f] = area[f];
    }
    long ng = n_seeds - n_hydro;
    mesh->ghost_ids = (hsize_t*)malloc((ng > 0 ? ng : 1) * sizeof(hsize_t));
    for (long g = 0; g < ng; g++) mesh->ghost_ids[g] = (hsize_t)ghost_ids[g];
    return mesh;
}

REF_API void ref_mesh_free(void* m) { voronoi::free_vmesh((VMesh*)m); }

// Sets the VMesh seeds (n_seeds x 3 doubles) of a mesh made by ref_mesh_wrap.
REF_API void ref_mesh_set_seeds(void* m, const double* seeds) {
    VMesh* mesh = (VMesh*)m;
    for (hsize_t i = 0; i < mesh->n_seeds; i++) {
        mesh->seeds[i].x = seeds[3 * i];
        mesh->seeds[i].y = seeds[3 * i + 1];
        mesh->seeds[i].z = seeds[3 * i + 2];
    }
}

// voronoi::vmesh_to_meshdata (voronoi.cpp:339-421 in the reference build; the
// drop-in's own definition where this driver is linked with the drop-in units)
// and every field of the MeshCellData it fills (io/output.h:14-48): header as
// (dimension, extent, n, k, nmax, seed, store_edge_coords), the dims arrays as
// (seeds rows, seeds cols, normal rows, normal cols), then the vectors.  The
// caller sizes cell_ids / volumes / face_counts by n_hydro, seeds by
// n_hydro x D, neighbor / area by num_faces and normal by num_faces x D.
// Returns the number of faces in the MeshCellData.
REF_API long ref_meshdata(void* m, double* header7, long* dims4, int* cell_ids, double* seeds, double* volumes,
                          int* face_counts, int* neighbor, double* normal, double* area) {
    MeshCellData d;
    voronoi::vmesh_to_meshdata((VMesh*)m, d);
    header7[0] = d.header.dimension;
    header7[1] = d.header.extent;
    header7[2] = d.header.n;
    header7[3] = d.header.k;
    header7[4] = d.header.nmax;
    header7[5] = d.header.seed;
    header7[6] = d.header.store_edge_coords ? 1.0 : 0.0;
    dims4[0] = d.seeds_dims.size() > 0 ? (long)d.seeds_dims[0] : -1;
    dims4[1] = d.seeds_dims.size() > 1 ? (long)d.seeds_dims[1] : -1;
    dims4[2] = d.faces.normal_dims.size() > 0 ? (long)d.faces.normal_dims[0] : -1;
    dims4[3] = d.faces.normal_dims.size() > 1 ? (long)d.faces.normal_dims[1] : -1;
    for (size_t i = 0; i < d.cell_ids.size(); i++) cell_ids[i] = d.cell_ids[i];
    for (size_t i = 0; i < d.seeds.size(); i++) seeds[i] = d.seeds[i];
    for (size_t i = 0; i < d.volumes.size(); i++) volumes[i] = d.volumes[i];
    for (size_t i = 0; i < d.face_counts.size(); i++) face_counts[i] = d.face_counts[i];
    for (size_t f = 0; f < d.faces.neighbor_cell.size(); f++) neighbor[f] = d.faces.neighbor_cell[f];
    for (size_t f = 0; f < d.faces.normal.size(); f++) normal[f] = d.faces.normal[f];
    for (size_t f = 0; f < d.faces.area.size(); f++) area[f] = d.faces.area[f];
    return (long)d.faces.area.size();
}

// knn::init + knn::solve (knn.cpp:16-234) on n points in [0,1]^D.  Writes the
// K neighbour lists translated to input ids (query in input order, UINT_MAX
// kept for unfilled slots).  Returns N_grid, or -1 when it is below 16.
REF_API int ref_knn(const double* pts, long n, unsigned* knn_out) {
    if (n_grid_for(n) < 16) return -1;
    QuietStdout q;
    knn_problem* knn = knn::init((POINT_TYPE*)pts, (int)n);
    knn::solve(knn);
    unsigned* lists = knn::get_knearest(knn);
    unsigned* perm = knn::get_permutation(knn);
    for (long s = 0; s < n; s++) {
        unsigned qi = perm[s];
        for (int j = 0; j < _K_; j++) {
            unsigned v = lists[s * _K_ + j];
            knn_out[(long)qi * _K_ + j] = (v == UINT_MAX) ? UINT_MAX : perm[v];
        }
    }
    int ng = knn->N_grid;
    free(lists);
    free(perm);
    knn::knn_free(&knn);
    return ng;
}

// hydro::dt_CFL (finite_volume_solver.cpp:151-186) on caller-held primitives.
REF_API double ref_dt_cfl(void* m, double cfl, double* rho, double* v, double* E) {
    primvars pv;
    pv.rho = rho;
    pv.v = (POINT_TYPE*)v;
    pv.E = E;
    return hydro::dt_CFL(cfl, (const VMesh*)m, &pv);
}

// hydro::hydro_step (finite_volume_solver.cpp:43-123), in place on caller-held
// primitives of the mesh's n_hydro cells.
REF_API void ref_hydro_step(void* m, double dt, double* rho, double* v, double* E) {
    primvars pv;
    pv.rho = rho;
    pv.v = (POINT_TYPE*)v;
    pv.E = E;
    hydro::hydro_step(dt, (const VMesh*)m, &pv);
}
