// Drop-in replacement for the reference's src/voronoi/voronoi.cpp (and
// src/voronoi/cell.cpp, whose functions only voronoi.cpp called).
//
// Keeps every entry point voronoi.h declares (src/voronoi/voronoi.h:43-84) and
// the VMesh layout (voronoi.h:22-41).  The cells are computed on the GPU through
// the C ABI: Ray et al. clipping with the security-radius certificate and the
// extraction of faces, areas and volumes.  Neighbour lists, face order and the
// per-cell Status codes equal the reference's; see include/proteus_gpu.h.
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <vector>

#include "pgpu_dropin.h"
#include "voronoi.h"

namespace pgpu_dropin {

VMesh* download_vmesh(pgpu_ctx* c, bool periodic, std::vector<int>* status) {
    int64_t n = 0, nh = 0, F = 0;
    pgpu_mesh_sizes(c, &n, &nh, &F);
    VMesh* m = voronoi::allocate_vmesh((hsize_t)n, (hsize_t)(F > 0 ? F : 1));
    std::vector<double> seeds(3 * (size_t)n + 3), normal(3 * (size_t)F + 3);
    std::vector<int32_t> st((size_t)n + 1);
    std::vector<uint64_t> gid((size_t)(n - nh) + 1);
    int rc = pgpu_download_mesh(c, seeds.data(), m->volumes, (uint64_t*)m->face_counts, (uint64_t*)m->face_ptr,
                                m->neighbor_cell, normal.data(), m->face_area, gid.data(), st.data(), nullptr,
                                nullptr);
    if (rc) die("pgpu_download_mesh", rc);
    for (int64_t i = 0; i < n; i++) {
        m->cell_ids[i] = (hsize_t)i;
        m->seeds[i].x = seeds[3 * i];
        m->seeds[i].y = seeds[3 * i + 1];
        m->seeds[i].z = seeds[3 * i + 2];
    }
    for (int64_t f = 0; f < F; f++) {
        m->face_normal[f].x = normal[3 * f];
        m->face_normal[f].y = normal[3 * f + 1];
        m->face_normal[f].z = normal[3 * f + 2];
    }
    m->num_faces = (hsize_t)F;
    if (periodic) {
        m->n_hydro = (hsize_t)nh;
        m->ghost_ids = (hsize_t*)malloc(((size_t)(n - nh) + 1) * sizeof(hsize_t));
        for (int64_t g = 0; g < n - nh; g++) m->ghost_ids[g] = (hsize_t)gid[g];
    }
    if (status) status->assign(st.begin(), st.begin() + n);
    return m;
}

}  // namespace pgpu_dropin

namespace voronoi {

VMesh* compute_mesh(POINT_TYPE* pts_data, int num_points) {
    pgpu_ctx* c = pgpu_dropin::context();
    int64_t nf = 0;
    int rc = pgpu_compute_mesh(c, (const double*)pts_data, num_points, &nf);
    if (rc) pgpu_dropin::die("voronoi::compute_mesh", rc);
    pgpu_dropin::invalidate_mesh();
    return pgpu_dropin::download_vmesh(c, false, nullptr);
}

// Cells of the knn problem's (grid-sorted) points; the mesh is in that sorted
// order, with neighbour ids in it, as the reference's compute_cells leaves it
// before unpermute_vmesh (voronoi.cpp:68-111).
void compute_cells(int N_seedpts, knn_problem* knn, std::vector<Status>& stat, VMesh* mesh) {
    pgpu_ctx* c = pgpu_dropin::context();
    int64_t nf = 0;
    int rc = pgpu_compute_mesh(c, (const double*)knn->d_stored_points, N_seedpts, &nf);
    if (rc) pgpu_dropin::die("voronoi::compute_cells", rc);
    pgpu_dropin::invalidate_mesh();
    std::vector<int> st;
    VMesh* m = pgpu_dropin::download_vmesh(c, false, &st);
    // move the arrays into the caller's mesh (allocated by allocate_vmesh)
    std::swap(mesh->cell_ids, m->cell_ids);
    std::swap(mesh->seeds, m->seeds);
    std::swap(mesh->volumes, m->volumes);
    std::swap(mesh->face_counts, m->face_counts);
    std::swap(mesh->face_ptr, m->face_ptr);
    std::swap(mesh->neighbor_cell, m->neighbor_cell);
    std::swap(mesh->face_normal, m->face_normal);
    std::swap(mesh->face_area, m->face_area);
    mesh->num_faces = m->num_faces;
    free_vmesh(m);
    for (int i = 0; i < N_seedpts && i < (int)stat.size(); i++) stat[i] = (Status)st[i];
    for (int i = 0; i < N_seedpts && i < (int)stat.size(); i++)
        if (stat[i] != success) std::cout << "VORONOI: cell " << i << " failed with status: " << stat[i] << std::endl;
}

VMesh* allocate_vmesh(hsize_t n_seeds, hsize_t initial_face_capacity) {
    VMesh* m = (VMesh*)calloc(1, sizeof(VMesh));
    m->n_seeds = n_seeds;
    m->cell_ids = (hsize_t*)calloc(n_seeds + 1, sizeof(hsize_t));
    m->seeds = (double3*)calloc(n_seeds + 1, sizeof(double3));
    m->volumes = (double*)calloc(n_seeds + 1, sizeof(double));
    m->face_counts = (hsize_t*)calloc(n_seeds + 1, sizeof(hsize_t));
    m->face_ptr = (hsize_t*)calloc(n_seeds + 1, sizeof(hsize_t));
    m->neighbor_cell = (int*)malloc((initial_face_capacity + 1) * sizeof(int));
    m->face_normal = (double3*)malloc((initial_face_capacity + 1) * sizeof(double3));
    m->face_area = (double*)malloc((initial_face_capacity + 1) * sizeof(double));
#ifdef DEBUG_MODE
    m->edge_coords = nullptr;  // face vertex coordinates are not produced by the device path
    m->edge_coords_offsets = (hsize_t*)calloc(initial_face_capacity + 1, sizeof(hsize_t));
    m->num_edge_coord_verts = 0;
#endif
    return m;
}

void free_vmesh(VMesh* m) {
    if (!m) return;
    pgpu_dropin::MeshKey& k = pgpu_dropin::device_mesh_key();
    if (k.mesh == m) pgpu_dropin::invalidate_mesh();
    free(m->cell_ids);
    free(m->seeds);
    free(m->volumes);
    free(m->face_counts);
    free(m->face_ptr);
    free(m->neighbor_cell);
    free(m->face_normal);
    free(m->face_area);
#ifdef DEBUG_MODE
    free(m->edge_coords);
    free(m->edge_coords_offsets);
#endif
    free(m->ghost_ids);
    free(m);
}

// Reorders a mesh whose cells and neighbour ids are in sorted order into input
// order (the contract of voronoi.cpp:212-333); faces stay contiguous per cell.
void unpermute_vmesh(VMesh* m, const unsigned int* sorted_to_original) {
    const hsize_t n = m->n_seeds;
    if (n == 0 || !sorted_to_original) return;
    std::vector<long long> from(n, -1);  // original id -> sorted id
    for (hsize_t s = 0; s < n; s++)
        if (sorted_to_original[s] < n) from[sorted_to_original[s]] = (long long)s;
    hsize_t* ids = (hsize_t*)malloc((n + 1) * sizeof(hsize_t));
    double3* seeds = (double3*)malloc((n + 1) * sizeof(double3));
    double* vol = (double*)malloc((n + 1) * sizeof(double));
    hsize_t* cnt = (hsize_t*)malloc((n + 1) * sizeof(hsize_t));
    hsize_t* ptr = (hsize_t*)malloc((n + 1) * sizeof(hsize_t));
    int* nb = (int*)malloc((m->num_faces + 1) * sizeof(int));
    double3* nrm = (double3*)malloc((m->num_faces + 1) * sizeof(double3));
    double* ar = (double*)malloc((m->num_faces + 1) * sizeof(double));
    hsize_t at = 0;
    for (hsize_t o = 0; o < n; o++) {
        const long long s = from[o];
        if (s < 0) continue;
        ids[o] = o;
        seeds[o] = m->seeds[s];
        vol[o] = m->volumes[s];
        cnt[o] = m->face_counts[s];
        ptr[o] = at;
        for (hsize_t q = 0; q < m->face_counts[s]; q++, at++) {
            const hsize_t f = m->face_ptr[s] + q;
            const int v = m->neighbor_cell[f];
            nb[at] = (v >= 0 && (hsize_t)v < n) ? (int)sorted_to_original[v] : v;
            nrm[at] = m->face_normal[f];
            ar[at] = m->face_area[f];
        }
    }
    free(m->cell_ids);
    free(m->seeds);
    free(m->volumes);
    free(m->face_counts);
    free(m->face_ptr);
    free(m->neighbor_cell);
    free(m->face_normal);
    free(m->face_area);
    m->cell_ids = ids;
    m->seeds = seeds;
    m->volumes = vol;
    m->face_counts = cnt;
    m->face_ptr = ptr;
    m->neighbor_cell = nb;
    m->face_normal = nrm;
    m->face_area = ar;
}

#ifdef USE_HDF5
// VMesh -> MeshCellData for the HDF5 writer (the contract of voronoi.cpp:339-421):
// hydro cells only, flat seed and normal arrays of DIMENSION components.
void vmesh_to_meshdata(VMesh* m, MeshCellData& d) {
    const int n = (int)m->n_hydro;
    d.header.dimension = DIMENSION;
    d.header.extent = 1.0;
    d.header.n = n;
    d.header.k = _K_;
    d.header.nmax = _MAX_P_;
    d.header.seed = 0;
    d.seeds_dims = {(hsize_t)n, (hsize_t)DIMENSION};
    d.cell_ids.resize(n);
    d.seeds.resize((size_t)n * DIMENSION);
    d.volumes.resize(n);
    d.face_counts.resize(n);
    for (int i = 0; i < n; i++) {
        d.cell_ids[i] = (int)m->cell_ids[i];
        const double c[3] = {m->seeds[i].x, m->seeds[i].y, m->seeds[i].z};
        for (int a = 0; a < DIMENSION; a++) d.seeds[(size_t)i * DIMENSION + a] = c[a];
        d.volumes[i] = m->volumes[i];
        d.face_counts[i] = (int)m->face_counts[i];
    }
    const hsize_t F = m->num_faces;
    d.faces.neighbor_cell.resize(F);
    d.faces.normal.resize(F * DIMENSION);
    d.faces.area.resize(F);
    d.faces.normal_dims = {F, (hsize_t)DIMENSION};
    for (hsize_t f = 0; f < F; f++) {
        d.faces.neighbor_cell[f] = m->neighbor_cell[f];
        const double c[3] = {m->face_normal[f].x, m->face_normal[f].y, m->face_normal[f].z};
        for (int a = 0; a < DIMENSION; a++) d.faces.normal[f * DIMENSION + a] = c[a];
        d.faces.area[f] = m->face_area[f];
    }
}
#endif

}  // namespace voronoi
