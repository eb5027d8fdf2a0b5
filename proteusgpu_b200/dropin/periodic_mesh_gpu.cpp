// Drop-in replacement for the reference's src/voronoi/periodic_mesh.cpp.
//
// voronoi::compute_periodic_mesh (periodic_mesh.h:22) keeps its signature and
// result: the VMesh of all hydro and ghost cells in input order, seeds, volumes
// and areas scaled back to [-buff, 1 + buff], n_hydro and ghost_ids set.  The
// ghost layer, unit-box scaling, KNN, clipping and extraction all run on the
// GPU in one call of the C ABI.
#include "periodic_mesh.h"
#include "pgpu_dropin.h"

namespace voronoi {

// The region test and ghost append of periodic_mesh.h:18-20, kept for callers
// that use them directly; the device path does not call them.
inline bool is_in(POINT_TYPE pt, double xa, double xb, double ya, double yb, double za, double zb) {
#ifdef dim_2D
    (void)za;
    (void)zb;
    return pt.x > xa && pt.x < xb && pt.y > ya && pt.y < yb;
#else
    return pt.x > xa && pt.x < xb && pt.y > ya && pt.y < yb && pt.z > za && pt.z < zb;
#endif
}

inline void add_ghost(POINT_TYPE* pts, hsize_t index, hsize_t* n_ghosts, const hsize_t* n_hydro,
                      hsize_t* original_ids, double shift_x, double shift_y, double shift_z) {
    POINT_TYPE g = pts[index];
    g.x += shift_x;
    g.y += shift_y;
#ifdef dim_3D
    g.z += shift_z;
#else
    (void)shift_z;
#endif
    pts[*n_hydro + *n_ghosts] = g;
    original_ids[*n_ghosts] = index;
    (*n_ghosts)++;
}

VMesh* compute_periodic_mesh(POINT_TYPE* pts_data, hsize_t num_points) {
    pgpu_ctx* c = pgpu_dropin::context();
    int64_t ns = 0, nf = 0;
    int rc = pgpu_periodic_mesh(c, (const double*)pts_data, (int64_t)num_points, &ns, &nf);
    if (rc) pgpu_dropin::die("voronoi::compute_periodic_mesh", rc);
    pgpu_dropin::invalidate_mesh();
    return pgpu_dropin::download_vmesh(c, true, nullptr);
}

}  // namespace voronoi
