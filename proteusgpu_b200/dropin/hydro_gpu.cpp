// Drop-in replacement for the reference's src/hydro/finite_volume_solver.cpp
// and src/hydro/riemann.cpp.
//
// Keeps every entry point finite_volume_solver.h (:18-27) and riemann.h (:24-31)
// declare and the primvars layout (src/global/allvars.h:203-207).  dt_CFL and
// hydro_step run on the GPU through the C ABI with the reference's arithmetic
// (stored normal, own face area: the same results bit for bit on the same mesh).
// The host VMesh is uploaded on the first call that sees it and kept on the
// device until another mesh is passed or freed; the primitives are copied in
// before and out after every call, because the caller owns them on the host.
#include <cmath>
#include <cstdlib>
#include <iostream>

#include "finite_volume_solver.h"
#include "pgpu_dropin.h"
#include "riemann.h"

namespace {

void sync_mesh(pgpu_ctx* c, const VMesh* m) {
    pgpu_dropin::MeshKey& k = pgpu_dropin::device_mesh_key();
    if (k.mesh == m && k.volumes == m->volumes && k.num_faces == m->num_faces && k.n_seeds == m->n_seeds) return;
    int rc = pgpu_upload_mesh(c, (int64_t)m->n_seeds, (int64_t)m->n_hydro, (int64_t)m->num_faces, m->volumes,
                              (const uint64_t*)m->face_counts, (const uint64_t*)m->face_ptr, m->neighbor_cell,
                              (const double*)m->face_normal, m->face_area, (const uint64_t*)m->ghost_ids);
    if (rc) pgpu_dropin::die("hydro: mesh upload", rc);
    k.mesh = m;
    k.volumes = m->volumes;
    k.num_faces = m->num_faces;
    k.n_seeds = m->n_seeds;
}

void put_prim(pgpu_ctx* c, const VMesh* m, const primvars* pv) {
    int rc = pgpu_set_prim(c, pv->rho, (const double*)pv->v, pv->E, (int64_t)m->n_hydro);
    if (rc) pgpu_dropin::die("hydro: primitives upload", rc);
}

}  // namespace

namespace hydro {

primvars* init(int n_hydro) {
    primvars* pv = new primvars();
    pv->rho = (double*)malloc((n_hydro + 1) * sizeof(double));
    pv->v = (POINT_TYPE*)malloc((n_hydro + 1) * sizeof(POINT_TYPE));
    pv->E = (double*)malloc((n_hydro + 1) * sizeof(double));
    for (int i = 0; i < n_hydro; i++) {
        pv->rho[i] = icData.rho[i];
        pv->E[i] = icData.Energy[i];
        pv->v[i].x = icData.vel[(size_t)DIMENSION * i];
        pv->v[i].y = icData.vel[(size_t)DIMENSION * i + 1];
#ifdef dim_3D
        pv->v[i].z = icData.vel[(size_t)DIMENSION * i + 2];
#endif
    }
    std::cout << "HYDRO: Initialized primitive variables for " << n_hydro << " particles" << std::endl;
    return pv;
}

void free_prim(primvars** pv) {
    free((*pv)->rho);
    free((*pv)->v);
    free((*pv)->E);
    delete *pv;
    *pv = NULL;
}

void hydro_step(double dt, const VMesh* mesh, primvars* pv) {
    pgpu_ctx* c = pgpu_dropin::context();
    sync_mesh(c, mesh);
    put_prim(c, mesh, pv);
    int rc = pgpu_hydro_step(c, dt);
    if (rc) pgpu_dropin::die("hydro::hydro_step", rc);
    rc = pgpu_get_prim(c, pv->rho, (double*)pv->v, pv->E);
    if (rc) pgpu_dropin::die("hydro::hydro_step", rc);
}

double dt_CFL(double CFL, const VMesh* mesh, const primvars* pv) {
    pgpu_ctx* c = pgpu_dropin::context();
    sync_mesh(c, mesh);
    put_prim(c, mesh, pv);
    double dt = 0.0;
    int rc = pgpu_dt_cfl(c, CFL, &dt);
    if (rc) pgpu_dropin::die("hydro::dt_CFL", rc);
    return dt;
}

// State on the far side of face j of cell i; ghost neighbours map to the hydro
// cell they copy (finite_volume_solver.h:23).
prim get_state_j(hsize_t i, int j, const VMesh* mesh, primvars* pv) {
    hsize_t id = (hsize_t)mesh->neighbor_cell[mesh->face_ptr[i] + j];
    if (id >= mesh->n_hydro) id = mesh->ghost_ids[id - mesh->n_hydro];
    prim s;
    s.rho = pv->rho[id];
    s.v = pv->v[id];
    s.E = pv->E[id];
    return s;
}

// ---- riemann.h: one face on the host, with the device's HLL arithmetic

prim riemann_hll(hsize_t i, hsize_t j, prim st_l, prim st_r, const VMesh* mesh) {
    const double3 n = mesh->face_normal[mesh->face_ptr[i] + j];
    double L[5] = {st_l.rho, st_l.v.x, st_l.v.y, 0.0, st_l.E}, R[5] = {st_r.rho, st_r.v.x, st_r.v.y, 0.0, st_r.E};
#ifdef dim_3D
    L[3] = st_l.v.z;
    R[3] = st_r.v.z;
#endif
    const double nn[3] = {n.x, n.y, n.z};
    double F[5];
    if (pgpu_riemann_hll(DIMENSION, _gamma_, L, R, nn, F)) pgpu_dropin::die("hydro::riemann_hll", PGPU_EINVAL);
    prim f;
    f.rho = F[0];
    f.v.x = F[1];
    f.v.y = F[2];
#ifdef dim_3D
    f.v.z = F[3];
#endif
    f.E = F[4];
    return f;
}

// Orthonormal face frame: n, a unit vector m orthogonal to n in the xy-plane
// (x axis if n is along z), p = n x m.
geom compute_geom(double3 normal) {
    geom g;
    const double nn = std::sqrt(normal.x * normal.x + normal.y * normal.y + normal.z * normal.z);
    g.n = {normal.x / nn, normal.y / nn, normal.z / nn};
    double3 m = (g.n.x != 0.0 || g.n.y != 0.0) ? double3{-g.n.y, g.n.x, 0.0} : double3{1.0, 0.0, 0.0};
    const double mm = std::sqrt(m.x * m.x + m.y * m.y + m.z * m.z);
    g.m = {m.x / mm, m.y / mm, m.z / mm};
    g.p = {g.n.y * g.m.z - g.n.z * g.m.y, g.n.z * g.m.x - g.n.x * g.m.z, g.n.x * g.m.y - g.n.y * g.m.x};
    return g;
}

void rotate_to_face(prim* s, geom* g) {
    const double a = s->v.x, b = s->v.y;
#ifdef dim_2D
    s->v.x = a * g->n.x + b * g->n.y;
    s->v.y = a * g->m.x + b * g->m.y;
#else
    const double c = s->v.z;
    s->v.x = a * g->n.x + b * g->n.y + c * g->n.z;
    s->v.y = a * g->m.x + b * g->m.y + c * g->m.z;
    s->v.z = a * g->p.x + b * g->p.y + c * g->p.z;
#endif
}

void rotate_from_face(prim* s, geom* g) {
    const double a = s->v.x, b = s->v.y;
#ifdef dim_2D
    s->v.x = a * g->n.x + b * g->m.x;
    s->v.y = a * g->n.y + b * g->m.y;
#else
    const double c = s->v.z;
    s->v.x = a * g->n.x + b * g->m.x + c * g->p.x;
    s->v.y = a * g->n.y + b * g->m.y + c * g->p.y;
    s->v.z = a * g->n.z + b * g->m.z + c * g->p.z;
#endif
}

// Ideal-gas pressure from the total energy density.
double get_P_ideal_gas(prim* s) {
#ifdef dim_2D
    const double v2 = s->v.x * s->v.x + s->v.y * s->v.y;
#else
    const double v2 = s->v.x * s->v.x + s->v.y * s->v.y + s->v.z * s->v.z;
#endif
    return (_gamma_ - 1) * (s->E - (0.5 * s->rho * v2));
}

// Euler flux along the face-frame x axis.
prim get_flux(prim* s) {
    const double P = get_P_ideal_gas(s);
    prim f;
    f.rho = s->rho * s->v.x;
    f.v.x = s->rho * s->v.x * s->v.x + P;
    f.v.y = s->rho * s->v.x * s->v.y;
#ifdef dim_3D
    f.v.z = s->rho * s->v.x * s->v.z;
#endif
    f.E = (s->E + P) * s->v.x;
    return f;
}

}  // namespace hydro
