// Process-wide device context of the drop-in translation units.
#include "pgpu_dropin.h"

#include <cstdio>
#include <cstdlib>

#include "global/allvars.h"

namespace pgpu_dropin {
namespace {
pgpu_ctx* g_ctx = nullptr;
double g_buff = -1.0, g_gamma = -1.0;
MeshKey g_key;
}  // namespace

pgpu_ctx* context() {
    if (g_ctx && g_buff == buff && g_gamma == _gamma_) return g_ctx;
    if (g_ctx) pgpu_destroy(g_ctx);
    g_ctx = nullptr;
    pgpu_params p;
    pgpu_default_params(&p);
    p.dim = DIMENSION;
    p.k = _K_;
    p.buff = buff;
    p.gamma = _gamma_;
    p.boundary = PGPU_PERIODIC;
    p.flux_mode = PGPU_FLUX_REFERENCE;
    p.predicates = PGPU_PRED_REFERENCE;
    int rc = pgpu_create(&p, &g_ctx);
    if (rc) die("pgpu_create", rc);
    g_buff = buff;
    g_gamma = _gamma_;
    g_key = MeshKey();
    return g_ctx;
}

void die(const char* what, int rc) {
    std::fprintf(stderr, "PROTEUS-GPU: %s failed (%d): %s\n", what, rc, g_ctx ? pgpu_last_error(g_ctx) : "");
    std::exit(EXIT_FAILURE);
}

void invalidate_mesh() { g_key = MeshKey(); }

MeshKey& device_mesh_key() { return g_key; }

}  // namespace pgpu_dropin
