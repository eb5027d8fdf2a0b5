// Shared state of the drop-in translation units: one device context for the
// process, created on first use with the reference's compile-time dimension and
// _K_ and its current globals `buff` and `_gamma_` (src/global/allvars.cpp:13-14).
#pragma once

#include <vector>

#include "proteus_gpu.h"

struct VMesh;  // src/voronoi/voronoi.h:22-41

namespace pgpu_dropin {

// The context for the current (DIMENSION, _K_, buff, _gamma_); recreated if a
// global changed since the last call.  Exits on failure, as the reference does
// on unrecoverable errors (knn.cpp:33-36).
pgpu_ctx* context();

// Prints the C ABI's error message for `what` and exits with EXIT_FAILURE.
[[noreturn]] void die(const char* what, int rc);

// Forgets the device mesh so that the next hydro:: call uploads the host VMesh again.
void invalidate_mesh();

// Identity of the host VMesh currently on the device (see hydro_gpu.cpp).
struct MeshKey {
    const void* mesh = nullptr;
    const void* volumes = nullptr;
    unsigned long long num_faces = 0, n_seeds = 0;
};
MeshKey& device_mesh_key();

// Copies the context's device mesh into a newly allocated host VMesh (cells in
// input order, faces CSR per cell).  n_hydro and ghost_ids are filled when
// periodic is true; statuses go to *status when it is not null.
VMesh* download_vmesh(pgpu_ctx* c, bool periodic, std::vector<int>* status);

}  // namespace pgpu_dropin
