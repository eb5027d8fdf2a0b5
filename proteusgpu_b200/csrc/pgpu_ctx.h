// Host-side context of the C ABI and the launch wrappers shared by the .cu files.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <utility>

#include "../../include/proteus_gpu.h"

namespace pgpu {

// A device allocation that only grows.  Contents are not preserved on growth.
struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
};

cudaError_t ensure_bytes(DevBuf& b, size_t bytes);
template <class T>
inline T* ensure(DevBuf& b, size_t n, cudaError_t* err) {
    cudaError_t e = ensure_bytes(b, n * sizeof(T) + 16);
    if (e != cudaSuccess && err) *err = e;
    return (T*)b.p;
}

// Device-side counters/scalars of one context (one allocation).
struct DevScalars {
    unsigned long long dt_bits;     // atomicMin target for the CFL step
    unsigned long long face_count;  // faces reserved by the extraction
    unsigned long long knn_cand;    // candidate evaluations (statistics)
    unsigned int overflow;          // face storage overflow flag
    unsigned int box_faces;         // hydro faces on the bounding box
    unsigned int unpaired;          // faces without a reverse partner
    unsigned int failed;            // hydro cells not certified
    int cert_k_max;
    unsigned int uncertified;       // hydro cells with SECURITY_RADIUS_NOT_REACHED in the last clip
    unsigned int reclip;            // cells the FP32 clip could not decide
    double dt;                      // the step's dt (device copy)
    double sums[5];                 // mass, mom x/y/z, energy
};

}  // namespace pgpu

struct pgpu_ctx {
    pgpu_params prm{};
    cudaStream_t stream = nullptr;
    std::string err;
    bool timing = false;
    cudaEvent_t ev[6] = {};
    float stage_ms[5] = {};

    // sizes of the current mesh
    int64_t n_hydro = 0, n_ext = 0, num_faces = 0, n_query = 0;
    int grid_G = 0;
    int64_t morton_slots = 0;
    bool have_mesh = false, all_cells = false, have_prim = false, have_sim = false;
    bool mesh_uploaded = false;  // mesh came from pgpu_upload_mesh (no points)
    double unit_scale = 1.0;     // 1 + 2 buff: unit box -> physical

    // ---- device buffers ----
    pgpu::DevBuf pos;          // hydro positions (physical), n x dim
    pgpu::DevBuf ext;          // extended unit-box points, ext-id order (PointOf<D>)
    pgpu::DevBuf gcnt, goff;   // ghosts per hydro point and their offsets
    pgpu::DevBuf ghost_src;    // u32: hydro id copied by each ghost
    pgpu::DevBuf ghost_code;   // u32: image code of each ghost
    pgpu::DevBuf bin_cnt, bin_start, bin_key;  // grid bins (Morton slots) and per-point key
    pgpu::DevBuf spts, perm, inv;  // sorted points, sorted->ext id, ext id->sorted
    pgpu::DevBuf qflag, qoff, qs;  // query list (sorted positions of the cells to compute)
    pgpu::DevBuf knn;          // n_query x K ext ids
    pgpu::DevBuf vol, fptr, fcnt, status, certk, centroid;  // per cell, indexed by ext id
    pgpu::DevBuf f_nb, f_own, f_geo;  // faces: ext id, owner|code, (normal, area)
    pgpu::DevBuf scan_tmp;     // scan block sums
    pgpu::DevBuf knn_table;    // neighbour-bin offsets sorted by lower-bound distance (int2)
    int knn_table_n = 0, knn_table_r = 0;
    pgpu::DevBuf scalars;      // DevScalars
    // hydro state
    pgpu::DevBuf rho, vel, energy, rho2, vel2, energy2;  // primitives (drop-in hydro)
    pgpu::DevBuf mass, mom, en;   // conserved (moving mesh)
    pgpu::DevBuf w4, we;          // per-step primitives (rho, v) and E
    pgpu::DevBuf red_tmp;         // reduction partials
    // download staging
    pgpu::DevBuf dl_ptr, dl_a, dl_b, dl_c;
    size_t face_cap = 0;
    int64_t n_uncertified = 0;  // hydro cells of the last clip with SECURITY_RADIUS_NOT_REACHED
    int64_t n_refit = 0;        // cells recomputed with the fallback budget in the last step
    int64_t n_reclip = 0;       // cells the FP32 clip handed to the FP64 clip in the last step
    pgpu::DevBuf fb_qs, fb_knn; // fallback query list and lists
};

namespace pgpu {

// Process-wide count of kernel launches (statistics, pgpu_launch_count).
void count_launches(int n);

// ---- launch wrappers (defined in the .cu files) ----
// scan.cu
cudaError_t exclusive_scan_u32(const uint32_t* in, uint32_t* out, int64_t n, DevBuf& tmp, cudaStream_t s);
// mesh_prep.cu
cudaError_t launch_ghosts(pgpu_ctx* c, const double* pos_dev, int64_t n, bool scale_only);
cudaError_t launch_grid_sort(pgpu_ctx* c);
cudaError_t launch_query_list(pgpu_ctx* c, bool all_cells);
// knn.cu
cudaError_t launch_knn(pgpu_ctx* c);
cudaError_t launch_knn_list(pgpu_ctx* c, const uint32_t* qs, int64_t nq, int K, uint32_t* out);
// clip.cu
cudaError_t launch_clip(pgpu_ctx* c);
cudaError_t launch_fallback(pgpu_ctx* c);
// hydro.cu
cudaError_t launch_prim_dt(pgpu_ctx* c, double cfl, double fixed_dt);
cudaError_t launch_flux_update(pgpu_ctx* c, double fixed_dt);
cudaError_t launch_dt_ref(pgpu_ctx* c, double cfl);
cudaError_t launch_hydro_ref(pgpu_ctx* c, double dt);
cudaError_t launch_cons_from_prim(pgpu_ctx* c, const double* deposit_dev);
cudaError_t launch_sums(pgpu_ctx* c);
// download.cu
cudaError_t launch_mesh_compact(pgpu_ctx* c, uint32_t* new_ptr, int32_t* nb_out, double* nrm_out, double* area_out);
cudaError_t launch_seeds(pgpu_ctx* c, double* out, bool no_scale);
cudaError_t launch_knn_rows(pgpu_ctx* c, uint32_t* out);
cudaError_t launch_unpack_points(pgpu_ctx* c, const void* pts, int64_t n, double* out);

}  // namespace pgpu
