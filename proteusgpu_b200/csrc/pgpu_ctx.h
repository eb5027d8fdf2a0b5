// Host-side context of the C ABI and the launch wrappers shared by the .cu files.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <utility>
#include <vector>

#include "../../include/proteus_gpu.h"

namespace pgpu {

// Per-simulation parameters.  A context advances one simulation, or a batch of
// independent ones whose points are concatenated (hydro points of every
// instance first, then every instance's ghosts); each instance keeps its own
// unit box, ghost layer, grid, gamma, boundary and time step, so that its
// results are those of a run on its own.
struct InstPar {
    double buff;       // ghost layer width
    double scale_in;   // 1 / (1 + 2 buff): physical -> unit box
    double scale_out;  // 1 + 2 buff: unit box -> physical
    double gamma;
    int mirror;        // reflective walls
    int G;             // coarse grid bins per axis
    uint32_t slot0;    // first coarse Morton slot of this instance's grid
    uint32_t count;    // hydro points
};

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
    unsigned long long walk_points; // grid walk: points clipped (statistics; after the
    unsigned long long walk_boxes;  //   per-step counters, which are cleared up to dt)
    unsigned int sort_big;          // grid sort: sub-bins too large for one thread
    unsigned int knn_redo;          // KNN: queries listed for the exact-key search (per launch)
    unsigned int knn_redo_total;    // and their total over the last KNN stage (statistics)
};

// Learned neighbour budget: a per-cell MLP (8 features -> 32 -> 32 -> 6 classes,
// GELU) proposes each cell's K; training and inference run on the device.
constexpr int KB_FEATURES = 8;
constexpr int KB_HIDDEN = 32;
constexpr int KB_CLASSES = 6;
// FP32 master parameters: W1[32][8], b1[32], W2[32][32], b2[32], W3[6][32], b3[6]
constexpr int KB_W1 = 0, KB_B1 = 256, KB_W2 = 288, KB_B2 = 1312, KB_W3 = 1344, KB_B3 = 1536;
constexpr int KB_NPARAM = 1542;
constexpr int KB_PART = 1544;  // per-warp partial gradient row (parameters, loss, pad)
// BF16 operand copies (u16): W1[32][8], W2[32][32], W2^T, W3[8][32] (rows 6-7 zero), W3^T[32][8]
constexpr int KB_BW1 = 0, KB_BW2 = 256, KB_BW2T = 1280, KB_BW3 = 2304, KB_BW3T = 2560, KB_NBF = 2816;
constexpr int KB_GRAD_BLOCKS = 148, KB_GRAD_WARPS = 4;

// The simulations a context advances (one unless pgpu_batch_init made a batch).
struct Instances {
    int n = 1;
    std::vector<int64_t> count;      // hydro points per instance
    std::vector<int64_t> hydro0;     // first hydro id (n + 1 entries)
    std::vector<int64_t> ext_count;  // hydro + ghost points per instance (last mesh)
    std::vector<InstPar> par;        // host copy of the parameters
    DevBuf d_par;                    // InstPar[n]
    DevBuf d_inst_h;                 // u16 per hydro id
    DevBuf d_inst_e;                 // u16 per extended id
    DevBuf d_dt;                     // u64 dt bits per instance
    std::vector<unsigned long long> dt_init;  // staging for their reset
    DevBuf d_gather;                 // u32 scratch for per-instance ghost totals
};

// Launch shapes chosen by pgpu_autotune (defaults until it runs).
struct Tuning {
    double ppb = 2.0;    // mean points per coarse grid bin
    int knn_warps = 4;   // queries (warps) per KNN block: 2, 4 or 8
    int clip_warps = 4;  // cells (warps) per clipping block: 2 or 4
    bool clip_thread = false;  // 2D: one thread per cell instead of one warp
    int knn_thread = 0;        // queries with K <= 32 or 64 searched one per thread (0 = none)
};

struct KBudget {
    bool enabled = false;
    bool trained = false;
    int train_steps = 0;       // steps of the plain method whose certified K train the model
    int iters = 64;            // optimiser iterations per training step
    int batch = 16384;         // cells per iteration
    float quantile = 0.99f;    // smallest class whose cumulative probability reaches this
    float lr = 3e-3f;
    uint64_t seed = 1;
    int64_t steps_seen = 0, adam_t = 0;
    double last_loss = 0.0;
    int64_t cells = 0, misses = 0;  // last step: cells proposed, cells that needed the fallback
    double mean_k = 0.0;            // last step: mean proposed K
    DevBuf w, wbf, adam_m, adam_v, part, feat, hist_vol, miss, ksum, labels, tmp_out;
};

}  // namespace pgpu

struct pgpu_ctx {
    pgpu_params prm{};
    cudaStream_t stream = nullptr;
    cudaStream_t copy_stream = nullptr;  // pgpu_sim_step_host: the conserved state's upload
    cudaEvent_t copy_ev[2] = {};          // the main stream's entry point; the upload's end
    bool copy_pending = false;            // the step must wait for copy_ev[1] before using the state
    std::string err;
    bool timing = false;
    cudaEvent_t ev[9] = {};    // 0-5: stage boundaries; 6-8: after the main clip, the fallback, the walk
    unsigned ev_mask = 0;      // events recorded since the last build began
    float stage_ms[5] = {};
    float clip_ms[3] = {};     // the clip stage split: main clip (+ re-clip), fallback, grid walk

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
    pgpu::DevBuf bin_lvl;      // u8 per coarse bin: refinement level L ((2^L)^D sub-bins)
    pgpu::DevBuf sub_off;      // u32 per coarse bin: first sub-bin slot (M + 1 entries)
    pgpu::DevBuf sub_cnt, sub_start;  // per sub-bin slot: counts, first sorted point (T + 1)
    pgpu::DevBuf sort_big, sort_keys, sort_pts;  // large sub-bins: their slots, key and point scratch
    int64_t sub_slots = 0;     // T
    pgpu::DevBuf spts, perm, inv;  // sorted points, sorted->ext id, ext id->sorted
    pgpu::DevBuf qflag, qoff, qs;  // query list (sorted positions of the cells to compute)
    pgpu::DevBuf knn;          // n_query rows of knn_stride ext ids
    pgpu::DevBuf knn_redo;     // u32 query indices whose packed-key search met a tie
    int knn_stride = 0;        // ids per row: prm.k, or the largest learned budget
    pgpu::DevBuf kq;           // u16 per query slot: learned neighbour budget
    bool use_kq = false;       // this step's lists and clip use kq
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
    pgpu::DevBuf ale_wp, ale_grad; // moving-face modes: predicted primitives and their gradients
    pgpu::DevBuf red_tmp;         // reduction partials
    // download staging
    pgpu::DevBuf dl_ptr, dl_a, dl_b, dl_c;
    size_t face_cap = 0;
    int64_t n_uncertified = 0;  // hydro cells of the last clip with SECURITY_RADIUS_NOT_REACHED
    int64_t n_refit = 0;        // cells recomputed with the fallback budget in the last step
    int64_t n_reclip = 0;       // cells the FP32 clip handed to the FP64 clip in the last step
    int64_t n_pruned = 0;       // cells certified by the grid walk in the last step
    pgpu::DevBuf fb_qs, fb_knn; // fallback query list and lists
    pgpu::KBudget kb;           // learned neighbour budget (optional form)
    pgpu::Instances inst;       // the simulation(s) of this context
    pgpu::Tuning tune;          // launch shapes (pgpu_autotune)
};

namespace pgpu {

// Process-wide count of kernel launches (statistics, pgpu_launch_count).
void count_launches(int n);

// ---- launch wrappers (defined in the .cu files) ----
// scan.cu
cudaError_t exclusive_scan_u32(const uint32_t* in, uint32_t* out, int64_t n, DevBuf& tmp, cudaStream_t s);
// mesh_prep.cu
// one instance from the context's parameters, n hydro points
cudaError_t set_single_instance(pgpu_ctx* c, int64_t n);
// a batch: counts[b] points per instance, with their own buff, gamma and boundary
cudaError_t set_instances(pgpu_ctx* c, int nb, const int64_t* counts, const double* buff, const double* gamma,
                          const int* boundary);
cudaError_t launch_ghosts(pgpu_ctx* c, const double* pos_dev, int64_t n, bool scale_only);
cudaError_t launch_grid_sort(pgpu_ctx* c);
cudaError_t launch_query_list(pgpu_ctx* c, bool all_cells);
// knn.cu
cudaError_t launch_knn(pgpu_ctx* c);
// K neighbours of each query (or kq[t] of query t, <= K) into rows of `stride` ids
cudaError_t launch_knn_list(pgpu_ctx* c, const uint32_t* qs, int64_t nq, int K, uint32_t* out, const uint16_t* kq,
                            int stride);
// clip.cu
cudaError_t launch_clip(pgpu_ctx* c);
// uncertified hydro cells of the last clip: KNN and clipping again with budget K2
cudaError_t launch_fallback(pgpu_ctx* c, int K2);
// uncertified hydro cells of the last clip: clipped by walking the grid (no neighbour budget)
cudaError_t launch_pruned(pgpu_ctx* c);
// kbudget.cu
cudaError_t kb_init_weights(pgpu_ctx* c);
cudaError_t kb_features(pgpu_ctx* c);                 // before the step's clip (reads the previous mesh)
cudaError_t kb_infer(pgpu_ctx* c, const float* feat, int64_t n, uint16_t* kq, float* logits);
cudaError_t kb_train_step(pgpu_ctx* c);               // after the step's clip (labels = certified K)
cudaError_t kb_grad(pgpu_ctx* c, const float* feat, const int32_t* labels, int64_t n, const uint32_t* sample,
                    int64_t nb, bool update);
cudaError_t kb_mark_miss(pgpu_ctx* c, const uint32_t* sorted_pos, int64_t n);
cudaError_t kb_sync_bf16(pgpu_ctx* c);               // BF16 operand copies from the FP32 master weights
int kb_class_k(int dim, int cls);
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
// ics.cu: a generated initial condition into device arrays (dep may be NULL)
cudaError_t ic_generate(pgpu_ctx* c, const pgpu_ic_spec* s, int64_t n, double* pos, double* rho, double* vel,
                        double* en, double* dep);
// sampled query slots: ext ids, main-clip neighbour rows (width knn_stride or k), per-cell outputs
cudaError_t launch_sample_cells(pgpu_ctx* c, const uint32_t* slots, int64_t n, uint32_t* ext_out, uint16_t* len_out,
                                uint32_t* rows_out, int32_t* st_out, int32_t* ck_out, double* vol_out,
                                double* cen_out, uint32_t* fc_out);
cudaError_t launch_sample_faces(pgpu_ctx* c, const uint32_t* ext_ids, const uint32_t* fc, const uint64_t* dst_ptr,
                                int64_t n, int32_t* nb_out, double* nrm_out, double* area_out);

}  // namespace pgpu
