"""ctypes binding of libproteus_gpu.so (the C ABI in include/proteus_gpu.h).

The library is built in-tree by proteusgpu_b200/build.py.  There is no CPU
fallback: if the library cannot be loaded, or no CUDA device is present, the
calls raise.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libproteus_gpu.so")

PGPU_PERIODIC, PGPU_REFLECTIVE = 0, 1
PGPU_FLUX_REFERENCE, PGPU_FLUX_PHYSICAL = 0, 1
ERRORS = {0: "ok", -1: "invalid argument", -2: "CUDA error", -3: "call out of order",
          -4: "capacity exceeded", -5: "mesh unusable"}

# every symbol include/proteus_gpu.h declares
EXPORTED = [
    "pgpu_default_params", "pgpu_create", "pgpu_destroy", "pgpu_last_error", "pgpu_abi_version",
    "pgpu_knn", "pgpu_knn_sorted", "pgpu_periodic_mesh", "pgpu_compute_mesh", "pgpu_download_mesh",
    "pgpu_mesh_sizes", "pgpu_upload_mesh", "pgpu_set_prim", "pgpu_get_prim", "pgpu_dt_cfl",
    "pgpu_hydro_step", "pgpu_sim_init", "pgpu_sim_step", "pgpu_sim_step_host", "pgpu_sim_get",
    "pgpu_sim_set", "pgpu_sim_stats", "pgpu_enable_timing", "pgpu_stage_times", "pgpu_stream",
    "pgpu_launch_count", "pgpu_fp64_peak", "pgpu_riemann_hll", "pgpu_dt_cfl_static",
    "pgpu_kbudget_enable", "pgpu_kbudget_classes", "pgpu_kbudget_stats", "pgpu_kbudget_weights",
    "pgpu_mlp_forward", "pgpu_mlp_grad", "pgpu_fp32_peak", "pgpu_batch_init", "pgpu_batch_dt", "pgpu_autotune",
    "pgpu_set_tuning", "pgpu_download_points", "pgpu_walked_slots", "pgpu_sample_cells",
    "pgpu_ic_generate", "pgpu_sim_init_ic", "pgpu_batch_init_ic",
]

IC_KINDS = {"sod": 0, "sedov": 1, "kh": 2, "clustered": 3}


class ICSpec(C.Structure):
    _fields_ = [("kind", C.c_int32), ("dim", C.c_int32), ("n", C.c_int64), ("n_side", C.c_int32),
                ("n_clumps", C.c_int32), ("seed", C.c_uint64), ("gamma", C.c_double), ("jitter", C.c_double),
                ("split_cos", C.c_double), ("split_sin", C.c_double), ("p0", C.c_double), ("e_blast", C.c_double),
                ("rho_ratio", C.c_double), ("frac_clumped", C.c_double)]


def ic_spec(spec: dict) -> ICSpec:
    """The pgpu_ic_spec of a generator's spec dict (ics.IC.spec)."""
    s = ICSpec()
    s.kind = IC_KINDS[spec["kind"]]
    s.dim = spec["dim"]
    s.n = spec.get("n", 0)
    s.n_side = spec.get("n_side", 0)
    s.n_clumps = spec.get("n_clumps", 0)
    s.seed = spec["seed"]
    s.gamma = spec["gamma"]
    s.jitter = spec.get("jitter", 0.1)
    s.split_cos = spec.get("split_cos", 1.0)
    s.split_sin = spec.get("split_sin", 0.0)
    s.p0 = spec.get("p0", 1e-5)
    s.e_blast = spec.get("e_blast", 1.0)
    s.rho_ratio = spec.get("rho_ratio", 2.0)
    s.frac_clumped = spec.get("frac_clumped", 0.7)
    return s


class Params(C.Structure):
    _fields_ = [("dim", C.c_int), ("k", C.c_int), ("boundary", C.c_int), ("flux_mode", C.c_int),
                ("buff", C.c_double), ("gamma", C.c_double), ("device", C.c_int), ("verbose", C.c_int),
                ("predicates", C.c_int), ("k_fallback", C.c_int), ("precision", C.c_int)]


class Stats(C.Structure):
    _fields_ = [("n_hydro", C.c_int64), ("n_ext", C.c_int64), ("num_faces", C.c_int64),
                ("failed_cells", C.c_int64), ("box_faces", C.c_int64), ("unpaired_faces", C.c_int64),
                ("knn_candidates", C.c_int64), ("last_dt", C.c_double), ("total_mass", C.c_double),
                ("total_energy", C.c_double), ("total_mom", C.c_double * 3), ("cert_k_max", C.c_int32),
                ("n_grid", C.c_int32), ("refit_cells", C.c_int64), ("uncertified_cells", C.c_int64),
                ("reclip_cells", C.c_int64), ("pruned_cells", C.c_int64), ("walk_points", C.c_int64),
                ("walk_boxes", C.c_int64), ("clip_split_ms", C.c_float * 3), ("knn_redone", C.c_int32)]


class KBudgetInfo(C.Structure):
    _fields_ = [("active", C.c_int32), ("steps_trained", C.c_int64), ("last_loss", C.c_double),
                ("cells", C.c_int64), ("misses", C.c_int64), ("mean_k", C.c_double)]


BOUNDARY = {"periodic": 0, "reflective": 1}


class Tuning(C.Structure):
    _fields_ = [("ppb", C.c_double), ("knn_warps", C.c_int32), ("clip_warps", C.c_int32),
                ("clip_thread", C.c_int32), ("knn_thread", C.c_int32), ("ms_default", C.c_float), ("ms_tuned", C.c_float),
                ("from_cache", C.c_int32)]
KB_NPARAM = 1542  # W1[32][8], b1[32], W2[32][32], b2[32], W3[6][32], b3[6]

_LIB = None
vp = C.c_void_p
i64 = C.c_int64
dbl = C.c_double


def load(path: str = LIB_PATH):
    """Loads the library (build it with ``python -m proteusgpu_b200.build``)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(path):
        raise RuntimeError(f"{path} is missing: build it with `python -m proteusgpu_b200.build` "
                           "(there is no CPU fallback)")
    L = C.CDLL(path)
    L.pgpu_default_params.argtypes = [C.POINTER(Params)]
    L.pgpu_default_params.restype = None
    L.pgpu_create.argtypes = [C.POINTER(Params), C.POINTER(vp)]
    L.pgpu_destroy.argtypes = [vp]
    L.pgpu_destroy.restype = None
    L.pgpu_last_error.argtypes = [vp]
    L.pgpu_last_error.restype = C.c_char_p
    L.pgpu_abi_version.restype = C.c_int
    L.pgpu_knn.argtypes = [vp, vp, i64, vp]
    L.pgpu_knn_sorted.argtypes = [vp, vp, vp, vp]
    L.pgpu_periodic_mesh.argtypes = [vp, vp, i64, vp, vp]
    L.pgpu_compute_mesh.argtypes = [vp, vp, i64, vp]
    L.pgpu_download_mesh.argtypes = [vp] + [vp] * 11
    L.pgpu_mesh_sizes.argtypes = [vp, vp, vp, vp]
    L.pgpu_upload_mesh.argtypes = [vp, i64, i64, i64] + [vp] * 7
    L.pgpu_set_prim.argtypes = [vp, vp, vp, vp, i64]
    L.pgpu_get_prim.argtypes = [vp, vp, vp, vp]
    L.pgpu_dt_cfl.argtypes = [vp, dbl, vp]
    L.pgpu_hydro_step.argtypes = [vp, dbl]
    L.pgpu_sim_init.argtypes = [vp, vp, vp, vp, vp, vp, i64]
    L.pgpu_sim_step.argtypes = [vp, dbl, dbl, vp]
    L.pgpu_sim_step_host.argtypes = [vp, dbl, dbl, vp, vp, vp, vp, vp]
    L.pgpu_sim_get.argtypes = [vp, vp, vp, vp, vp]
    L.pgpu_sim_set.argtypes = [vp, vp, vp, vp, vp]
    L.pgpu_sim_stats.argtypes = [vp, C.POINTER(Stats)]
    L.pgpu_enable_timing.argtypes = [vp, C.c_int]
    L.pgpu_stage_times.argtypes = [vp, vp]
    L.pgpu_stream.argtypes = [vp]
    L.pgpu_stream.restype = vp
    L.pgpu_launch_count.restype = C.c_int64
    L.pgpu_fp64_peak.argtypes = [C.c_int, C.c_float, vp]
    L.pgpu_fp32_peak.argtypes = [C.c_int, C.c_float, vp]
    L.pgpu_batch_init.argtypes = [vp, C.c_int, vp, vp, vp, vp, vp, vp, vp, vp, vp]
    L.pgpu_batch_dt.argtypes = [vp, vp]
    L.pgpu_autotune.argtypes = [vp, C.POINTER(Tuning)]
    L.pgpu_set_tuning.argtypes = [vp, C.POINTER(Tuning)]
    L.pgpu_riemann_hll.argtypes = [C.c_int, dbl, vp, vp, vp, vp]
    L.pgpu_dt_cfl_static.argtypes = [C.c_int, dbl, dbl, vp, vp, vp, vp, i64, vp, vp]
    L.pgpu_kbudget_enable.argtypes = [vp, C.c_int, C.c_int, dbl, C.c_uint64]
    L.pgpu_kbudget_classes.argtypes = [C.c_int, vp]
    L.pgpu_kbudget_stats.argtypes = [vp, C.POINTER(KBudgetInfo)]
    L.pgpu_kbudget_weights.argtypes = [vp, vp, vp]
    L.pgpu_mlp_forward.argtypes = [vp, vp, i64, vp, vp]
    L.pgpu_mlp_grad.argtypes = [vp, vp, vp, i64, vp, vp]
    L.pgpu_ic_generate.argtypes = [vp, C.POINTER(ICSpec), vp, vp, vp, vp, vp]
    L.pgpu_sim_init_ic.argtypes = [vp, C.POINTER(ICSpec)]
    L.pgpu_batch_init_ic.argtypes = [vp, C.c_int, vp, vp, vp]
    L.pgpu_download_points.argtypes = [vp, vp]
    L.pgpu_walked_slots.argtypes = [vp, vp, i64, vp]
    L.pgpu_sample_cells.argtypes = [vp, vp, i64] + [vp] * 11 + [i64]
    for name in EXPORTED:
        getattr(L, name)  # raises AttributeError if a declared symbol is missing
    _LIB = L
    return L


class PGPUError(RuntimeError):
    pass


def check(ctx, rc: int, what: str):
    if rc != 0:
        msg = ""
        if ctx:
            m = load().pgpu_last_error(ctx)
            msg = m.decode() if m else ""
        raise PGPUError(f"{what} failed ({rc}: {ERRORS.get(rc, '?')}) {msg}")
