"""ctypes access to the reference build in oracle/_ref (test infrastructure only).

oracle/_ref/libref_<dim>d_k<K>.so are the reference's own hot-path translation
units compiled by oracle/Makefile (``make ref``) and linked with
oracle/ref_driver.cpp.  This module loads them and converts the reference's
VMesh (src/voronoi/voronoi.h:22-41) into numpy arrays.

Only tests, ``__graft_entry__.smoke()`` and bench.py's CPU arms use this module.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_lp = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")
_up = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")

_LIBS: dict = {}


# Libraries with the same extern "C" surface: the reference build (oracle/_ref) and
# the drop-in translation units linked with the same driver (proteusgpu_b200/dropin).
DROPIN_DIR = os.path.join(os.path.dirname(HERE), "proteusgpu_b200", "dropin", "_build")
_PREFIX = {"ref": (REF_DIR, "libref"), "dropin": (DROPIN_DIR, "libdropin")}
_FLAVOR = "ref"


def use(flavor: str):
    """Selects which library the functions below call: "ref" (the reference build) or
    "dropin" (the drop-in units over the GPU path).  Returns the previous choice."""
    global _FLAVOR
    prev, _FLAVOR = _FLAVOR, flavor
    return prev


def lib_path(dim: int, k: int, flavor: str | None = None) -> str:
    d, p = _PREFIX[flavor or _FLAVOR]
    return os.path.join(d, f"{p}_{dim}d_k{k}.so")


def available(dim: int, k: int, flavor: str | None = None) -> bool:
    return os.path.exists(lib_path(dim, k, flavor))


def _bind(lib):
    lib.ref_dim.restype = C.c_int
    lib.ref_k.restype = C.c_int
    lib.ref_set_params.argtypes = [C.c_double, C.c_double, C.c_int, C.c_int]
    lib.ref_n_grid.argtypes = [C.c_long]
    lib.ref_n_grid.restype = C.c_int
    lib.ref_max_threads.restype = C.c_int
    lib.ref_periodic_mesh.argtypes = [_dp, C.c_long]
    lib.ref_periodic_mesh.restype = C.c_void_p
    lib.ref_compute_mesh.argtypes = [_dp, C.c_long, _ip]
    lib.ref_compute_mesh.restype = C.c_void_p
    lib.ref_mesh_sizes.argtypes = [C.c_void_p, C.POINTER(C.c_long), C.POINTER(C.c_long), C.POINTER(C.c_long)]
    lib.ref_mesh_copy.argtypes = [C.c_void_p, _dp, _dp, _lp, _lp, _ip, _dp, _dp, _lp]
    lib.ref_mesh_wrap.argtypes = [C.c_long, C.c_long, C.c_long, _dp, _lp, _lp, _ip, _dp, _dp, _lp]
    lib.ref_mesh_wrap.restype = C.c_void_p
    lib.ref_mesh_free.argtypes = [C.c_void_p]
    lib.ref_knn.argtypes = [_dp, C.c_long, _up]
    lib.ref_knn.restype = C.c_int
    lib.ref_dt_cfl.argtypes = [C.c_void_p, C.c_double, _dp, _dp, _dp]
    lib.ref_dt_cfl.restype = C.c_double
    lib.ref_hydro_step.argtypes = [C.c_void_p, C.c_double, _dp, _dp, _dp]
    lib.ref_mesh_set_seeds.argtypes = [C.c_void_p, _dp]
    lib.ref_meshdata.argtypes = [C.c_void_p, _dp, _lp, _ip, _dp, _dp, _ip, _ip, _dp, _dp]
    lib.ref_meshdata.restype = C.c_long
    return lib


def load(dim: int, k: int):
    path = lib_path(dim, k)
    if path not in _LIBS:
        if not os.path.exists(path):
            raise FileNotFoundError(f"library {path} missing (run `make -C oracle ref REF=<reference tree>` or "
                                    "`make -C proteusgpu_b200/dropin REF=<reference tree>`)")
        _LIBS[path] = _bind(C.CDLL(path, mode=os.RTLD_LOCAL))
    return _LIBS[path]


@dataclass
class RefMesh:
    """A VMesh copied into numpy (input order; seeds/normals are 3-vectors even in 2D)."""
    n_seeds: int
    n_hydro: int
    seeds: np.ndarray
    volumes: np.ndarray
    face_counts: np.ndarray
    face_ptr: np.ndarray
    neighbor: np.ndarray
    normal: np.ndarray
    area: np.ndarray
    ghost_ids: np.ndarray
    status: np.ndarray | None = None
    handle: int | None = None      # live VMesh* (freed by RefMeshOwner)

    @property
    def num_faces(self) -> int:
        return int(len(self.neighbor))


def _copy_mesh(lib, h) -> RefMesh:
    ns, nh, nf = C.c_long(), C.c_long(), C.c_long()
    lib.ref_mesh_sizes(h, C.byref(ns), C.byref(nh), C.byref(nf))
    n, F = ns.value, nf.value
    seeds = np.zeros((n, 3)); vol = np.zeros(n)
    fc = np.zeros(n, np.int64); fp = np.zeros(n, np.int64)
    nb = np.zeros(max(F, 1), np.int32); nrm = np.zeros((max(F, 1), 3)); ar = np.zeros(max(F, 1))
    gid = np.zeros(max(n - nh.value, 1), np.int64)
    lib.ref_mesh_copy(h, seeds, vol, fc, fp, nb, nrm, ar, gid)
    return RefMesh(n, nh.value, seeds, vol, fc, fp, nb[:F], nrm[:F], ar[:F], gid[: n - nh.value])


def set_params(dim: int, k: int, buff: float = 0.04, gamma: float = 5.0 / 3.0, quiet: bool = True,
               nthreads: int = 0):
    load(dim, k).ref_set_params(buff, gamma, int(quiet), nthreads)


def periodic_mesh(pts: np.ndarray, k: int, buff: float = 0.04, gamma: float = 5.0 / 3.0,
                  keep_handle: bool = False, nthreads: int = 0) -> RefMesh:
    """voronoi::compute_periodic_mesh on hydro points in [0,1)^D (periodic ghosts within buff)."""
    pts = np.ascontiguousarray(pts, dtype=np.float64)
    dim = pts.shape[1]
    lib = load(dim, k)
    lib.ref_set_params(buff, gamma, 1, nthreads)
    h = lib.ref_periodic_mesh(pts.ravel(), len(pts))
    if not h:
        raise ValueError("reference KNN grid below 16^D (knn.cpp:32-36)")
    m = _copy_mesh(lib, h)
    if keep_handle:
        m.handle = h
    else:
        lib.ref_mesh_free(h)
    return m


def compute_mesh(pts_unit: np.ndarray, k: int, nthreads: int = 0) -> RefMesh:
    """voronoi::compute_mesh's call sequence on points already in [0,1]^D, with per-cell Status."""
    pts = np.ascontiguousarray(pts_unit, dtype=np.float64)
    dim = pts.shape[1]
    lib = load(dim, k)
    if nthreads:
        lib.ref_set_params(0.04, 5.0 / 3.0, 1, nthreads)
    st = np.zeros(len(pts), np.int32)
    h = lib.ref_compute_mesh(pts.ravel(), len(pts), st)
    if not h:
        raise ValueError("reference KNN grid below 16^D (knn.cpp:32-36)")
    m = _copy_mesh(lib, h)
    lib.ref_mesh_free(h)
    m.status = st
    return m


def knn(pts_unit: np.ndarray, k: int) -> np.ndarray:
    """knn::init + knn::solve; (N, K) neighbour lists in input ids, ascending distance."""
    pts = np.ascontiguousarray(pts_unit, dtype=np.float64)
    lib = load(pts.shape[1], k)
    out = np.zeros(len(pts) * k, np.uint32)
    if lib.ref_knn(pts.ravel(), len(pts), out) < 0:
        raise ValueError("reference KNN grid below 16^D (knn.cpp:32-36)")
    return out.reshape(len(pts), k)


def free_handle(dim: int, k: int, h):
    if h:
        load(dim, k).ref_mesh_free(h)


def wrap_mesh(dim: int, k: int, m) -> int:
    """Builds a reference VMesh from arrays of any mesh object with RefMesh fields."""
    lib = load(dim, k)
    F = len(m.neighbor)
    return lib.ref_mesh_wrap(
        m.n_seeds, m.n_hydro, F,
        np.ascontiguousarray(m.volumes, np.float64), np.ascontiguousarray(m.face_counts, np.int64),
        np.ascontiguousarray(m.face_ptr, np.int64), np.ascontiguousarray(m.neighbor, np.int32),
        np.ascontiguousarray(m.normal, np.float64).ravel(), np.ascontiguousarray(m.area, np.float64),
        np.ascontiguousarray(m.ghost_ids if len(m.ghost_ids) else np.zeros(1), np.int64))


def dt_cfl(dim: int, k: int, handle, cfl: float, rho, vel, energy, gamma: float) -> float:
    lib = load(dim, k)
    lib.ref_set_params(0.04, gamma, 1, 0)
    return lib.ref_dt_cfl(handle, cfl, np.ascontiguousarray(rho, np.float64),
                          np.ascontiguousarray(vel, np.float64).ravel(), np.ascontiguousarray(energy, np.float64))


def hydro_step(dim: int, k: int, handle, dt: float, rho, vel, energy, gamma: float):
    """hydro::hydro_step on copies of the primitives; returns (rho, vel, E)."""
    lib = load(dim, k)
    lib.ref_set_params(0.04, gamma, 1, 0)
    r = np.array(rho, np.float64, copy=True)
    v = np.array(vel, np.float64, copy=True)
    e = np.array(energy, np.float64, copy=True)
    vflat = v.reshape(-1)
    lib.ref_hydro_step(handle, dt, r, vflat, e)
    return r, vflat.reshape(v.shape), e


def set_seeds(dim: int, k: int, handle, seeds) -> None:
    """Sets the seeds (n_seeds x 3) of a VMesh made by wrap_mesh."""
    load(dim, k).ref_mesh_set_seeds(handle, np.ascontiguousarray(seeds, np.float64).reshape(-1))


def meshdata(dim: int, k: int, handle) -> dict:
    """voronoi::vmesh_to_meshdata of a live VMesh and every field of its MeshCellData."""
    lib = load(dim, k)
    ns, nh, nf = C.c_long(), C.c_long(), C.c_long()
    lib.ref_mesh_sizes(handle, C.byref(ns), C.byref(nh), C.byref(nf))
    n, F = nh.value, nf.value
    hdr, dims = np.zeros(7), np.zeros(4, np.int64)
    out = dict(cell_ids=np.zeros(max(n, 1), np.int32), seeds=np.zeros(max(n * dim, 1)),
               volumes=np.zeros(max(n, 1)), face_counts=np.zeros(max(n, 1), np.int32),
               neighbor_cell=np.zeros(max(F, 1), np.int32), normal=np.zeros(max(F * dim, 1)),
               area=np.zeros(max(F, 1)))
    nfd = lib.ref_meshdata(handle, hdr, dims, out["cell_ids"], out["seeds"], out["volumes"], out["face_counts"],
                           out["neighbor_cell"], out["normal"], out["area"])
    for key, size in (("cell_ids", n), ("seeds", n * dim), ("volumes", n), ("face_counts", n),
                      ("neighbor_cell", nfd), ("normal", nfd * dim), ("area", nfd)):
        out[key] = out[key][:size]
    out["header"] = dict(zip(("dimension", "extent", "n", "k", "nmax", "seed", "store_edge_coords"), hdr.tolist()))
    out["seeds_dims"] = dims[:2].tolist()
    out["normal_dims"] = dims[2:].tolist()
    return out
