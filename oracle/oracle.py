"""ctypes access to the plain-C restatement oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: tests, ``__graft_entry__.smoke()`` and bench.py's CPU
arms use it as the checker and as the "port" CPU baseline; the product never
imports it.  The library is built by ``make -C oracle restate`` (and by
``__graft_entry__.build()``); if it is missing, :func:`lib` builds it with gcc.

Every function here mirrors one in oracle/restate/om.h, which cites the
reference file:line each restates.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

PERIODIC, REFLECTIVE = 0, 1
STATUS_NAMES = {0: "triangle_overflow", 1: "vertex_overflow", 2: "inconsistent_boundary",
                3: "security_radius_not_reached", 4: "success", 5: "needs_exact_predicates",
                6: "not_computed"}
SUCCESS = 4


class _Mesh(C.Structure):
    _fields_ = [("dim", C.c_int), ("n_seeds", C.c_long), ("n_hydro", C.c_long), ("num_faces", C.c_long),
                ("seeds", C.POINTER(C.c_double)), ("volumes", C.POINTER(C.c_double)),
                ("face_counts", C.POINTER(C.c_long)), ("face_ptr", C.POINTER(C.c_long)),
                ("neighbor", C.POINTER(C.c_int)), ("normal", C.POINTER(C.c_double)),
                ("area", C.POINTER(C.c_double)), ("ghost_ids", C.POINTER(C.c_long)),
                ("ghost_code", C.POINTER(C.c_int)), ("status", C.POINTER(C.c_int)),
                ("cert_k", C.POINTER(C.c_int)), ("centroid", C.POINTER(C.c_double)),
                ("ext", C.POINTER(C.c_double)), ("unit_scale", C.c_double)]


_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_lp = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_up = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
_LIB = None


def build():
    subprocess.run(["make", "-s", "-C", HERE, "restate"], check=True)


def lib():
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH, mode=os.RTLD_LOCAL)
        L.om_ghosts.argtypes = [C.c_int, C.c_int, C.c_double, _dp, C.c_long, _dp, _lp, _ip]
        L.om_ghosts.restype = C.c_long
        L.om_knn.argtypes = [C.c_int, _dp, C.c_long, C.c_int, _up]
        L.om_cells.argtypes = [C.c_int, _dp, C.c_long, C.c_long, _up, C.c_int, C.c_long, C.POINTER(_Mesh)]
        L.om_build_mesh.argtypes = [C.c_int, C.c_int, C.c_double, C.c_int, _dp, C.c_long, C.c_int, C.POINTER(_Mesh)]
        L.om_mesh_free.argtypes = [C.POINTER(_Mesh)]
        L.om_dt_cfl.argtypes = [C.POINTER(_Mesh), C.c_double, C.c_double, _dp, _dp, _dp]
        L.om_dt_cfl.restype = C.c_double
        L.om_hydro_step_ref.argtypes = [C.POINTER(_Mesh), C.c_double, C.c_double, _dp, _dp, _dp]
        L.om_hydro_step_ref.restype = C.c_long
        L.om_step_moving.argtypes = [C.POINTER(_Mesh), C.c_double, C.c_double, C.c_double, C.c_int,
                                     _dp, _dp, _dp, _dp, C.POINTER(C.c_long)]
        L.om_step_moving.restype = C.c_double
        L.om_symmetric_area.argtypes = [C.POINTER(_Mesh), _dp]
        L.om_symmetric_area.restype = C.c_long
        L.om_num_regions.argtypes = [C.c_int]
        L.om_get_counters.argtypes = [_lp]
        L.om_set_predicate_mode.argtypes = [C.c_int]
        L.om_set_fallback_k.argtypes = [C.c_int]
        L.om_set_boundary_mode.argtypes = [C.c_int]
        L.om_set_expand_k.argtypes = [C.c_int]
        L.om_step_ale.argtypes = [C.POINTER(_Mesh), C.c_int, C.c_double, C.c_double, C.c_double, _dp, _dp, _dp,
                                  _dp, C.POINTER(C.c_long)]
        L.om_step_ale.restype = C.c_double
        L.om_grid_new.argtypes = [C.c_int, _dp, C.c_long]
        L.om_grid_new.restype = C.c_void_p
        L.om_grid_free.argtypes = [C.c_void_p]
        L.om_grid_knn.argtypes = [C.c_void_p, _lp, C.c_long, C.c_int, _up]
        L.om_cells_list.argtypes = [C.c_int, _dp, C.c_long, _lp, C.c_long, _up, C.c_int, C.POINTER(_Mesh)]
        L.om_cells_certified.argtypes = [C.c_void_p, _dp, C.c_long, _lp, C.c_long, C.c_int, C.c_int,
                                         C.POINTER(_Mesh), _ip]
        _LIB = L
    return _LIB


@dataclass
class Mesh:
    """A mesh in the reference's VMesh layout (input order, CSR faces) plus extras."""
    dim: int
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
    ghost_code: np.ndarray
    status: np.ndarray
    cert_k: np.ndarray
    centroid: np.ndarray
    _c: object = None   # the live C struct (for the hydro calls)

    @property
    def num_faces(self):
        return int(len(self.neighbor))

    def free(self):
        if self._c is not None:
            lib().om_mesh_free(C.byref(self._c))
            self._c = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def _arr(ptr, n, dtype):
    if n <= 0 or not ptr:
        return np.zeros(max(n, 0), dtype)
    return np.ctypeslib.as_array(ptr, shape=(n,)).astype(dtype, copy=True)


def _wrap(m: _Mesh) -> Mesh:
    n, F, nh = m.n_seeds, m.num_faces, m.n_hydro
    return Mesh(m.dim, n, nh, _arr(m.seeds, 3 * n, np.float64).reshape(n, 3), _arr(m.volumes, n, np.float64),
                _arr(m.face_counts, n, np.int64), _arr(m.face_ptr, n, np.int64), _arr(m.neighbor, F, np.int32),
                _arr(m.normal, 3 * F, np.float64).reshape(F, 3), _arr(m.area, F, np.float64),
                _arr(m.ghost_ids, n - nh, np.int64), _arr(m.ghost_code, n - nh, np.int32),
                _arr(m.status, n, np.int32), _arr(m.cert_k, n, np.int32),
                _arr(m.centroid, 3 * n, np.float64).reshape(n, 3), m)


def ghosts(pts: np.ndarray, buff: float = 0.04, boundary: int = PERIODIC):
    """Extended unit-box point set, ghost sources and image codes."""
    pts = np.ascontiguousarray(pts, np.float64)
    n, dim = pts.shape
    nreg = lib().om_num_regions(dim)
    ext = np.zeros((nreg + 1) * max(n, 1) * dim)
    src = np.zeros(nreg * max(n, 1), np.int64)
    code = np.zeros(nreg * max(n, 1), np.int32)
    ntot = lib().om_ghosts(dim, boundary, buff, pts.ravel(), n, ext, src, code)
    return ext[: ntot * dim].reshape(ntot, dim), src[: ntot - n], code[: ntot - n]


def knn(pts_unit: np.ndarray, k: int) -> np.ndarray:
    pts = np.ascontiguousarray(pts_unit, np.float64)
    out = np.zeros(len(pts) * k, np.uint32)
    lib().om_knn(pts.shape[1], pts.ravel(), len(pts), k, out)
    return out.reshape(len(pts), k)


def cells(ext_unit: np.ndarray, n_hydro: int, knn_lists: np.ndarray, n_compute: int | None = None) -> Mesh:
    """Clip + extract cells of a unit-box point set (mesh stays in unit-box units)."""
    ext = np.ascontiguousarray(ext_unit, np.float64)
    kl = np.ascontiguousarray(knn_lists, np.uint32)
    m = _Mesh()
    lib().om_cells(ext.shape[1], ext.ravel(), len(ext), n_hydro, kl.ravel(), kl.shape[1],
                   len(ext) if n_compute is None else n_compute, C.byref(m))
    return _wrap(m)


class Grid:
    """The KNN grid of one extended unit-box point set (om_grid_new): exact K
    nearest neighbours of listed queries, each row identical to the one
    :func:`knn` gives that point."""

    def __init__(self, ext_unit: np.ndarray):
        self.ext = np.ascontiguousarray(ext_unit, np.float64)
        self.dim = self.ext.shape[1]
        self._g = lib().om_grid_new(self.dim, self.ext.ravel(), len(self.ext))

    def knn(self, queries, k: int) -> np.ndarray:
        q = np.ascontiguousarray(queries, np.int64)
        out = np.zeros(max(len(q), 1) * k, np.uint32)
        lib().om_grid_knn(self._g, q, len(q), k, out)
        return out[: len(q) * k].reshape(len(q), k)

    def close(self):
        if getattr(self, "_g", None):
            lib().om_grid_free(self._g)
            self._g = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def cells_list(ext_unit: np.ndarray, ids, knn_rows: np.ndarray) -> Mesh:
    """Listed cells clipped with their neighbour rows (om_cells_list): cell t of the
    result is ids[t]; unit-box units; face neighbours are extended ids."""
    ext = np.ascontiguousarray(ext_unit, np.float64)
    ids = np.ascontiguousarray(ids, np.int64)
    kl = np.ascontiguousarray(knn_rows, np.uint32)
    m = _Mesh()
    lib().om_cells_list(ext.shape[1], ext.ravel(), len(ext), ids, len(ids), kl.ravel(), kl.shape[1], C.byref(m))
    return _wrap(m)


def cells_certified(grid: Grid, ids, k0: int = 190, k_max: int = 1 << 16):
    """Listed cells clipped by the reference's algorithm with a budget large enough to
    certify each (om_cells_certified): K0 neighbours, then 4x budgets up to k_max for
    the cells whose certificate did not close.  Returns (mesh, budget of the final
    attempt per cell)."""
    ids = np.ascontiguousarray(ids, np.int64)
    m = _Mesh()
    ku = np.zeros(max(len(ids), 1), np.int32)
    lib().om_cells_certified(grid._g, grid.ext.ravel(), len(grid.ext), ids, len(ids), k0, k_max, C.byref(m), ku)
    return _wrap(m), ku[: len(ids)]


def build_mesh(pts: np.ndarray, k: int, buff: float = 0.04, boundary: int = PERIODIC,
               hydro_only: bool = False, robust: bool = False, k_fallback: int = 0, expand_k: int = 0) -> Mesh:
    """The whole mesh build.  robust / k_fallback / expand_k: the moving-mesh extensions (om.h)."""
    pts = np.ascontiguousarray(pts, np.float64)
    m = _Mesh()
    L = lib()
    L.om_set_predicate_mode(1 if robust else 0)
    L.om_set_fallback_k(k_fallback)
    L.om_set_expand_k(expand_k)
    try:
        L.om_build_mesh(pts.shape[1], boundary, buff, k, pts.ravel(), len(pts), int(hydro_only), C.byref(m))
    finally:
        L.om_set_predicate_mode(0)
        L.om_set_fallback_k(0)
        L.om_set_expand_k(0)
    return _wrap(m)


def dt_cfl(mesh: Mesh, cfl: float, gamma: float, rho, vel, energy) -> float:
    return lib().om_dt_cfl(C.byref(mesh._c), cfl, gamma, np.ascontiguousarray(rho, np.float64),
                           np.ascontiguousarray(vel, np.float64).ravel(), np.ascontiguousarray(energy, np.float64))


def hydro_step_ref(mesh: Mesh, dt: float, gamma: float, rho, vel, energy):
    r = np.array(rho, np.float64, copy=True)
    v = np.array(vel, np.float64, copy=True)
    e = np.array(energy, np.float64, copy=True)
    vf = v.reshape(-1)
    nbox = lib().om_hydro_step_ref(C.byref(mesh._c), dt, gamma, r, vf, e)
    return r, vf.reshape(v.shape), e, nbox


def symmetric_area(mesh: Mesh):
    out = np.zeros(max(mesh.num_faces, 1))
    unp = lib().om_symmetric_area(C.byref(mesh._c), out)
    return out[: mesh.num_faces], unp


def reset_counters():
    lib().om_reset_counters()


def counters() -> dict:
    """Work counters since the last reset: KNN candidates, clip predicates, vertices created, cells."""
    out = np.zeros(4, np.int64)
    lib().om_get_counters(out)
    return dict(zip(("knn_candidates", "predicates", "new_vertices", "cells"), out.tolist()))


def prim_to_cons(mesh: Mesh, rho, vel, energy, deposit=None):
    """Conserved (mass, momentum, energy) per hydro cell on this mesh: m = rho V,
    p = (rho v) V, e = E V (+ deposit)."""
    V = mesh.volumes[: mesh.n_hydro]
    mass = rho * V
    mom = (rho[:, None] * vel) * V[:, None]
    en = energy * V
    if deposit is not None:
        en = en + deposit
    return mass, np.ascontiguousarray(mom), en


def step_moving(mesh: Mesh, cfl: float, gamma: float, boundary: int, x, mass, mom, energy, fixed_dt: float = 0.0):
    """One conserved moving-mesh step on copies; returns (dt, x, mass, mom, energy, n_unpaired)."""
    x = np.array(x, np.float64, copy=True)
    m = np.array(mass, np.float64, copy=True)
    p = np.array(mom, np.float64, copy=True)
    e = np.array(energy, np.float64, copy=True)
    unp = C.c_long(0)
    dt = lib().om_step_moving(C.byref(mesh._c), cfl, fixed_dt, gamma, boundary, x.reshape(-1), m,
                              p.reshape(-1), e, C.byref(unp))
    return dt, x, m, p, e, unp.value


def step_ale(mesh: Mesh, order: int, cfl: float, gamma: float, x, mass, mom, energy, fixed_dt: float = 0.0):
    """One moving-face step (order 1, or 2: MUSCL-Hancock) on copies, periodic boxes;
    returns (dt, x, mass, mom, energy, n_unpaired).  The mesh must come from build_mesh."""
    x = np.array(x, np.float64, copy=True)
    m = np.array(mass, np.float64, copy=True)
    p = np.array(mom, np.float64, copy=True)
    e = np.array(energy, np.float64, copy=True)
    unp = C.c_long(0)
    dt = lib().om_step_ale(C.byref(mesh._c), order, cfl, fixed_dt, gamma, x.reshape(-1), m, p.reshape(-1), e,
                           C.byref(unp))
    if dt < 0:
        raise ValueError("om_step_ale needs a mesh from build_mesh of a periodic box and order 1 or 2")
    return dt, x, m, p, e, unp.value
