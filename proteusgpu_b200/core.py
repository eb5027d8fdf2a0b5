"""Host-side mirror of the reference's knn:: / voronoi:: / hydro:: interface.

Each method forwards to one C ABI entry point of libproteus_gpu.so; the
reference function it stands for is named in its docstring.  Arrays are numpy
(float64 / uint32 / int32 / uint64), C-contiguous, in host memory.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import check

STATUS_SUCCESS = 4
STATUS_NOT_COMPUTED = 6


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _c64(a, dtype=np.float64):
    return np.ascontiguousarray(a, dtype=dtype)


@dataclass
class Mesh:
    """A mesh in the reference's VMesh layout (src/voronoi/voronoi.h:22-41):
    cells in input order (hydro ids first, then ghosts), faces CSR per cell.
    seeds and normal are 3-vectors even in 2D; status, cert_k and centroid are
    per-cell extras."""
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
    status: np.ndarray
    cert_k: np.ndarray
    centroid: np.ndarray

    @property
    def num_faces(self) -> int:
        return int(len(self.neighbor))


@dataclass
class SampledCells:
    """Cells of the current mesh read back by query slot (pgpu_sample_cells):
    extended ids, the neighbour row of the main clipping pass (n x k, list_len
    used), per-cell outputs (physical units) and the cells' faces as CSR."""
    slots: np.ndarray
    ext_id: np.ndarray
    list_len: np.ndarray
    lists: np.ndarray
    status: np.ndarray
    cert_k: np.ndarray
    volumes: np.ndarray
    centroid: np.ndarray
    face_ptr: np.ndarray
    neighbor: np.ndarray
    normal: np.ndarray
    area: np.ndarray


class Context:
    """One device context: a CUDA stream plus the device buffers of one mesh/simulation.

    dim, k: the reference's compile-time dimension and _K_ (Config.sh:4-34),
    here runtime parameters.  boundary: "periodic" (reference) or "reflective".
    flux: "reference" (stored inward normal, own face area, as riemann.cpp),
    "physical" (outward normal, face-pair-symmetric area), or, for moving-mesh
    steps in periodic boxes, "ale1" / "ale2" (faces moving with the generators,
    first / second order).  predicates:
    "reference" (a near-degenerate predicate fails the cell, cell.cpp:216-218) or
    "robust" (the vertex is kept).  k_fallback: moving-mesh steps recompute cells
    whose certificate does not close within k neighbours with this budget.
    precision: "fp64" (the reference's arithmetic) or "fp32" (local-frame FP32 clipping,
    FP64 re-clip of undecided cells, FP64 extraction; same mesh)."""

    def __init__(self, dim: int = 3, k: int = 190, boundary: str = "periodic", flux: str = "reference",
                 buff: float = 0.04, gamma: float = 5.0 / 3.0, device: int = 0, predicates: str = "reference",
                 k_fallback: int = 0, precision: str = "fp64"):
        L = _lib.load()
        p = _lib.Params()
        L.pgpu_default_params(C.byref(p))
        p.dim, p.k, p.buff, p.gamma, p.device = dim, k, buff, gamma, device
        p.boundary = {"periodic": 0, "reflective": 1}[boundary]
        p.flux_mode = {"reference": 0, "physical": 1, "ale1": 2, "ale2": 3}[flux]
        p.predicates = {"reference": 0, "robust": 1}[predicates]
        p.k_fallback = k_fallback
        p.precision = {"fp64": 0, "fp32": 1}[precision]
        h = C.c_void_p()
        rc = L.pgpu_create(C.byref(p), C.byref(h))
        if rc != 0:
            raise _lib.PGPUError(f"pgpu_create failed ({rc}: {_lib.ERRORS.get(rc, '?')})")
        self._h = h
        self.dim, self.k, self.boundary, self.flux, self.buff, self.gamma = dim, k, boundary, flux, buff, gamma
        self._L = L

    def close(self):
        if getattr(self, "_h", None):
            self._L.pgpu_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def stream(self) -> int:
        return int(self._L.pgpu_stream(self._h) or 0)

    # ---------------------------------------------------------------- knn::
    def knn(self, pts: np.ndarray) -> np.ndarray:
        """knn::init + knn::solve (src/knn/knn.cpp:16-234): (n, k) neighbour ids in input ids,
        ascending by (squared distance, id); UINT32_MAX where fewer than k exist."""
        pts = _c64(pts)
        n = len(pts)
        out = np.zeros((n, self.k), np.uint32)
        check(self._h, self._L.pgpu_knn(self._h, _ptr(pts), n, _ptr(out)), "pgpu_knn")
        return out

    def knn_sorted(self):
        """knn::get_points / get_permutation (src/knn/knn.cpp:445-455) of the last knn():
        (sorted points, perm sorted->input id, grid resolution)."""
        n = C.c_int64()
        self._L.pgpu_mesh_sizes(self._h, C.byref(n), None, None)
        pts = np.zeros((n.value, self.dim))
        perm = np.zeros(n.value, np.uint32)
        g = C.c_int()
        check(self._h, self._L.pgpu_knn_sorted(self._h, _ptr(pts), _ptr(perm), C.byref(g)), "pgpu_knn_sorted")
        return pts, perm, g.value

    # ------------------------------------------------------------ voronoi::
    def compute_periodic_mesh(self, pts: np.ndarray, download: bool = True) -> Mesh | None:
        """voronoi::compute_periodic_mesh (src/voronoi/periodic_mesh.cpp:44-184)."""
        pts = _c64(pts)
        ns, nf = C.c_int64(), C.c_int64()
        check(self._h, self._L.pgpu_periodic_mesh(self._h, _ptr(pts), len(pts), C.byref(ns), C.byref(nf)),
              "pgpu_periodic_mesh")
        return self.download_mesh() if download else None

    def compute_mesh(self, pts_unit: np.ndarray, download: bool = True) -> Mesh | None:
        """voronoi::compute_mesh (src/voronoi/voronoi.cpp:17-64) on points in the unit box."""
        pts = _c64(pts_unit)
        nf = C.c_int64()
        check(self._h, self._L.pgpu_compute_mesh(self._h, _ptr(pts), len(pts), C.byref(nf)), "pgpu_compute_mesh")
        return self.download_mesh() if download else None

    def mesh_sizes(self):
        ns, nh, nf = C.c_int64(), C.c_int64(), C.c_int64()
        self._L.pgpu_mesh_sizes(self._h, C.byref(ns), C.byref(nh), C.byref(nf))
        return ns.value, nh.value, nf.value

    def download_mesh(self) -> Mesh:
        """The device mesh in VMesh layout (unpermute_vmesh, src/voronoi/voronoi.cpp:212-333)."""
        n, nh, F = self.mesh_sizes()
        m = Mesh(self.dim, n, nh, np.zeros((n, 3)), np.zeros(n), np.zeros(n, np.uint64), np.zeros(n, np.uint64),
                 np.zeros(F, np.int32), np.zeros((F, 3)), np.zeros(F), np.zeros(n - nh, np.uint64),
                 np.zeros(n, np.int32), np.zeros(n, np.int32), np.zeros((n, 3)))
        check(self._h, self._L.pgpu_download_mesh(
            self._h, _ptr(m.seeds), _ptr(m.volumes), _ptr(m.face_counts), _ptr(m.face_ptr), _ptr(m.neighbor),
            _ptr(m.normal), _ptr(m.area), _ptr(m.ghost_ids), _ptr(m.status), _ptr(m.cert_k), _ptr(m.centroid)),
            "pgpu_download_mesh")
        return m

    def download_volumes(self) -> np.ndarray:
        """Volumes of the current mesh's cells in input order (hydro ids first), physical units."""
        n, _, _ = self.mesh_sizes()
        vol = np.zeros(n)
        check(self._h, self._L.pgpu_download_mesh(self._h, None, _ptr(vol), *([None] * 9)), "pgpu_download_mesh")
        return vol

    def download_points(self) -> np.ndarray:
        """The extended unit-box point set of the current mesh (hydro points, then ghosts)."""
        n, _, _ = self.mesh_sizes()
        out = np.zeros((n, self.dim))
        check(self._h, self._L.pgpu_download_points(self._h, _ptr(out)), "pgpu_download_points")
        return out

    def walked_slots(self) -> np.ndarray:
        """Query slots of the cells the last build certified by the grid walk."""
        cnt = C.c_int64()
        check(self._h, self._L.pgpu_walked_slots(self._h, None, 0, C.byref(cnt)), "pgpu_walked_slots")
        out = np.zeros(max(cnt.value, 1), np.uint32)
        check(self._h, self._L.pgpu_walked_slots(self._h, _ptr(out), len(out), C.byref(cnt)), "pgpu_walked_slots")
        return out[: cnt.value]

    def sample_cells(self, slots) -> SampledCells:
        """Cells of the current mesh by query slot, with their neighbour rows and faces."""
        slots = _c64(slots, np.uint32)
        n = len(slots)
        ext = np.zeros(n, np.uint32)
        ln = np.zeros(n, np.uint16)
        rows = np.zeros((n, self.k), np.uint32)
        st, ck = np.zeros(n, np.int32), np.zeros(n, np.int32)
        vol, cen = np.zeros(n), np.zeros((n, 3))
        fp = np.zeros(n + 1, np.uint64)
        args = [_ptr(ext), _ptr(ln), _ptr(rows), _ptr(st), _ptr(ck), _ptr(vol), _ptr(cen), _ptr(fp)]
        check(self._h, self._L.pgpu_sample_cells(self._h, _ptr(slots), n, *args, None, None, None, 0),
              "pgpu_sample_cells")
        F = int(fp[-1])
        nb, nrm, ar = np.zeros(max(F, 1), np.int32), np.zeros((max(F, 1), 3)), np.zeros(max(F, 1))
        check(self._h, self._L.pgpu_sample_cells(self._h, _ptr(slots), n, *args, _ptr(nb), _ptr(nrm), _ptr(ar),
                                                 max(F, 1)), "pgpu_sample_cells")
        return SampledCells(slots, ext, ln, rows, st, ck, vol, cen, fp.astype(np.int64), nb[:F], nrm[:F], ar[:F])

    def upload_mesh(self, m) -> None:
        """Makes a host VMesh (any object with the Mesh fields) the device mesh."""
        F = len(m.neighbor)
        check(self._h, self._L.pgpu_upload_mesh(
            self._h, m.n_seeds, m.n_hydro, F, _ptr(_c64(m.volumes)), _ptr(_c64(m.face_counts, np.uint64)),
            _ptr(_c64(m.face_ptr, np.uint64)), _ptr(_c64(m.neighbor, np.int32)), _ptr(_c64(m.normal)),
            _ptr(_c64(m.area)), _ptr(_c64(m.ghost_ids, np.uint64) if len(m.ghost_ids) else None)),
            "pgpu_upload_mesh")

    # -------------------------------------------------------------- hydro::
    def set_prim(self, rho, v, E) -> None:
        """hydro::init (src/hydro/finite_volume_solver.cpp:8-31)."""
        rho, v, E = _c64(rho), _c64(v), _c64(E)
        check(self._h, self._L.pgpu_set_prim(self._h, _ptr(rho), _ptr(v), _ptr(E), len(rho)), "pgpu_set_prim")

    def get_prim(self):
        _, nh, _ = self.mesh_sizes()
        rho, v, E = np.zeros(nh), np.zeros((nh, self.dim)), np.zeros(nh)
        check(self._h, self._L.pgpu_get_prim(self._h, _ptr(rho), _ptr(v), _ptr(E)), "pgpu_get_prim")
        return rho, v, E

    def dt_cfl(self, cfl: float) -> float:
        """hydro::dt_CFL (src/hydro/finite_volume_solver.cpp:151-186)."""
        dt = C.c_double()
        check(self._h, self._L.pgpu_dt_cfl(self._h, cfl, C.byref(dt)), "pgpu_dt_cfl")
        return dt.value

    def hydro_step(self, dt: float) -> None:
        """hydro::hydro_step (src/hydro/finite_volume_solver.cpp:43-123)."""
        check(self._h, self._L.pgpu_hydro_step(self._h, dt), "pgpu_hydro_step")

    # ------------------------------------------------------- moving mesh
    def sim_init(self, pos, rho, v, E, deposit=None) -> None:
        pos, rho, v, E = _c64(pos), _c64(rho), _c64(v), _c64(E)
        dep = None if deposit is None else _c64(deposit)
        check(self._h, self._L.pgpu_sim_init(self._h, _ptr(pos), _ptr(rho), _ptr(v), _ptr(E), _ptr(dep), len(pos)),
              "pgpu_sim_init")

    def ic_generate(self, spec: dict):
        """The initial condition of a generator spec (ics.IC.spec) made on the device and
        copied back: (pos, rho, vel, energy, deposit)."""
        s = _lib.ic_spec(spec)
        n = s.n_side ** s.dim if spec["kind"] in ("sod", "kh") else s.n
        pos, rho, v, E, dep = np.zeros((n, s.dim)), np.zeros(n), np.zeros((n, s.dim)), np.zeros(n), np.zeros(n)
        check(self._h, self._L.pgpu_ic_generate(self._h, C.byref(s), _ptr(pos), _ptr(rho), _ptr(v), _ptr(E),
                                                _ptr(dep)), "pgpu_ic_generate")
        return pos, rho, v, E, dep

    def sim_init_ic(self, spec: dict) -> None:
        """pgpu_sim_init from the initial condition of spec generated on the device."""
        s = _lib.ic_spec(spec)
        check(self._h, self._L.pgpu_sim_init_ic(self._h, C.byref(s)), "pgpu_sim_init_ic")

    def batch_init_ic(self, specs, buff, boundary) -> None:
        """pgpu_batch_init from per-instance generator specs, each generated on the device."""
        nb = len(specs)
        arr = (_lib.ICSpec * nb)(*[_lib.ic_spec(sp) for sp in specs])
        bf = np.ascontiguousarray(np.broadcast_to(np.asarray(buff, np.float64), (nb,)))
        bd = np.ascontiguousarray([_lib.BOUNDARY[b] if isinstance(b, str) else int(b) for b in
                                   np.broadcast_to(np.asarray(boundary, object), (nb,))], np.int32)
        check(self._h, self._L.pgpu_batch_init_ic(self._h, nb, C.cast(arr, C.c_void_p), _ptr(bf), _ptr(bd)),
              "pgpu_batch_init_ic")
        self._n_inst = nb

    def batch_init(self, counts, buff, gamma, boundary, pos, rho, v, E, deposit=None) -> None:
        """Independent simulations advanced together (extension): instance b owns the
        next counts[b] rows of pos/rho/v/E; buff, gamma, boundary ("periodic" or
        "reflective") per instance."""
        counts = np.ascontiguousarray(counts, np.int64)
        nb = len(counts)
        bf = np.ascontiguousarray(np.broadcast_to(np.asarray(buff, np.float64), (nb,)))
        gm = np.ascontiguousarray(np.broadcast_to(np.asarray(gamma, np.float64), (nb,)))
        bd = np.ascontiguousarray([_lib.BOUNDARY[b] if isinstance(b, str) else int(b) for b in
                                   np.broadcast_to(np.asarray(boundary, object), (nb,))], np.int32)
        pos, rho, v, E = _c64(pos), _c64(rho), _c64(v), _c64(E)
        dep = None if deposit is None else _c64(deposit)
        check(self._h, self._L.pgpu_batch_init(self._h, nb, _ptr(counts), _ptr(bf), _ptr(gm), _ptr(bd), _ptr(pos),
                                               _ptr(rho), _ptr(v), _ptr(E), _ptr(dep)), "pgpu_batch_init")
        self._n_inst = nb

    def autotune(self) -> dict:
        """Launch shapes for this workload (grid bin size, KNN and clipping block sizes),
        timed on mesh builds of the current state; cached per workload class."""
        t = _lib.Tuning()
        check(self._h, self._L.pgpu_autotune(self._h, C.byref(t)), "pgpu_autotune")
        return {f: getattr(t, f) for f, _ in t._fields_}

    def set_tuning(self, ppb: float = 2.0, knn_warps: int = 4, clip_warps: int = 4, clip_thread: bool = False,
                   knn_thread: int = 0):
        """Launch shapes set directly (what pgpu_autotune would pick)."""
        t = _lib.Tuning(ppb=ppb, knn_warps=knn_warps, clip_warps=clip_warps, clip_thread=int(clip_thread),
                        knn_thread=int(knn_thread))
        check(self._h, self._L.pgpu_set_tuning(self._h, C.byref(t)), "pgpu_set_tuning")

    def batch_dt(self) -> np.ndarray:
        """Each instance's dt of the last step."""
        out = np.zeros(getattr(self, "_n_inst", 1))
        check(self._h, self._L.pgpu_batch_dt(self._h, _ptr(out)), "pgpu_batch_dt")
        return out

    def sim_step(self, cfl: float = 0.3, fixed_dt: float = 0.0, want_dt: bool = True) -> float | None:
        dt = C.c_double()
        check(self._h, self._L.pgpu_sim_step(self._h, cfl, fixed_dt, C.byref(dt) if want_dt else None),
              "pgpu_sim_step")
        return dt.value if want_dt else None

    def sim_step_host(self, cfl, fixed_dt, pos, mass, mom, energy) -> float:
        """One step with the state in (pinned or pageable) host arrays, updated in place."""
        dt = C.c_double()
        check(self._h, self._L.pgpu_sim_step_host(self._h, cfl, fixed_dt, _ptr(pos), _ptr(mass), _ptr(mom),
                                                  _ptr(energy), C.byref(dt)), "pgpu_sim_step_host")
        return dt.value

    def sim_get(self):
        _, nh, _ = self.mesh_sizes()
        pos, mass, mom, en = np.zeros((nh, self.dim)), np.zeros(nh), np.zeros((nh, self.dim)), np.zeros(nh)
        check(self._h, self._L.pgpu_sim_get(self._h, _ptr(pos), _ptr(mass), _ptr(mom), _ptr(en)), "pgpu_sim_get")
        return pos, mass, mom, en

    def sim_set(self, pos=None, mass=None, mom=None, energy=None) -> None:
        arrs = [None if a is None else _c64(a) for a in (pos, mass, mom, energy)]
        check(self._h, self._L.pgpu_sim_set(self._h, *[_ptr(a) for a in arrs]), "pgpu_sim_set")

    def stats(self) -> dict:
        s = _lib.Stats()
        check(self._h, self._L.pgpu_sim_stats(self._h, C.byref(s)), "pgpu_sim_stats")
        return {f: (list(getattr(s, f)) if f in ("total_mom", "clip_split_ms") else getattr(s, f))
                for f, _ in s._fields_}

    # ---- learned neighbour budget (extension; the reference has one _K_ for all cells)
    def kbudget_enable(self, train_steps: int = 3, iters_per_step: int = 64, quantile: float = 0.99,
                       seed: int = 1) -> None:
        """Per-cell K from the device MLP on every moving-mesh step after train_steps
        plain steps that train it; rejected proposals are recomputed at the plain K."""
        check(self._h, self._L.pgpu_kbudget_enable(self._h, train_steps, iters_per_step, quantile, seed),
              "pgpu_kbudget_enable")

    def kbudget_stats(self) -> dict:
        s = _lib.KBudgetInfo()
        check(self._h, self._L.pgpu_kbudget_stats(self._h, C.byref(s)), "pgpu_kbudget_stats")
        return {f: getattr(s, f) for f, _ in s._fields_}

    def kbudget_weights(self, set_to: np.ndarray | None = None) -> np.ndarray:
        """The MLP's FP32 master parameters (1542 floats); optionally replaces them first."""
        out = np.zeros(_lib.KB_NPARAM, np.float32)
        src = None if set_to is None else np.ascontiguousarray(set_to, np.float32)
        if src is not None and src.size != _lib.KB_NPARAM:
            raise ValueError("expected 1542 parameters")
        check(self._h, self._L.pgpu_kbudget_weights(self._h, None, None if src is None else _ptr(src)),
              "pgpu_kbudget_weights")
        check(self._h, self._L.pgpu_kbudget_weights(self._h, _ptr(out), None), "pgpu_kbudget_weights")
        return out

    def mlp_forward(self, feat: np.ndarray):
        """Device MLP on n x 8 features: (logits n x 6, proposed K per row)."""
        f = np.ascontiguousarray(feat, np.float32)
        n = len(f)
        logits, kq = np.zeros((n, 6), np.float32), np.zeros(n, np.uint16)
        check(self._h, self._L.pgpu_mlp_forward(self._h, _ptr(f), n, _ptr(logits), _ptr(kq)), "pgpu_mlp_forward")
        return logits, kq

    def mlp_grad(self, feat: np.ndarray, labels: np.ndarray):
        """Gradient (1542 floats) and value of the mean cross-entropy at the current weights."""
        f = np.ascontiguousarray(feat, np.float32)
        y = np.ascontiguousarray(labels, np.int32)
        g = np.zeros(_lib.KB_NPARAM, np.float32)
        loss = C.c_float()
        check(self._h, self._L.pgpu_mlp_grad(self._h, _ptr(f), _ptr(y), len(f), _ptr(g), C.byref(loss)),
              "pgpu_mlp_grad")
        return g, loss.value

    def enable_timing(self, on: bool = True) -> None:
        check(self._h, self._L.pgpu_enable_timing(self._h, int(on)), "pgpu_enable_timing")

    def stage_times(self):
        """Device ms of the last mesh/step: ghosts, sort, knn, clip, hydro."""
        a = (C.c_float * 5)()
        check(self._h, self._L.pgpu_stage_times(self._h, a), "pgpu_stage_times")
        return list(a)
