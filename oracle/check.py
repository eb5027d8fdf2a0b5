"""Checks of the CUDA path's meshes and states against the oracle at full size.

TEST INFRASTRUCTURE ONLY: used by tests/ and by bench.py's checking leg (after
the timed region) as the checker; the product never imports it.

sampled_cells():  a mesh of any size is read back in part (pgpu_download_points,
pgpu_sample_cells) and a sample of its cells, stratified to include cells the
GPU certified by its grid walk, is recomputed by the oracle on the GPU's own
extended point set: exact KNN rows (om_grid_knn, the same lists as the
restatement of src/knn/knn.cpp:225-315) and clipping with the reference's
algorithm at a budget large enough to certify each cell (om_cells_certified,
src/voronoi/voronoi.cpp:115-155 with a larger _K_).  When the positions the
step started from are given, the extended point set itself is rebuilt by the
oracle (src/voronoi/periodic_mesh.cpp:44-126) and compared bit for bit.

oracle_moving_run():  the whole moving-mesh run on the oracle (hydro-only
builds with the growing budget, om_step_moving), for the density error of a
full step sequence.
"""
from __future__ import annotations

import numpy as np

import oracle as om

# Per-field tolerances of a sampled cell against the oracle.  Topology is exact.
# Cells clipped from their neighbour list clip the same planes in the same order as the
# oracle, but hold their vertices in another order inside the cell, which moves the fan
# sums of areas and volumes at rounding level; cells certified by the grid walk clip in
# another order (the list's head, then grid order) in the seed's local frame.  The cells
# of the clustered workloads are as small as 2e-4 of the box, while their vertex
# coordinates are O(1), so a rounding of 1e-16 in a coordinate is ~5e-13 of the cell's
# size per term of a volume's ~30-term sum:
#   volume: relative, 1e-10;
#   area: a face's error relative to its cell's largest face (a sliver face's own
#         relative error grows as the face shrinks; its absolute error does not), 1e-10;
#   centroid: absolute in the unit box, 1e-11;  normal: absolute, 0 (same plane equation
#   and normalisation) for listed cells, 1e-12 for walked cells.
TOL = {"volume": 1e-10, "area": 1e-10, "centroid_abs": 1e-11, "normal_abs": 0.0,
       "volume_walk": 1e-10, "area_walk": 1e-10, "centroid_walk_abs": 1e-11, "normal_walk_abs": 1e-12}


def _rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    if a.size == 0:
        return 0.0
    return float((np.abs(a - b) / np.maximum(np.abs(b), 1e-300)).max())


def sampled_cells(ctx, *, n_random: int = 20000, n_walked: int = 2000, seed: int = 0, k_max: int = 1 << 16,
                  pos_before=None, buff: float | None = None, boundary: str = "periodic") -> dict:
    """Compares a stratified sample of the current mesh's hydro cells with the oracle.

    Topology is compared exactly: status, and each cell's face neighbours (extended
    ids) in stored order for cells clipped from their list, as a set for walked cells;
    the main pass's neighbour rows are compared with the oracle's exact KNN rows of
    the same length.  Geometry within TOL.  Returns a report dict."""
    buff = ctx.buff if buff is None else buff
    ext = ctx.download_points()
    n_ext, n_hydro, _ = ctx.mesh_sizes()
    rep = {"n_hydro": int(n_hydro), "n_ext": int(n_ext)}
    if pos_before is not None:
        b = om.PERIODIC if boundary == "periodic" else om.REFLECTIVE
        ext_o, _src, _code = om.ghosts(np.asarray(pos_before, np.float64), buff, b)
        rep["ghosts_identical"] = bool(ext_o.shape == ext.shape and np.array_equal(ext_o, ext))
    rng = np.random.default_rng(seed)
    rand = rng.choice(n_hydro, size=min(n_random, n_hydro), replace=False).astype(np.uint32)
    walked_all = ctx.walked_slots()
    walked = (rng.choice(walked_all, size=min(n_walked, len(walked_all)), replace=False)
              if len(walked_all) else np.zeros(0, np.uint32))
    slots = np.unique(np.concatenate([rand, walked.astype(np.uint32)]))
    is_walk = np.isin(slots, walked_all)
    g = ctx.sample_cells(slots)
    ids = g.ext_id.astype(np.int64)
    grid = om.Grid(ext)
    o, k_used = om.cells_certified(grid, ids, ctx.k, k_max)
    # neighbour rows of the main pass against the oracle's exact rows of the same length
    lmax = int(g.list_len.max()) if len(ids) else 0
    rows_o = grid.knn(ids, lmax) if lmax else np.zeros((len(ids), 0), np.uint32)
    row_bad = 0
    for i in range(len(ids)):
        L = int(g.list_len[i])
        row_bad += not np.array_equal(g.lists[i, :L], rows_o[i, :L])
    grid.close()
    us = 1.0 + 2.0 * buff
    dim = ctx.dim
    vscale = us * us if dim == 2 else us * us * us
    ascale = us if dim == 2 else us * us
    st_g, st_o = g.status, o.status
    oracle_ok = st_o == om.SUCCESS
    status_bad = int(((st_g == om.SUCCESS) != oracle_ok).sum())
    topo_bad = order_bad = 0
    vol_err = {False: 0.0, True: 0.0}
    area_err = {False: 0.0, True: 0.0}    # per face, relative to the cell's largest face (the tolerance)
    area_face = {False: 0.0, True: 0.0}   # per face, relative to the face itself (reported)
    cen_err = {False: 0.0, True: 0.0}
    nrm_err = {False: 0.0, True: 0.0}
    ok_both = 0
    for i in range(len(ids)):
        if not (st_g[i] == om.SUCCESS and oracle_ok[i]):
            topo_bad += (st_g[i] == om.SUCCESS) != oracle_ok[i]
            continue
        ok_both += 1
        w = bool(is_walk[i])
        fg = slice(int(g.face_ptr[i]), int(g.face_ptr[i + 1]))
        fo = slice(int(o.face_ptr[i]), int(o.face_ptr[i] + o.face_counts[i]))
        nb_g, nb_o = g.neighbor[fg], o.neighbor[fo]
        if not np.array_equal(np.sort(nb_g), np.sort(nb_o)):
            topo_bad += 1
            continue
        if w:
            pg, po = np.argsort(nb_g, kind="stable"), np.argsort(nb_o, kind="stable")
        else:
            if not np.array_equal(nb_g, nb_o):
                order_bad += 1
                topo_bad += 1
                continue
            pg = po = np.arange(len(nb_g))
        ag, ao = g.area[fg][pg], ascale * o.area[fo][po]
        if len(ao):
            area_err[w] = max(area_err[w], float(np.abs(ag - ao).max() / max(np.abs(ao).max(), 1e-300)))
            area_face[w] = max(area_face[w], _rel(ag, ao))
        nrm_err[w] = max(nrm_err[w], float(np.abs(g.normal[fg][pg] - o.normal[fo][po]).max()) if len(pg) else 0.0)
        vol_err[w] = max(vol_err[w], _rel(g.volumes[i], vscale * o.volumes[i]))
        co = (o.centroid[i, :dim] - 0.5) * us + 0.5
        cen_err[w] = max(cen_err[w], float(np.abs(g.centroid[i, :dim] - co).max()))
    rep.update({
        "cells_sampled": int(len(ids)), "walked_sampled": int(is_walk.sum()), "walked_total": int(len(walked_all)),
        "status_mismatch": status_bad, "topology_mismatch": int(topo_bad), "face_order_mismatch": int(order_bad),
        "neighbour_list_mismatch": int(row_bad), "compared_cells": int(ok_both),
        "oracle_unresolved": int((~oracle_ok).sum()), "oracle_budget_max": int(k_used.max()) if len(ids) else 0,
        "tolerances": dict(TOL),
        "volume_rel_max": vol_err[False], "area_rel_max": area_err[False], "centroid_abs_max": cen_err[False],
        "normal_abs_max": nrm_err[False], "area_rel_to_face_max": area_face[False],
        "walked_area_rel_to_face_max": area_face[True],
        "walked_volume_rel_max": vol_err[True], "walked_area_rel_max": area_err[True],
        "walked_centroid_abs_max": cen_err[True], "walked_normal_abs_max": nrm_err[True],
    })
    rep["within_tolerance"] = bool(
        rep["topology_mismatch"] == 0 and rep["status_mismatch"] == 0 and rep["neighbour_list_mismatch"] == 0
        and rep.get("ghosts_identical", True) and rep["volume_rel_max"] <= TOL["volume"]
        and rep["area_rel_max"] <= TOL["area"] and rep["centroid_abs_max"] <= TOL["centroid_abs"]
        and rep["normal_abs_max"] <= TOL["normal_abs"] and rep["walked_volume_rel_max"] <= TOL["volume_walk"]
        and rep["walked_area_rel_max"] <= TOL["area_walk"]
        and rep["walked_centroid_abs_max"] <= TOL["centroid_walk_abs"]
        and rep["walked_normal_abs_max"] <= TOL["normal_walk_abs"])
    return rep


def oracle_moving_run(ic, k: int, buff: float, boundary: str, steps: int, cfl: float = 0.3,
                      k_max: int = 1 << 16, robust: bool = False):
    """The moving-mesh run of an initial condition on the oracle: a hydro-only mesh per
    step (budget k, growing up to k_max for cells whose certificate does not close),
    then om_step_moving.  Returns (dts, x, mass, mom, energy, hydro volumes of the
    last step's mesh)."""
    b = om.PERIODIC if boundary == "periodic" else om.REFLECTIVE
    kw = dict(buff=buff, boundary=b, hydro_only=True, robust=robust, expand_k=k_max)
    m = om.build_mesh(ic.pos, k, **kw)
    mass, mom, en = om.prim_to_cons(m, ic.rho, ic.vel, ic.energy, ic.deposit)
    m.free()
    x = ic.pos.copy()
    dts, vol = [], None
    for _ in range(steps):
        m = om.build_mesh(x, k, **kw)
        vol = m.volumes[: m.n_hydro].copy()
        dt, x, mass, mom, en, _unp = om.step_moving(m, cfl, ic.gamma, b, x, mass, mom, en)
        m.free()
        dts.append(dt)
    return dts, x, mass, mom, en, vol


def state_errors(gpu, ora) -> dict:
    """Relative L1 errors of a GPU run against the oracle's: density (mass over the
    last step's volume), mass, momentum, energy, position; the time steps' largest
    relative difference."""
    dts_g, x_g, m_g, p_g, e_g, v_g = gpu
    dts_o, x_o, m_o, p_o, e_o, v_o = ora

    def l1(a, b):
        a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
        return float(np.abs(a - b).sum() / max(np.abs(b).sum(), 1e-300))

    rho_g, rho_o = m_g / v_g, m_o / v_o
    return {"density_l1_rel": l1(rho_g, rho_o), "mass_l1_rel": l1(m_g, m_o), "momentum_l1_rel": l1(p_g, p_o),
            "energy_l1_rel": l1(e_g, e_o), "position_l1_rel": l1(x_g, x_o),
            "dt_rel_max": _rel(dts_g, dts_o), "cells_differing": int(
                (~((m_g == m_o) & (e_g == e_o) & (x_g == x_o).all(axis=1) & (p_g == p_o).all(axis=1))).sum())}
