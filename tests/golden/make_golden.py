"""Generates the golden fixtures in tests/golden/ from the reference itself.

The reference has no golden vectors of its own (its CI only builds and runs a
dry run), so the fixtures here are outputs of the reference's own hot-path code,
compiled from its sources by oracle/Makefile (``make -C oracle ref REF=<reference tree>``) and run
in-process through oracle/ref_driver.cpp on small seeded inputs.

Run from the repository root in a checkout where the reference tree is
available:  python tests/golden/make_golden.py
Outputs are committed; tests never need the reference tree.
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import refbuild as rb  # noqa: E402
from proteusgpu_b200 import ics  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def mesh_arrays(m, prefix, cells=None):
    """Full VMesh arrays, or only the listed cells' rows (with their face lists)."""
    d = {}
    if cells is None:
        d[prefix + "volumes"] = m.volumes
        d[prefix + "face_counts"] = m.face_counts.astype(np.int32)
        d[prefix + "neighbor"] = m.neighbor
        d[prefix + "normal"] = m.normal
        d[prefix + "area"] = m.area
        d[prefix + "seeds"] = m.seeds
        d[prefix + "ghost_ids"] = m.ghost_ids
    else:
        cells = np.asarray(cells)
        fl = [np.arange(m.face_ptr[c], m.face_ptr[c] + m.face_counts[c]) for c in cells]
        fidx = np.concatenate(fl) if fl else np.zeros(0, np.int64)
        d[prefix + "cells"] = cells
        d[prefix + "volumes"] = m.volumes[cells]
        d[prefix + "face_counts"] = m.face_counts[cells].astype(np.int32)
        d[prefix + "neighbor"] = m.neighbor[fidx]
        d[prefix + "normal"] = m.normal[fidx]
        d[prefix + "area"] = m.area[fidx]
        d[prefix + "seeds"] = m.seeds[cells]
    d[prefix + "n_seeds"] = np.int64(m.n_seeds)
    d[prefix + "n_hydro"] = np.int64(m.n_hydro)
    d[prefix + "num_faces"] = np.int64(m.num_faces)
    d[prefix + "volume_sum_hydro"] = np.float64(m.volumes[: m.n_hydro].sum())
    return d


def main():
    # 1. 2D: 40x40 jittered lattice, K=16, periodic ghosts (buff 0.08), full mesh + 3 hydro steps
    pts2 = ics.jittered_lattice(40, 2, 0.1, np.random.default_rng(11))
    gamma = 1.4
    m2 = rb.periodic_mesh(pts2, 16, buff=0.08, gamma=gamma, keep_handle=True)
    rng = np.random.default_rng(12)
    n2 = len(pts2)
    rho = 1.0 + 0.5 * rng.random(n2)
    vel = 0.1 * rng.standard_normal((n2, 2))
    E = 2.0 + rng.random(n2) + 0.5 * rho * (vel ** 2).sum(1)
    dt = rb.dt_cfl(2, 16, m2.handle, 0.3, rho, vel, E, gamma)
    r, v, e = rho, vel, E
    for _ in range(3):
        r, v, e = rb.hydro_step(2, 16, m2.handle, dt, r, v, e, gamma)
    rb.free_handle(2, 16, m2.handle)
    d = {"pts2": pts2, "rho0": rho, "vel0": vel, "E0": E, "dt2": np.float64(dt), "rho3": r, "vel3": v, "E3": e}
    d.update(mesh_arrays(m2, "m2_"))
    # statuses of compute_mesh's call sequence on 1,500 uniform unit-box points (some fail at K=16)
    ext2 = ics.uniform_points(1500, 2, 16)
    cm = rb.compute_mesh(ext2, 16)
    d["cm2_status"] = cm.status
    d["cm2_face_counts"] = cm.face_counts.astype(np.int32)
    d["cm2_neighbor"] = cm.neighbor
    d["cm2_area"] = cm.area
    d["cm2_volumes"] = cm.volumes
    np.savez_compressed(os.path.join(OUT, "ref_2d_k16.npz"), **d)

    # 2. 3D: 12,000 uniform points, K=64 and K=190, periodic ghosts (buff 0.15); 300 sampled cells
    pts3 = ics.uniform_points(12000, 3, 13)
    d = {"pts3": pts3}
    for k in (64, 190):
        m3 = rb.periodic_mesh(pts3, k, buff=0.15)
        sample = np.random.default_rng(14).choice(m3.n_hydro, 300, replace=False)
        d.update(mesh_arrays(m3, f"m3k{k}_", cells=np.sort(sample)))
        d[f"m3k{k}_zero_volume_hydro"] = np.int64((m3.volumes[: m3.n_hydro] == 0).sum())
    # KNN lists of 200 sampled points of the extended set (input ids)
    ext3 = (pts3 - 0.5) / (1 + 2 * 0.15) + 0.5
    kl = rb.knn(ext3, 64)
    qs = np.sort(np.random.default_rng(15).choice(len(ext3), 200, replace=False))
    d["knn_q"] = qs
    d["knn_k64"] = kl[qs]
    np.savez_compressed(os.path.join(OUT, "ref_3d.npz"), **d)
    for f in ("ref_2d_k16.npz", "ref_3d.npz"):
        print(f, os.path.getsize(os.path.join(OUT, f)))


if __name__ == "__main__":
    main()
