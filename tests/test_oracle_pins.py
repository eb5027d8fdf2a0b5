"""The C restatement oracle against the reference itself (CPU).

Two pins: (1) the committed golden fixtures, which were produced by the
reference's own code (tests/golden/make_golden.py); (2) when the reference build
in oracle/_ref is present, a direct bit-for-bit comparison on fresh inputs.
"""
import numpy as np
import pytest

import oracle as om
from conftest import ref_available
from proteusgpu_b200 import ics


def test_oracle_2d_mesh_matches_golden(golden2):
    d = golden2
    m = om.build_mesh(d["pts2"], 16, buff=0.08)
    assert m.n_seeds == d["m2_n_seeds"] and m.num_faces == d["m2_num_faces"]
    assert (m.status == 4).all()
    for f in ("volumes", "normal", "area", "seeds"):
        assert np.array_equal(getattr(m, f), d["m2_" + f]), f
    assert np.array_equal(m.face_counts, d["m2_face_counts"])
    assert np.array_equal(m.neighbor, d["m2_neighbor"])
    assert np.array_equal(m.ghost_ids, d["m2_ghost_ids"])


def test_oracle_2d_hydro_matches_golden(golden2):
    d = golden2
    m = om.build_mesh(d["pts2"], 16, buff=0.08)
    dt = om.dt_cfl(m, 0.3, 1.4, d["rho0"], d["vel0"], d["E0"])
    assert dt == d["dt2"]
    r, v, e = d["rho0"], d["vel0"], d["E0"]
    for _ in range(3):
        r, v, e, nbox = om.hydro_step_ref(m, dt, 1.4, r, v, e)
        assert nbox == 0
    assert np.array_equal(r, d["rho3"]) and np.array_equal(v, d["vel3"]) and np.array_equal(e, d["E3"])


def test_oracle_compute_mesh_status_matches_golden(golden2):
    d = golden2
    ext = ics.uniform_points(1500, 2, 16)
    kl = om.knn(ext, 16)
    m = om.cells(ext, len(ext), kl)
    assert np.array_equal(m.status, d["cm2_status"])
    assert np.array_equal(m.face_counts, d["cm2_face_counts"])
    assert np.array_equal(m.neighbor, d["cm2_neighbor"])
    assert np.array_equal(m.area, d["cm2_area"])
    assert np.array_equal(m.volumes, d["cm2_volumes"])
    assert (m.status != 4).sum() > 0  # the record includes uncertified cells


@pytest.mark.parametrize("k", [64, 190])
def test_oracle_3d_sampled_cells_match_golden(golden3, k):
    d = golden3
    m = om.build_mesh(d["pts3"], k, buff=0.15)
    p = f"m3k{k}_"
    assert m.n_seeds == d[p + "n_seeds"] and m.num_faces == d[p + "num_faces"]
    assert int((m.volumes[: m.n_hydro] == 0).sum()) == d[p + "zero_volume_hydro"]
    cells = d[p + "cells"]
    assert np.array_equal(m.volumes[cells], d[p + "volumes"])
    assert np.array_equal(m.face_counts[cells], d[p + "face_counts"])
    fidx = np.concatenate([np.arange(m.face_ptr[c], m.face_ptr[c] + m.face_counts[c]) for c in cells])
    assert np.array_equal(m.neighbor[fidx], d[p + "neighbor"])
    assert np.array_equal(m.area[fidx], d[p + "area"])
    assert np.array_equal(m.normal[fidx], d[p + "normal"])
    assert m.volumes[: m.n_hydro].sum() == d[p + "volume_sum_hydro"]


def test_oracle_knn_matches_golden(golden3):
    d = golden3
    ext = (d["pts3"] - 0.5) / (1 + 2 * 0.15) + 0.5
    kl = om.knn(ext, 64)
    assert np.array_equal(kl[d["knn_q"]], d["knn_k64"])


@pytest.mark.skipif(not ref_available(2, 20), reason="reference build oracle/_ref not present")
def test_oracle_bitexact_vs_reference_2d_sod():
    import refbuild as rb
    ic = ics.sod_2d(n_side=60, seed=21)
    r = rb.periodic_mesh(ic.pos, 20, buff=0.06, gamma=1.4)
    o = om.build_mesh(ic.pos, 20, buff=0.06)
    for f in ("seeds", "volumes", "face_counts", "face_ptr", "neighbor", "normal", "area", "ghost_ids"):
        assert np.array_equal(getattr(r, f), getattr(o, f)), f


@pytest.mark.skipif(not ref_available(3, 32), reason="reference build oracle/_ref not present")
def test_oracle_bitexact_vs_reference_3d_failing_cells():
    """K=32 in 3D leaves many cells uncertified: failed cells must agree too."""
    import refbuild as rb
    pts = ics.uniform_points(13000, 3, 22)
    ext = np.ascontiguousarray((pts - 0.5) / 1.2 + 0.5)
    r = rb.compute_mesh(ext, 32)
    o = om.cells(ext, len(ext), om.knn(ext, 32))
    assert np.array_equal(r.status, o.status)
    assert (r.status != 4).sum() > 1000
    for f in ("volumes", "face_counts", "neighbor", "normal", "area"):
        assert np.array_equal(getattr(r, f), getattr(o, f)), f


@pytest.mark.skipif(not ref_available(3, 64), reason="reference build oracle/_ref not present")
def test_oracle_knn_bitexact_vs_reference():
    import refbuild as rb
    pts = ics.uniform_points(14000, 3, 23)
    assert np.array_equal(rb.knn(pts, 64), om.knn(pts, 64))
