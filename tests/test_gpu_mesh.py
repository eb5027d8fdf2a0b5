"""GPU mesh parity: the CUDA path through the C ABI against the oracle (same seeded inputs).

Topology (statuses, face counts, ordered neighbour ids) must be identical;
normals, 2D edge lengths and seeds bit-identical; 3D areas, volumes and
centroids within the tolerances in tests/helpers.py.
"""
import numpy as np
import pytest

import oracle as om
from helpers import TOL, assert_same_topology, rel_err
from proteusgpu_b200 import Context, ics

pytestmark = pytest.mark.gpu


def check_fields(g, o, dim, floor_frac=1e-9):
    """floor_frac: values below floor_frac x median count as zero-size (degenerate faces)."""
    ok = np.asarray(o.status) == 4
    assert np.array_equal(g.normal, o.normal)
    if dim == 2:
        assert np.array_equal(g.area, o.area)
        assert rel_err(g.volumes, o.volumes) <= TOL["volume_2d"]
    else:
        assert rel_err(g.area, o.area, floor_frac) <= TOL["area_3d"]
        assert rel_err(g.volumes[ok], o.volumes[ok], floor_frac) <= TOL["volume_3d"]
    assert np.array_equal(g.seeds, o.seeds)
    assert np.array_equal(np.asarray(g.cert_k)[ok], np.asarray(o.cert_k)[ok])
    assert np.abs(g.centroid[ok] - o.centroid[ok]).max() <= TOL["centroid"]


@pytest.mark.parametrize("k", [16, 20, 24, 32])
def test_sod_2d_periodic_mesh(k):
    ic = ics.sod_2d()
    with Context(dim=2, k=k, gamma=1.4) as ctx:
        g = ctx.compute_periodic_mesh(ic.pos)
    o = om.build_mesh(ic.pos, k)
    assert_same_topology(g, o)
    assert np.array_equal(g.ghost_ids.astype(np.int64), o.ghost_ids)
    check_fields(g, o, 2)
    assert abs(g.volumes[: g.n_hydro].sum() - 1.0) < 1e-12


def test_sod_2d_reflective_mesh():
    ic = ics.sod_2d()
    with Context(dim=2, k=16, boundary="reflective", gamma=1.4) as ctx:
        g = ctx.compute_periodic_mesh(ic.pos)
    o = om.build_mesh(ic.pos, 16, boundary=om.REFLECTIVE)
    assert_same_topology(g, o)
    check_fields(g, o, 2)


def test_golden_2d_full_mesh(golden2):
    d = golden2
    with Context(dim=2, k=16, buff=0.08, gamma=1.4) as ctx:
        g = ctx.compute_periodic_mesh(d["pts2"])
    assert g.n_seeds == d["m2_n_seeds"] and g.num_faces == d["m2_num_faces"]
    assert np.array_equal(g.face_counts.astype(np.int32), d["m2_face_counts"])
    assert np.array_equal(g.neighbor, d["m2_neighbor"])
    assert np.array_equal(g.normal, d["m2_normal"]) and np.array_equal(g.area, d["m2_area"])
    assert np.array_equal(g.seeds, d["m2_seeds"])
    assert rel_err(g.volumes, d["m2_volumes"]) <= TOL["volume_2d"]


@pytest.mark.parametrize("k", [64, 190])
def test_golden_3d_sampled_cells(golden3, k):
    d, p = golden3, f"m3k{k}_"
    with Context(dim=3, k=k, buff=0.15) as ctx:
        g = ctx.compute_periodic_mesh(d["pts3"])
    assert g.n_seeds == d[p + "n_seeds"] and g.num_faces == d[p + "num_faces"]
    assert int((g.volumes[: g.n_hydro] == 0).sum()) == d[p + "zero_volume_hydro"]
    cells = d[p + "cells"]
    fp, fc = g.face_ptr.astype(np.int64), g.face_counts.astype(np.int64)
    fidx = np.concatenate([np.arange(fp[c], fp[c] + fc[c]) for c in cells])
    assert np.array_equal(g.face_counts[cells].astype(np.int32), d[p + "face_counts"])
    assert np.array_equal(g.neighbor[fidx], d[p + "neighbor"])
    assert np.array_equal(g.normal[fidx], d[p + "normal"])
    assert rel_err(g.area[fidx], d[p + "area"]) <= TOL["area_3d"]
    assert rel_err(g.volumes[cells], d[p + "volumes"]) <= TOL["volume_3d"]
    assert abs(g.volumes[: g.n_hydro].sum() - d[p + "volume_sum_hydro"]) <= 1e-12


def test_golden_compute_mesh_statuses(golden2):
    """compute_mesh on unit-box points where some cells fail the certificate at K=16."""
    d = golden2
    pts = ics.uniform_points(1500, 2, 16)
    with Context(dim=2, k=16) as ctx:
        g = ctx.compute_mesh(pts)
    assert np.array_equal(g.status, d["cm2_status"])
    assert np.array_equal(g.face_counts.astype(np.int32), d["cm2_face_counts"])
    assert np.array_equal(g.neighbor, d["cm2_neighbor"])
    assert np.array_equal(g.area, d["cm2_area"])
    assert rel_err(g.volumes, d["cm2_volumes"]) <= TOL["volume_2d"]


@pytest.mark.parametrize("k", [64, 190])
def test_uniform_3d_periodic_mesh(k):
    pts = ics.uniform_points(20000, 3, 7)
    with Context(dim=3, k=k, buff=0.1) as ctx:
        g = ctx.compute_periodic_mesh(pts)
    o = om.build_mesh(pts, k, buff=0.1)
    assert_same_topology(g, o)
    check_fields(g, o, 3)


def test_uniform_3d_reflective_mesh():
    pts = ics.uniform_points(15000, 3, 8)
    with Context(dim=3, k=190, buff=0.1, boundary="reflective") as ctx:
        g = ctx.compute_periodic_mesh(pts)
    o = om.build_mesh(pts, 190, buff=0.1, boundary=om.REFLECTIVE)
    assert_same_topology(g, o, failure_codes_may_differ=True)
    check_fields(g, o, 3)


@pytest.mark.parametrize("dim", [2, 3])
def test_robust_predicates_reflective(dim):
    """Robust predicate mode on mirror walls: no cell fails, same topology as the oracle."""
    if dim == 2:
        pts, k, buff = ics.sod_2d().pos, 16, 0.04
    else:
        pts, k, buff = ics.uniform_points(15000, 3, 8), 190, 0.1
    with Context(dim=dim, k=k, buff=buff, boundary="reflective", predicates="robust") as ctx:
        ctx.sim_init(pts, np.ones(len(pts)), np.zeros_like(pts), np.ones(len(pts)))
        g = ctx.download_mesh()
    o = om.build_mesh(pts, k, buff=buff, boundary=om.REFLECTIVE, hydro_only=True, robust=True)
    nh = o.n_hydro
    if dim == 2:  # in 2D every mirror degeneracy resolves; in 3D a few wall cells still fail
        assert (o.status[:nh] == 4).all()
        assert abs(g.volumes[:nh].sum() - 1.0) < 1e-11
    assert_same_topology(g, o)
    if dim == 2:
        check_fields(g, o, dim)
        return
    # 3D mirror walls leave exactly-degenerate faces whose computed areas are pure rounding
    # (a sum of nearly cancelling fan triangles), and nearly degenerate vertices (mirror
    # images are cospherical) whose rounding is amplified: areas are compared as an
    # absolute error on the scale of the median face, observed below 5e-11 of it.
    assert rel_err(g.area, o.area, 1.0) <= 10 * TOL["area_3d"]
    # The reference orients each face by the cross product of its first three vertices
    # (cell.cpp:591-627); on wall cells that start is often (nearly) collinear, the sign is
    # rounding noise and a face's volume term enters with the wrong sign.  The device
    # orients faces by the clipping triangles' combinatorial orientation.  Volumes are
    # therefore checked against the pyramid volume sum_f area_f * |x_nb - x_c| / 6, which
    # needs no orientation: the device matches it on every certified cell, and the oracle
    # matches the device wherever the oracle itself matches it.
    ext, _, _ = om.ghosts(pts, buff, om.REFLECTIVE)
    fc = np.asarray(o.face_counts).astype(np.int64)
    owner = np.repeat(np.arange(len(fc)), fc)
    nb = np.asarray(o.neighbor).astype(np.int64)
    dist = np.linalg.norm(ext[nb] - ext[owner], axis=1) * (1.0 + 2.0 * buff)
    pyr = np.bincount(owner, np.asarray(o.area) * dist / 6.0, minlength=len(fc))
    ok = np.asarray(o.status) == 4
    ok[nh:] = False
    assert rel_err(g.volumes[ok], pyr[ok]) <= 1e-9
    ref_ok = ok & (np.abs(o.volumes - pyr) <= 1e-9 * pyr)
    assert (ok & ~ref_ok).sum() < 0.05 * ok.sum()
    assert rel_err(g.volumes[ref_ok], o.volumes[ref_ok]) <= TOL["volume_3d"]
    assert np.abs(g.centroid[ref_ok] - o.centroid[ref_ok]).max() <= TOL["centroid"]
    assert np.array_equal(g.normal, o.normal) and np.array_equal(g.seeds, o.seeds)
    assert np.array_equal(np.asarray(g.cert_k)[ok], np.asarray(o.cert_k)[ok])


def test_clustered_3d_mesh():
    ic = ics.clustered_3d(n=30000, seed=4)
    with Context(dim=3, k=190, buff=0.1) as ctx:
        g = ctx.compute_periodic_mesh(ic.pos)
    o = om.build_mesh(ic.pos, 190, buff=0.1)
    assert_same_topology(g, o)
    check_fields(g, o, 3)


def test_failed_cells_3d_k32():
    """K=32 in 3D leaves most cells uncertified; the failure set and codes must agree."""
    pts = ics.uniform_points(13000, 3, 22)
    ext = np.ascontiguousarray((pts - 0.5) / 1.2 + 0.5)
    with Context(dim=3, k=32) as ctx:
        g = ctx.compute_mesh(ext)
    o = om.cells(ext, len(ext), om.knn(ext, 32))
    assert (o.status != 4).sum() > 1000
    assert_same_topology(g, o)


@pytest.mark.parametrize("n", [0, 1, 2, 5, 40])
def test_tiny_inputs(n):
    pts = ics.uniform_points(n, 2, 30) if n else np.zeros((0, 2))
    with Context(dim=2, k=16) as ctx:
        g = ctx.compute_mesh(pts)
    assert g.n_seeds == n
    if n:
        o = om.cells(pts, n, om.knn(pts, 16))
        assert_same_topology(g, o)


def test_exact_lattice_ties():
    """An unjittered lattice has many equal distances and cocircular points: neighbour
    lists break ties by index and near-degenerate predicates are flagged the same way."""
    pts = ics.jittered_lattice(48, 2, 0.0, np.random.default_rng(0))
    with Context(dim=2, k=24) as ctx:
        g = ctx.compute_mesh(pts)
        kg = ctx.knn(pts)
    assert np.array_equal(kg, om.knn(pts, 24))
    o = om.cells(pts, len(pts), om.knn(pts, 24))
    assert_same_topology(g, o)
