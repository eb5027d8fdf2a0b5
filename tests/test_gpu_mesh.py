"""GPU mesh parity: the CUDA path through the C ABI against the oracle (same seeded inputs).

Topology (statuses, face counts, ordered neighbour ids) must be identical;
normals, 2D edge lengths and seeds bit-identical; 3D areas, volumes and
centroids within the tolerances in tests/helpers.py.
"""
import numpy as np
import pytest

import oracle as om
from helpers import TOL, assert_same_topology, faces_of, rel_err
from proteusgpu_b200 import Context, ics

pytestmark = pytest.mark.gpu


def check_fields(g, o, dim, floor_frac=1e-9, vol_tol=TOL["volume_3d"]):
    """floor_frac: values below floor_frac x median count as zero-size (degenerate faces)."""
    ok = np.asarray(o.status) == 4
    assert np.array_equal(g.normal, o.normal)
    if dim == 2:
        assert np.array_equal(g.area, o.area)
        assert rel_err(g.volumes, o.volumes) <= TOL["volume_2d"]
    else:
        assert rel_err(g.area, o.area, floor_frac) <= TOL["area_3d"]
        assert rel_err(g.volumes[ok], o.volumes[ok], floor_frac) <= vol_tol
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
    """Robust predicate mode on mirror walls: same topology as the oracle on the cells it certifies."""
    if dim == 2:
        pts, k, buff = ics.sod_2d().pos, 16, 0.04
    else:
        pts, k, buff = ics.uniform_points(15000, 3, 8), 190, 0.1
    with Context(dim=dim, k=k, buff=buff, boundary="reflective", predicates="robust") as ctx:
        ctx.sim_init(pts, np.ones(len(pts)), np.zeros_like(pts), np.ones(len(pts)))
        g = ctx.download_mesh()
    o = om.build_mesh(pts, k, buff=buff, boundary=om.REFLECTIVE, hydro_only=True, robust=True)
    nh = o.n_hydro
    if dim == 2:  # in 2D every mirror degeneracy resolves
        assert (o.status[:nh] == 4).all()
        assert abs(g.volumes[:nh].sum() - 1.0) < 1e-11
        assert_same_topology(g, o)
        check_fields(g, o, dim)
        return
    # In 3D a few wall cells fail within K (the oracle reports them); the moving-mesh
    # build walks the grid for those (cert_k = K + 1) and certifies most.
    gs, os_ = np.asarray(g.status), np.asarray(o.status)
    walked = (os_ != 4) & (gs == 4)
    assert walked.sum() > 0 and (np.asarray(g.cert_k)[walked] == k + 1).all()
    assert np.array_equal((gs == 4)[~walked], (os_ == 4)[~walked])
    okc = np.where(os_ == 4)[0]
    assert np.array_equal(np.asarray(g.face_counts)[okc], np.asarray(o.face_counts)[okc])
    gf, of = faces_of(g, okc), faces_of(o, okc)
    assert np.array_equal(np.asarray(g.neighbor)[gf], np.asarray(o.neighbor)[of])
    assert np.array_equal(np.asarray(g.normal)[gf], np.asarray(o.normal)[of])
    # 3D mirror walls leave exactly-degenerate faces whose computed areas are pure rounding
    # (a sum of nearly cancelling fan triangles), and nearly degenerate vertices (mirror
    # images are cospherical) whose rounding is amplified: areas are compared as an
    # absolute error on the scale of the median face, observed below 5e-11 of it.
    assert rel_err(np.asarray(g.area)[gf], np.asarray(o.area)[of], 1.0) <= 10 * TOL["area_3d"]
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
    assert np.array_equal(g.seeds[ok], o.seeds[ok])
    assert np.array_equal(np.asarray(g.cert_k)[ok], np.asarray(o.cert_k)[ok])
    # walked cells: closed polyhedra whose volume equals their own pyramid volume
    gfc = np.asarray(g.face_counts).astype(np.int64)
    gown = np.repeat(np.arange(len(gfc)), gfc)
    gnb = np.asarray(g.neighbor).astype(np.int64)
    gd = np.linalg.norm(ext[gnb] - ext[gown], axis=1) * (1.0 + 2.0 * buff)
    gpyr = np.bincount(gown, np.asarray(g.area) * gd / 6.0, minlength=len(gfc))
    assert rel_err(g.volumes[walked], gpyr[walked]) <= 1e-9


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


def test_dense_blob_3d_mesh():
    """Refined grid bins under the clipping: same topology and fields as the oracle."""
    rng = np.random.default_rng(31)
    blob = 0.5 + 0.003 * rng.standard_normal((20000, 3))
    pts = np.ascontiguousarray(np.concatenate([blob, rng.random((10000, 3))]))
    with Context(dim=3, k=190, buff=0.1) as ctx:
        g = ctx.compute_periodic_mesh(pts)
    o = om.build_mesh(pts, 190, buff=0.1)
    assert_same_topology(g, o)
    # blob cells are ~1e-3 of the coordinates' magnitude across, so their volumes
    # (sums of nearly cancelling tetrahedra) carry ~1e3 x the usual relative rounding
    check_fields(g, o, 3, vol_tol=10 * TOL["volume_3d"])


def _blob_with_background(seed=41):
    rng = np.random.default_rng(seed)
    blob = 0.5 + 0.004 * rng.standard_normal((12000, 3))
    return np.ascontiguousarray(np.concatenate([blob, rng.random((3000, 3))]))


def _cell_faces(m, c):
    a, b = int(m.face_ptr[c]), int(m.face_ptr[c] + m.face_counts[c])
    nb = np.asarray(m.neighbor[a:b]).astype(np.int64)
    order = np.argsort(nb, kind="stable")
    return nb[order], np.asarray(m.area[a:b])[order]


def test_grid_walk_certifies_cells_beside_a_dense_clump():
    """Background cells next to a clump 10^4 times denser need thousands of
    neighbours for the security radius (the oracle still leaves cells uncertified
    at K = 3000).  The moving-mesh build certifies them by walking the grid; the
    mesh must tile the box, pair every face, and agree with the oracle wherever
    the oracle's fallback budget certifies the cell."""
    pts = _blob_with_background()
    rho, v, E = np.ones(len(pts)), np.zeros_like(pts), np.ones(len(pts))
    runs = []
    for _ in range(2):
        with Context(dim=3, k=190, buff=0.15, flux="physical") as ctx:
            ctx.sim_init(pts, rho, v, E)
            runs.append((ctx.download_mesh(), ctx.stats()))
    (g, st), (g2, _) = runs
    nh = g.n_hydro
    assert st["pruned_cells"] > 100 and st["uncertified_cells"] == 0 and st["failed_cells"] == 0
    assert st["unpaired_faces"] == 0
    assert (np.asarray(g.status)[:nh] == 4).all()
    assert abs(g.volumes[:nh].sum() - 1.0) <= 1e-12
    # deterministic: the walk visits sub-bins in a fixed order
    assert np.array_equal(g.volumes, g2.volumes) and np.array_equal(g.neighbor, g2.neighbor)
    o = om.build_mesh(pts, 190, buff=0.15, hydro_only=True, k_fallback=1000)
    ost = np.asarray(o.status)[:nh]
    both = np.where(ost == 4)[0]
    walked = np.where(np.asarray(g.cert_k)[:nh] == 191)[0]
    assert len(np.intersect1d(walked, both)) > 100
    assert rel_err(g.volumes[both], o.volumes[both]) <= 1e-10
    for c in np.intersect1d(walked, both):
        gn, ga = _cell_faces(g, c)
        on, oa = _cell_faces(o, c)
        assert np.array_equal(gn, on)
        assert np.abs(ga - oa).max() <= 1e-10 * np.abs(oa).max()
