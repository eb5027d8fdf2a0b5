"""voronoi::vmesh_to_meshdata -- the VMesh -> MeshCellData conversion the HDF5
writer consumes (reference src/voronoi/voronoi.cpp:339-421, io/output.h:14-48) --
of the drop-in unit (proteusgpu_b200/dropin/voronoi_gpu.cpp) against the
reference's own function, field by field.

The CPU test hands the same VMesh (the reference build's mesh, rewrapped in each
library) to both functions: every field must be identical.  The GPU test lets
the drop-in build its mesh on the device and compares its MeshCellData with the
reference pipeline's, within the mesh tolerances.
"""
import numpy as np
import pytest

import refbuild as rb
from helpers import TOL, rel_err
from proteusgpu_b200 import ics

pytestmark = pytest.mark.skipif(not (rb.available(2, 16, "ref") and rb.available(2, 16, "dropin")
                                     and rb.available(3, 190, "ref") and rb.available(3, 190, "dropin")),
                                reason="reference or drop-in libraries not built")

FIELDS = ("cell_ids", "seeds", "volumes", "face_counts", "neighbor_cell", "normal", "area")


def _ref_mesh(dim, k, pts, buff):
    prev = rb.use("ref")
    try:
        return rb.periodic_mesh(pts, k, buff=buff, keep_handle=True)
    finally:
        rb.use(prev)


def _meshdata(flavor, dim, k, m):
    """MeshCellData of mesh m (any RefMesh-like object) converted by `flavor`'s function."""
    prev = rb.use(flavor)
    try:
        h = rb.wrap_mesh(dim, k, m)
        rb.set_seeds(dim, k, h, m.seeds)
        d = rb.meshdata(dim, k, h)
        rb.free_handle(dim, k, h)
        return d
    finally:
        rb.use(prev)


@pytest.mark.parametrize("dim,k,n,buff", [(2, 16, None, 0.04), (3, 190, 20000, 0.1)])
def test_dropin_meshdata_equals_reference_on_one_mesh(dim, k, n, buff):
    pts = ics.sod_2d().pos if dim == 2 else ics.uniform_points(n, 3, 21)
    m = _ref_mesh(dim, k, pts, buff)
    a, b = _meshdata("ref", dim, k, m), _meshdata("dropin", dim, k, m)
    prev = rb.use("ref")
    rb.free_handle(dim, k, m.handle)
    rb.use(prev)
    assert a["header"] == b["header"] and a["header"]["n"] == m.n_hydro
    assert a["seeds_dims"] == b["seeds_dims"] == [m.n_hydro, dim]
    assert a["normal_dims"] == b["normal_dims"] == [m.num_faces, dim]
    for f in FIELDS:
        assert a[f].dtype == b[f].dtype and np.array_equal(a[f], b[f]), f


@pytest.mark.gpu
def test_dropin_meshdata_of_device_mesh_2d():
    """2D Sod: the drop-in's mesh (built on the device) converted by the drop-in equals the
    reference pipeline's MeshCellData bit for bit (2D meshes are bit-identical)."""
    ic = ics.sod_2d()
    ref = _ref_mesh(2, 16, ic.pos, 0.04)
    a = _meshdata("ref", 2, 16, ref)
    prev = rb.use("dropin")
    try:
        g = rb.periodic_mesh(ic.pos, 16, buff=0.04, keep_handle=True)
        b = rb.meshdata(2, 16, g.handle)
        rb.free_handle(2, 16, g.handle)
    finally:
        rb.use(prev)
    assert a["header"] == b["header"] and a["seeds_dims"] == b["seeds_dims"] and a["normal_dims"] == b["normal_dims"]
    for f in ("cell_ids", "seeds", "face_counts", "neighbor_cell", "normal", "area"):
        assert np.array_equal(a[f], b[f]), f
    assert rel_err(b["volumes"], a["volumes"]) <= TOL["volume_2d"]


@pytest.mark.gpu
def test_dropin_meshdata_of_device_mesh_3d():
    """3D uniform points, K = 190: topology fields identical, areas and volumes within
    the 3D tolerances."""
    pts = ics.uniform_points(20000, 3, 22)
    ref = _ref_mesh(3, 190, pts, 0.1)
    a = _meshdata("ref", 3, 190, ref)
    prev = rb.use("dropin")
    try:
        g = rb.periodic_mesh(pts, 190, buff=0.1, keep_handle=True)
        b = rb.meshdata(3, 190, g.handle)
        rb.free_handle(3, 190, g.handle)
    finally:
        rb.use(prev)
    assert a["header"] == b["header"] and a["seeds_dims"] == b["seeds_dims"] and a["normal_dims"] == b["normal_dims"]
    for f in ("cell_ids", "seeds", "face_counts", "neighbor_cell", "normal"):
        assert np.array_equal(a[f], b[f]), f
    assert rel_err(b["area"], a["area"]) <= TOL["area_3d"]
    assert rel_err(b["volumes"], a["volumes"]) <= TOL["volume_3d"]
