"""The C++ drop-in units (proteusgpu_b200/dropin) through the reference's own call sequences.

The drop-in libraries link the drop-in knn/voronoi/hydro translation units,
compiled against the reference's headers, with the same test driver the
reference build uses (oracle/ref_driver.cpp), so knn::init, voronoi::compute_mesh's
sequence (knn::init, compute_cells, unpermute_vmesh), compute_periodic_mesh,
hydro::dt_CFL and hydro::hydro_step are the entry points exercised.
"""
import numpy as np
import pytest

import oracle as om
import refbuild as rb
from helpers import TOL, rel_err
from proteusgpu_b200 import ics

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not rb.available(2, 16, "dropin"), reason="drop-in libraries not built")]


@pytest.fixture(autouse=True)
def dropin_flavor():
    prev = rb.use("dropin")
    yield
    rb.use(prev)


def test_dropin_periodic_mesh_2d():
    ic = ics.sod_2d()
    g = rb.periodic_mesh(ic.pos, 16, buff=0.04, gamma=1.4)
    o = om.build_mesh(ic.pos, 16)
    assert g.n_seeds == o.n_seeds and g.n_hydro == o.n_hydro and g.num_faces == o.num_faces
    assert np.array_equal(g.face_counts, o.face_counts) and np.array_equal(g.face_ptr, o.face_ptr)
    assert np.array_equal(g.neighbor, o.neighbor) and np.array_equal(g.ghost_ids, o.ghost_ids)
    assert np.array_equal(g.normal, o.normal) and np.array_equal(g.area, o.area)
    assert np.array_equal(g.seeds, o.seeds)
    assert rel_err(g.volumes, o.volumes) <= TOL["volume_2d"]


def test_dropin_compute_mesh_sequence_statuses():
    """knn::init -> compute_cells -> unpermute_vmesh, with uncertified cells."""
    pts = ics.uniform_points(1500, 2, 16)
    g = rb.compute_mesh(pts, 16)
    o = om.cells(pts, len(pts), om.knn(pts, 16))
    assert np.array_equal(g.status, o.status) and (o.status != 4).any()
    assert np.array_equal(g.face_counts, o.face_counts) and np.array_equal(g.neighbor, o.neighbor)
    assert np.array_equal(g.area, o.area)


def test_dropin_knn_lists():
    pts = ics.uniform_points(5000, 2, 17)
    assert np.array_equal(rb.knn(pts, 16), om.knn(pts, 16))


def test_dropin_hydro_bitexact_on_same_mesh(golden2):
    d = golden2
    m = rb.periodic_mesh(d["pts2"], 16, buff=0.08, gamma=1.4, keep_handle=True)
    dt = rb.dt_cfl(2, 16, m.handle, 0.3, d["rho0"], d["vel0"], d["E0"], 1.4)
    assert dt == d["dt2"]
    r, v, e = d["rho0"], d["vel0"], d["E0"]
    for _ in range(3):
        r, v, e = rb.hydro_step(2, 16, m.handle, dt, r, v, e, 1.4)
    rb.free_handle(2, 16, m.handle)
    assert np.array_equal(r, d["rho3"]) and np.array_equal(v, d["vel3"]) and np.array_equal(e, d["E3"])


def test_dropin_3d_mesh_and_hydro():
    ic = ics.sedov_3d(n=20000, seed=5)
    g = rb.periodic_mesh(ic.pos, 190, buff=0.1, gamma=ic.gamma, keep_handle=True)
    o = om.build_mesh(ic.pos, 190, buff=0.1)
    assert np.array_equal(g.face_counts, o.face_counts) and np.array_equal(g.neighbor, o.neighbor)
    assert rel_err(g.area, o.area) <= TOL["area_3d"] and rel_err(g.volumes, o.volumes) <= TOL["volume_3d"]
    E = ic.energy + ic.deposit / g.volumes[: g.n_hydro]
    dt = rb.dt_cfl(3, 190, g.handle, 0.3, ic.rho, ic.vel, E, ic.gamma)
    r, v, e = rb.hydro_step(3, 190, g.handle, dt, ic.rho, ic.vel, E, ic.gamma)
    rb.free_handle(3, 190, g.handle)
    R, V, EE, _ = om.hydro_step_ref(o, dt, ic.gamma, ic.rho, ic.vel, E)
    assert rel_err(r, R) <= 1e-10 and rel_err(e, EE) <= 1e-10
