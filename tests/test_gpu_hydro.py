"""GPU hydro parity: hydro::dt_CFL and hydro::hydro_step semantics.

On the same (uploaded) mesh the CUDA flux/update is bit-identical to the oracle
(and to the reference's own numbers in the golden fixture); on the GPU's own
mesh it agrees within the stated tolerance.
"""
import numpy as np
import pytest

import oracle as om
from helpers import TOL, rel_err
from proteusgpu_b200 import Context, ics
from proteusgpu_b200._lib import PGPUError

pytestmark = pytest.mark.gpu


def test_golden_hydro_bitexact_on_reference_mesh(golden2):
    d = golden2
    m = om.build_mesh(d["pts2"], 16, buff=0.08)  # equals the reference's mesh (oracle pin)
    with Context(dim=2, k=16, buff=0.08, gamma=1.4) as ctx:
        ctx.upload_mesh(m)
        ctx.set_prim(d["rho0"], d["vel0"], d["E0"])
        dt = ctx.dt_cfl(0.3)
        assert dt == d["dt2"]
        for _ in range(3):
            ctx.hydro_step(dt)
        r, v, e = ctx.get_prim()
    assert np.array_equal(r, d["rho3"]) and np.array_equal(v, d["vel3"]) and np.array_equal(e, d["E3"])


@pytest.mark.parametrize("flux", ["reference", "physical"])
def test_sod_hydro_on_gpu_mesh(flux):
    ic = ics.sod_2d()
    o = om.build_mesh(ic.pos, 16)
    with Context(dim=2, k=16, gamma=1.4, flux=flux) as ctx:
        ctx.compute_periodic_mesh(ic.pos, download=False)
        ctx.set_prim(ic.rho, ic.vel, ic.energy)
        dtg = ctx.dt_cfl(0.3)
        dto = om.dt_cfl(o, 0.3, 1.4, ic.rho, ic.vel, ic.energy)
        assert rel_err(dtg, dto) <= 1e-13
        for _ in range(5):
            ctx.hydro_step(dto)
        r, v, e = ctx.get_prim()
    R, V, E = ic.rho, ic.vel, ic.energy
    if flux == "reference":
        for _ in range(5):
            R, V, E, _ = om.hydro_step_ref(o, dto, 1.4, R, V, E)
        assert rel_err(r, R) <= TOL["hydro"] and rel_err(e, E) <= TOL["hydro"]
        assert np.abs(v - V).max() <= 1e-10


def test_sedov_3d_hydro_bitexact_on_same_mesh():
    ic = ics.sedov_3d(n=20000, seed=3)
    m = om.build_mesh(ic.pos, 190, buff=0.1)
    E = ic.energy + ic.deposit / m.volumes[: m.n_hydro]
    with Context(dim=3, k=190, buff=0.1) as ctx:
        ctx.upload_mesh(m)
        ctx.set_prim(ic.rho, ic.vel, E)
        dt = ctx.dt_cfl(0.3)
        for _ in range(3):
            ctx.hydro_step(dt)
        r, v, e = ctx.get_prim()
    assert rel_err(dt, om.dt_cfl(m, 0.3, ic.gamma, ic.rho, ic.vel, E)) <= 1e-15
    R, V, EE = ic.rho, ic.vel, E
    for _ in range(3):
        R, V, EE, _ = om.hydro_step_ref(m, dt, ic.gamma, R, V, EE)
    assert np.array_equal(r, R) and np.array_equal(v, V) and np.array_equal(e, EE)


def test_thin_ghost_layer_is_reported():
    """Below ~1M points in 3D the reference's fixed buff leaves hydro cells touching the
    bounding box and its hydro step reads out of bounds; here the step returns an error."""
    pts = ics.uniform_points(3000, 3, 31)
    with Context(dim=3, k=190, buff=0.02) as ctx:
        ctx.compute_periodic_mesh(pts, download=False)
        ctx.set_prim(np.ones(3000), np.zeros((3000, 3)), np.ones(3000))
        with pytest.raises(PGPUError, match="bounding-box"):
            ctx.hydro_step(1e-4)
