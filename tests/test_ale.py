"""Moving-face steps (the faces move with the generators; first and second order)
on the oracle (oracle/restate/om_hydro.c om_step_ale) and, marked gpu, the CUDA
path (PGPU_FLUX_ALE1 / ALE2) against it.

The reference's solver is first order on a static mesh (src/hydro/
finite_volume_solver.cpp:43-148); a moving mesh needs the face velocity in the
Riemann problem.  The convergence test shows it: a plane sound wave in a periodic
box, density L1 error against the travelling linear solution at 16^2, 32^2 and
64^2 cells -- the static-face flux on the moving mesh does not converge, the
moving-face first-order step converges at first order, the second-order step at
about second order.
"""
import math

import numpy as np
import pytest

import oracle as om
from helpers import rel_err
from proteusgpu_b200 import Context, ics

K, BUFF = 16, 0.1
AMP = 1e-6  # small enough that the wave's own steepening stays far below the schemes' errors


def _oracle_run(ic, mode, t_end=None, steps=None, cfl=0.3, k=K, buff=BUFF):
    """mode: 'static' (om_step_moving), 1 or 2 (om_step_ale)."""
    m0 = om.build_mesh(ic.pos, k, buff=buff, hydro_only=True, expand_k=1 << 12)
    M, P, E = om.prim_to_cons(m0, ic.rho, ic.vel, ic.energy, ic.deposit)
    x, t, n, dts = ic.pos.copy(), 0.0, 0, []
    while (steps is not None and n < steps) or (t_end is not None and t < t_end - 1e-12):
        m = om.build_mesh(x, k, buff=buff, hydro_only=True, expand_k=1 << 12)
        fixed = 0.0
        if t_end is not None:
            dtc = om.dt_cfl(m, cfl, ic.gamma, M / m.volumes[: ic.n], P / M[:, None], E / m.volumes[: ic.n])
            fixed = min(dtc, t_end - t)
        if mode == "static":
            dt, x, M, P, E, _ = om.step_moving(m, cfl, ic.gamma, om.PERIODIC, x, M, P, E, fixed_dt=fixed)
        else:
            dt, x, M, P, E, unp = om.step_ale(m, mode, cfl, ic.gamma, x, M, P, E, fixed_dt=fixed)
            assert unp == 0
        t, n = t + dt, n + 1
        dts.append(dt)
    return dts, x, M, P, E, t


def _wave_error(ic, x, M, t):
    m = om.build_mesh(x, K, buff=BUFF, hydro_only=True, expand_k=1 << 12)
    V = m.volumes[: ic.n]
    exact = 1.0 + AMP * np.sin(2.0 * math.pi * (m.centroid[: ic.n, 0] - math.sqrt(ic.gamma) * t))
    return float(np.sum(np.abs(M / V - exact) * V) / AMP)


def test_moving_faces_converge_at_first_and_second_order():
    err = {mode: [] for mode in ("static", 1, 2)}
    for ns in (16, 32, 64):
        ic = ics.sound_wave_2d(ns, amp=AMP)
        for mode in err:
            _, x, M, _, _, t = _oracle_run(ic, mode, t_end=0.5)
            err[mode].append(_wave_error(ic, x, M, t))
    r = {mode: [e[i] / e[i + 1] for i in range(2)] for mode, e in err.items()}
    assert err["static"][2] > 0.3 and r["static"][1] < 1.2, err      # O(1), not converging
    assert min(r[1]) > 1.5 and err[1][2] < 0.2, err                  # first order
    assert min(r[2]) > 2.8 and err[2][2] < 0.01, err                 # about second order
    assert err[2][2] < err[1][2] / 10


def test_second_order_step_conserves_exactly():
    ic = ics.kh_2d(n_side=48, seed=3)
    m0 = om.build_mesh(ic.pos, K, buff=BUFF, hydro_only=True, expand_k=1 << 12)
    M, P, E = om.prim_to_cons(m0, ic.rho, ic.vel, ic.energy)
    x = ic.pos.copy()
    s0 = (M.sum(), P.sum(axis=0), E.sum())
    for _ in range(4):
        m = om.build_mesh(x, K, buff=BUFF, hydro_only=True, expand_k=1 << 12)
        _, x, M, P, E, unp = om.step_ale(m, 2, 0.3, ic.gamma, x, M, P, E)
        assert unp == 0
    assert abs(M.sum() - s0[0]) <= 1e-14 * s0[0] and abs(E.sum() - s0[2]) <= 1e-14 * s0[2]
    assert np.abs(P.sum(axis=0) - s0[1]).max() <= 1e-14


def _gpu_run(ic, flux, steps, k=K, buff=BUFF):
    with Context(dim=ic.dim, k=k, buff=buff, boundary="periodic", flux=flux, gamma=ic.gamma) as ctx:
        ctx.sim_init(ic.pos, ic.rho, ic.vel, ic.energy, ic.deposit)
        s0 = ctx.stats()
        dts = [ctx.sim_step(0.3) for _ in range(steps)]
        s1 = ctx.stats()
        x, M, P, E = ctx.sim_get()
    assert s1["failed_cells"] == 0 and s1["box_faces"] == 0 and s1["unpaired_faces"] == 0
    return dts, x, M, P, E, s0, s1


@pytest.mark.gpu
@pytest.mark.parametrize("order", [1, 2])
def test_gpu_moving_faces_2d_equal_oracle(order):
    ic = ics.kh_2d(n_side=64, seed=3)
    dg, xg, Mg, Pg, Eg, s0, s1 = _gpu_run(ic, f"ale{order}", 5)
    do, xo, Mo, Po, Eo, _ = _oracle_run(ic, order, steps=5)
    assert rel_err(dg, do) <= 1e-12
    assert np.abs(xg - xo).max() <= 1e-13
    assert rel_err(Mg, Mo) <= 1e-10 and rel_err(Eg, Eo) <= 1e-10 and np.abs(Pg - Po).max() <= 1e-12
    assert abs(s1["total_mass"] - s0["total_mass"]) <= 1e-14 * s0["total_mass"]
    assert abs(s1["total_energy"] - s0["total_energy"]) <= 1e-14 * s0["total_energy"]


@pytest.mark.gpu
def test_gpu_second_order_3d_equals_oracle_and_conserves():
    ic = ics.sedov_3d(n=20000, seed=6)
    dg, xg, Mg, Pg, Eg, s0, s1 = _gpu_run(ic, "ale2", 3, k=190, buff=0.1)
    do, xo, Mo, Po, Eo, _ = _oracle_run(ic, 2, steps=3, k=190, buff=0.1)
    assert rel_err(dg, do) <= 1e-12
    assert np.abs(xg - xo).max() <= 1e-13
    assert rel_err(Mg, Mo) <= 1e-10 and rel_err(Eg, Eo) <= 1e-10 and np.abs(Pg - Po).max() <= 1e-12
    assert abs(s1["total_mass"] - s0["total_mass"]) <= 1e-13 * s0["total_mass"]
    assert abs(s1["total_energy"] - s0["total_energy"]) <= 1e-13 * s0["total_energy"]
    assert np.abs(np.array(s1["total_mom"])).max() <= 1e-14


@pytest.mark.gpu
def test_gpu_moving_faces_converge():
    """The same convergence on the device: density L1 error of the sound wave."""
    err = {}
    for ns in (32, 64, 128):
        ic = ics.sound_wave_2d(ns, amp=AMP)
        for flux in ("physical", "ale2"):
            with Context(dim=2, k=K, buff=BUFF, boundary="periodic", flux=flux, gamma=ic.gamma) as ctx:
                ctx.sim_init(ic.pos, ic.rho, ic.vel, ic.energy)
                t = 0.0
                while t < 0.5 - 1e-12:
                    t += ctx.sim_step(0.3)
                x, M, _, _ = ctx.sim_get()
            err.setdefault(flux, []).append(_wave_error(ic, x, M, t))
    assert err["ale2"][2] < err["ale2"][1] / 2.8 < err["ale2"][0] / 2.8 ** 2, err
    assert err["physical"][2] > 0.3, err
