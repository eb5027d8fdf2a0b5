"""Parity at the benchmark configurations' full sizes (sampled cells and a full oracle run).

The meshes of the 3D Sedov workload (1,048,576 uniform points, K = 190) and of
the clustered 3D Sedov workload (16,777,216 points, 70 % in 64 Gaussian clumps)
are read back in part and a stratified sample of their hydro cells is
recomputed by the oracle on the GPU's own extended point set
(oracle/check.py: exact KNN rows, src/knn/knn.cpp:225-315; the reference's
clipping with a budget large enough to certify each cell,
src/voronoi/voronoi.cpp:115-155), including cells the GPU certified by its grid
walk; the extended point set itself is rebuilt by the oracle from the step's
positions (src/voronoi/periodic_mesh.cpp:44-126).  Topology is exact; geometry
within oracle/check.py's TOL.  The density error of a whole run is measured
against the oracle's own moving-mesh run of the clustered distribution at
1,048,576 points.
"""
import numpy as np
import pytest

import check
from proteusgpu_b200 import Context, ics

pytestmark = pytest.mark.gpu

DENSITY_L1_TOL = 1e-6  # relative L1 of the density against the FP64 oracle (headline target)


def _assert_clean(rep):
    assert rep.get("ghosts_identical", True), rep
    assert rep["status_mismatch"] == 0 and rep["topology_mismatch"] == 0, rep
    assert rep["neighbour_list_mismatch"] == 0, rep
    assert rep["oracle_unresolved"] == 0, rep
    assert rep["within_tolerance"], rep


def test_sedov_1m_uniform_sampled_cells():
    """3D Sedov, 1,048,576 uniform points, K = 190, plain FP64 form: the first mesh and the
    mesh of the third moving-mesh step, 20,000 cells each."""
    ic = ics.sedov_3d(n=1_048_576, seed=2)
    with Context(dim=3, k=190, buff=0.04, boundary="periodic", flux="physical", gamma=ic.gamma) as ctx:
        ctx.sim_init(ic.pos, ic.rho, ic.vel, ic.energy, ic.deposit)
        rep0 = check.sampled_cells(ctx, n_random=20000, pos_before=ic.pos, seed=1)
        ctx.sim_step(0.3)
        ctx.sim_step(0.3)
        x = ctx.sim_get()[0]
        ctx.sim_step(0.3)
        rep1 = check.sampled_cells(ctx, n_random=20000, pos_before=x, seed=2)
    _assert_clean(rep0)
    _assert_clean(rep1)
    assert rep0["cells_sampled"] >= 20000 and rep1["cells_sampled"] >= 20000


def test_clustered_16m_headline_form_sampled_cells():
    """Clustered 3D Sedov, 16,777,216 points, learned K + FP32 clipping: the first mesh
    (FP32 clipping at K = 190) and a mesh built from learned budgets after two training
    steps, 20,000 random cells plus 2,000 cells certified by the grid walk."""
    ic = ics.clustered_3d(n=16_777_216, seed=4)
    with Context(dim=3, k=190, buff=0.04, boundary="periodic", flux="physical", gamma=ic.gamma,
                 precision="fp32") as ctx:
        ctx.kbudget_enable(train_steps=2, iters_per_step=128, quantile=0.98, seed=1)
        ctx.sim_init(ic.pos, ic.rho, ic.vel, ic.energy, ic.deposit)
        rep0 = check.sampled_cells(ctx, n_random=20000, n_walked=2000, pos_before=ic.pos, seed=3)
        ctx.sim_step(0.3)
        ctx.sim_step(0.3)
        x = ctx.sim_get()[0]
        ctx.sim_step(0.3)
        kb = ctx.kbudget_stats()
        rep1 = check.sampled_cells(ctx, n_random=20000, n_walked=2000, pos_before=x, seed=4)
    assert kb["active"] and kb["mean_k"] < 190
    _assert_clean(rep0)
    _assert_clean(rep1)
    assert rep1["walked_sampled"] >= min(2000, rep1["walked_total"]) > 0


def _gpu_run(ic, buff, steps, precision, weights=None):
    with Context(dim=3, k=190, buff=buff, boundary="periodic", flux="physical", gamma=ic.gamma,
                 precision=precision) as ctx:
        if weights is not None:
            ctx.kbudget_enable(train_steps=0, iters_per_step=1, quantile=0.98, seed=1)
            ctx.kbudget_weights(set_to=weights)
        ctx.sim_init(ic.pos, ic.rho, ic.vel, ic.energy, ic.deposit)
        dts = [ctx.sim_step(0.3) for _ in range(steps)]
        vol = ctx.download_volumes()[: ic.n]
        x, m, p, e = ctx.sim_get()
        kb = ctx.kbudget_stats() if weights is not None else None
    return (dts, x, m, p, e, vol), kb


def _trained_weights(ic, buff):
    with Context(dim=3, k=190, buff=buff, boundary="periodic", flux="physical", gamma=ic.gamma,
                 precision="fp32") as ctx:
        ctx.kbudget_enable(train_steps=2, iters_per_step=128, quantile=0.98, seed=1)
        ctx.sim_init(ic.pos, ic.rho, ic.vel, ic.energy, ic.deposit)
        for _ in range(2):
            ctx.sim_step(0.3)
        return ctx.kbudget_weights()


def test_clustered_1m_density_error_against_oracle_run():
    """Clustered distribution at 1,048,576 points: three moving-mesh steps of the learned-K
    + FP32 form (proposals from a model trained on this distribution) and of the plain FP64
    form against the oracle's run; the density's relative L1 error is the headline target's."""
    buff = 0.04 * 16 ** (1 / 3)
    ic = ics.clustered_3d(n=1_048_576, seed=4)
    w = _trained_weights(ic, buff)
    head, kb = _gpu_run(ic, buff, 3, "fp32", weights=w)
    plain, _ = _gpu_run(ic, buff, 3, "fp64")
    ora = check.oracle_moving_run(ic, 190, buff, "periodic", 3)
    e_head = check.state_errors(head, ora)
    e_plain = check.state_errors(plain, ora)
    assert kb["active"] and kb["mean_k"] < 190
    for e in (e_head, e_plain):
        assert e["density_l1_rel"] <= DENSITY_L1_TOL, e
        assert e["dt_rel_max"] <= 1e-12, e
        assert e["mass_l1_rel"] <= 1e-10 and e["energy_l1_rel"] <= 1e-10, e
    # the two forms build the same meshes: their states are identical
    assert all(np.array_equal(np.asarray(a), np.asarray(b)) for a, b in zip(head[1:5], plain[1:5]))
