"""Autotuner: picks launch shapes from timed mesh builds; results never depend on them."""
import numpy as np
import pytest

from proteusgpu_b200 import Context, ics

pytestmark = pytest.mark.gpu


def _run(ic, tune, precision="fp64"):
    with Context(dim=3, k=190, buff=0.1, flux="physical", gamma=ic.gamma, precision=precision) as ctx:
        ctx.sim_init(ic.pos, ic.rho, ic.vel, ic.energy, ic.deposit)
        t = ctx.autotune() if tune else None
        for _ in range(3):
            ctx.sim_step(0.3)
        return t, ctx.sim_get(), ctx.download_mesh()


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_autotuned_shapes_give_identical_steps(precision):
    ic = ics.sedov_3d(n=25000, seed=12)
    _, ref, mref = _run(ic, False, precision)
    t, got, mgot = _run(ic, True, precision)
    assert t["ppb"] in (1.5, 2.0, 3.0, 4.0) and t["knn_warps"] in (2, 4, 8) and t["clip_warps"] in (2, 4)
    assert t["ms_tuned"] > 0 and t["ms_default"] > 0
    for a, b in zip(ref, got):
        assert np.array_equal(a, b)
    assert np.array_equal(mref.neighbor, mgot.neighbor) and np.array_equal(mref.area, mgot.area)


def test_autotune_is_cached_per_workload_class():
    ic = ics.sedov_3d(n=20000, seed=13)
    first, _, _ = _run(ic, True)
    again, _, _ = _run(ic, True)
    assert again["from_cache"] == 1
    assert (again["ppb"], again["knn_warps"], again["clip_warps"]) == (first["ppb"], first["knn_warps"],
                                                                        first["clip_warps"])
