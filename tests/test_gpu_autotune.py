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
    assert t["ppb"] in (1.5, 2.0, 3.0, 4.0) and t["knn_warps"] in (1, 2, 4, 8) and t["clip_warps"] in (1, 2, 4)
    assert t["knn_thread"] in (0, 32, 64)
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


def _mesh2d(pts, k, shapes, **kw):
    with Context(dim=2, k=k, gamma=1.4, **kw) as ctx:
        if shapes:
            ctx.set_tuning(**shapes)
        return ctx.compute_periodic_mesh(pts)


@pytest.mark.parametrize("case", ["sod", "uniform_k16", "kh"])
def test_thread_per_cell_2d_equals_warp_per_cell(case):
    """The 2D thread-per-cell clip gives the warp kernel's mesh bit for bit, including
    failing cells (uniform points at K = 16) and cells handed back for being too big."""
    if case == "sod":
        pts, k = ics.sod_2d().pos, 16
    elif case == "uniform_k16":
        pts, k = ics.uniform_points(20000, 2, 31), 16
    else:
        pts, k = ics.kh_2d(n_side=150, seed=3).pos, 32
    a = _mesh2d(pts, k, None)
    b = _mesh2d(pts, k, dict(clip_thread=True))
    for f in ("status", "cert_k", "face_counts", "neighbor", "normal", "area", "volumes", "centroid", "seeds"):
        assert np.array_equal(getattr(a, f), getattr(b, f)), f


def test_thread_per_cell_2d_moving_mesh_and_batch():
    B = ics.batch_2d(5, 21, 1000, 9000)
    outs = []
    for thread in (False, True):
        with Context(dim=2, k=32, flux="physical", predicates="robust") as ctx:
            ctx.set_tuning(clip_thread=thread, knn_thread=32 if thread else 0)
            ctx.batch_init(B.counts, B.buff, B.gamma, B.boundary, B.concat("pos"), B.concat("rho"),
                           B.concat("vel"), B.concat("energy"), B.concat("deposit"))
            for _ in range(3):
                ctx.sim_step(0.3)
            outs.append(ctx.sim_get())
    for u, v in zip(*outs):
        assert np.array_equal(u, v)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_clip_block_shapes_change_no_bit(precision):
    """One, two or four cells (warps) per clipping block give the same 3D mesh bit for bit,
    with the FP64 and with the FP32 clip."""
    pts = ics.clustered_3d(n=20000, seed=8).pos
    meshes = []
    for cw in (1, 2, 4):
        with Context(dim=3, k=96, buff=0.1, precision=precision) as ctx:
            ctx.set_tuning(clip_warps=cw)
            meshes.append(ctx.compute_periodic_mesh(pts))
    for m in meshes[1:]:
        for f in ("status", "cert_k", "face_counts", "neighbor", "normal", "area", "volumes", "centroid", "seeds"):
            assert np.array_equal(getattr(meshes[0], f), getattr(m, f)), f
