"""Batched form: independent 2D simulations of uneven sizes, mixed initial
conditions, gammas and boundaries, advanced together (one launch per stage).
Every instance's state and time step must equal a run of that instance alone."""
import numpy as np
import pytest

from proteusgpu_b200 import Context, ics

pytestmark = pytest.mark.gpu

K = 32


def _solo(ic, buff, steps, **kw):
    with Context(dim=2, k=K, buff=buff, boundary=ic.boundary, flux="physical", gamma=ic.gamma,
                 predicates="robust", **kw) as ctx:
        ctx.sim_init(ic.pos, ic.rho, ic.vel, ic.energy, ic.deposit)
        dts = [ctx.sim_step(0.3) for _ in range(steps)]
        return (dts,) + tuple(ctx.sim_get())


def _batch(B, steps, precision="fp64", kbudget=False):
    with Context(dim=2, k=K, flux="physical", predicates="robust", precision=precision) as ctx:
        if kbudget:
            ctx.kbudget_enable(train_steps=1, iters_per_step=64, quantile=0.98, seed=2)
        ctx.batch_init(B.counts, B.buff, B.gamma, B.boundary, B.concat("pos"), B.concat("rho"), B.concat("vel"),
                       B.concat("energy"), B.concat("deposit"))
        dts = []
        for _ in range(steps):
            ctx.sim_step(0.3)
            dts.append(ctx.batch_dt())
        st = ctx.stats()
        return (np.array(dts),) + tuple(ctx.sim_get()) + (st,)


def _check_equal_to_solo(B, out, steps):
    dts, x, m, p, e = out[:5]
    off = 0
    for b, ic in enumerate(B.instances):
        sd, sx, sm, sp, se = _solo(ic, B.buff[b], steps)
        sl = slice(off, off + ic.n)
        off += ic.n
        assert np.array_equal(dts[:, b], np.array(sd)), f"instance {b}: dt differs"
        assert np.array_equal(x[sl], sx) and np.array_equal(m[sl], sm), f"instance {b}: state differs"
        assert np.array_equal(p[sl], sp) and np.array_equal(e[sl], se), f"instance {b}: state differs"


def test_batch_equals_solo_runs():
    B = ics.batch_2d(6, 11, 1000, 12000)
    assert len(set(B.boundary)) == 2 and len(set(B.gamma.tolist())) == 2  # mixed on purpose
    out = _batch(B, 3)
    assert out[-1]["failed_cells"] == 0
    _check_equal_to_solo(B, out, 3)


def test_batch_of_64_instances_equals_solo_runs():
    """64 instances of every kind (Sod with walls, Sedov, Kelvin-Helmholtz), both gammas, both
    boundaries, 300 to 3000 points each: every one equals its solo run after 2 steps."""
    B = ics.batch_2d(64, 17, 300, 3000)
    assert len(B.instances) == 64 and len(set(B.boundary)) == 2
    out = _batch(B, 2)
    assert out[-1]["failed_cells"] == 0
    _check_equal_to_solo(B, out, 2)


def test_batch_learned_k_fp32_equals_plain_solo_runs():
    """The faster forms change no mesh: a learned-K + FP32 batch equals plain solo runs."""
    B = ics.batch_2d(4, 12, 2000, 15000)
    _check_equal_to_solo(B, _batch(B, 3, precision="fp32", kbudget=True), 3)


def test_batch_conserves_each_instance():
    B = ics.batch_2d(5, 13, 1500, 8000)
    with Context(dim=2, k=K, flux="physical", predicates="robust") as ctx:
        ctx.batch_init(B.counts, B.buff, B.gamma, B.boundary, B.concat("pos"), B.concat("rho"), B.concat("vel"),
                       B.concat("energy"), B.concat("deposit"))
        _, m0, _, e0 = ctx.sim_get()
        for _ in range(4):
            ctx.sim_step(0.3)
        _, m1, _, e1 = ctx.sim_get()
    off = 0
    for ic in B.instances:
        sl = slice(off, off + ic.n)
        off += ic.n
        assert abs(m1[sl].sum() - m0[sl].sum()) <= 1e-13 * m0[sl].sum()
        assert abs(e1[sl].sum() - e0[sl].sum()) <= 1e-12 * e0[sl].sum()
