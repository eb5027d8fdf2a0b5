"""Initial conditions generated on the device (pgpu_ic_generate, csrc/ics.cu) against the
host generators of proteusgpu_b200/ics.py: every field bit for bit, for each workload's
kind, up to the 16,777,216-point clustered workload; and simulations started from a
device-generated condition (pgpu_sim_init_ic, pgpu_batch_init_ic) equal the ones started
from the host arrays."""
import numpy as np
import pytest

from proteusgpu_b200 import Context, ics

pytestmark = pytest.mark.gpu


def _same(ic, got):
    pos, rho, vel, en, dep = got
    assert np.array_equal(pos, ic.pos), np.abs(pos - ic.pos).max()
    assert np.array_equal(rho, ic.rho) and np.array_equal(vel, ic.vel) and np.array_equal(en, ic.energy)
    want_dep = ic.deposit if ic.deposit is not None else np.zeros(ic.n)
    assert np.array_equal(dep, want_dep)


@pytest.mark.parametrize("make", [
    lambda: ics.sod_2d(),
    lambda: ics.sod_2d(n_side=37, seed=9, gamma=5.0 / 3.0, split_angle=1.1),
    lambda: ics.sedov_2d(50000, seed=12, e_blast=3.0),
    lambda: ics.sedov_3d(n=262144, seed=2),
    lambda: ics.kh_2d(n_side=256, seed=3, rho_ratio=4.5),
    lambda: ics.clustered_3d(n=1_048_576, seed=4),
], ids=["sod", "sod_split", "sedov2d", "sedov3d", "kh", "clustered_1m"])
def test_device_ic_equals_host_ic(make):
    ic = make()
    with Context(dim=ic.dim, k=16 if ic.dim == 2 else 190) as ctx:
        _same(ic, ctx.ic_generate(ic.spec))


def test_device_ic_clustered_16m_workload():
    """The headline workload's initial condition itself (16,777,216 points)."""
    ic = ics.clustered_3d(n=16_777_216, seed=4)
    with Context(dim=3, k=190) as ctx:
        _same(ic, ctx.ic_generate(ic.spec))


def test_sim_from_device_ic_equals_sim_from_host_arrays():
    ic = ics.clustered_3d(n=200_000, seed=7)
    states = []
    for dev in (False, True):
        with Context(dim=3, k=190, buff=0.12, boundary="periodic", flux="physical", gamma=ic.gamma) as ctx:
            if dev:
                ctx.sim_init_ic(ic.spec)
            else:
                ctx.sim_init(ic.pos, ic.rho, ic.vel, ic.energy, ic.deposit)
            ctx.sim_step(0.3)
            states.append(ctx.sim_get())
    for a, b in zip(*states):
        assert np.array_equal(a, b)


def test_batch_from_device_ics_equals_batch_from_host_arrays():
    B = ics.batch_2d(n_inst=12, seed=5, n_min=1000, n_max=20000)
    states = []
    for dev in (False, True):
        with Context(dim=2, k=32, buff=0.04, boundary="periodic", flux="physical", predicates="robust") as ctx:
            if dev:
                ctx.batch_init_ic([ic.spec for ic in B.instances], B.buff, B.boundary)
            else:
                ctx.batch_init(B.counts, B.buff, B.gamma, B.boundary, B.concat("pos"), B.concat("rho"),
                               B.concat("vel"), B.concat("energy"), B.concat("deposit"))
            for _ in range(2):
                ctx.sim_step(0.3)
            states.append(ctx.sim_get())
    for a, b in zip(*states):
        assert np.array_equal(a, b)
