"""FP32 local-frame clipping (precision form): the mesh must equal the FP64 path's bit for bit.

Undecided predicates go to the FP64 kernel, certified cells are extracted in FP64
from the same vertex lists, and the certificate is re-checked in FP64, so every
field -- statuses, certified K, neighbour lists, normals, areas, volumes,
centroids -- equals the FP64 mode's, and therefore the oracle's within the
FP64 tolerances.
"""
import numpy as np
import pytest

import oracle as om
from helpers import assert_same_topology
from proteusgpu_b200 import Context, ics

pytestmark = pytest.mark.gpu

FIELDS = ("status", "cert_k", "face_counts", "face_ptr", "neighbor", "normal", "area", "volumes", "seeds")


def both(dim, k, pts, unit=False, **kw):
    out = []
    for prec in ("fp64", "fp32"):
        with Context(dim=dim, k=k, precision=prec, **kw) as ctx:
            out.append(ctx.compute_mesh(pts) if unit else ctx.compute_periodic_mesh(pts))
            out.append(ctx.stats())
    return out


def assert_identical(a, b):
    for f in FIELDS:
        assert np.array_equal(getattr(a, f), getattr(b, f)), f
    ok = a.status == 4
    assert np.array_equal(a.centroid[ok], b.centroid[ok])


@pytest.mark.parametrize("k", [16, 32])
def test_fp32_sod_2d(k):
    ic = ics.sod_2d()
    g64, _, g32, st = both(2, k, ic.pos, gamma=1.4)
    assert_identical(g64, g32)
    assert_same_topology(g32, om.build_mesh(ic.pos, k))


@pytest.mark.parametrize("k", [64, 190])
def test_fp32_uniform_3d(k):
    pts = ics.uniform_points(20000, 3, 7)
    g64, _, g32, st = both(3, k, pts, buff=0.1)
    assert_identical(g64, g32)
    assert_same_topology(g32, om.build_mesh(pts, k, buff=0.1))


def test_fp32_clustered_3d():
    pts = ics.clustered_3d(n=30000, seed=4).pos
    g64, _, g32, st = both(3, 190, pts, buff=0.1)
    assert_identical(g64, g32)


def test_fp32_failing_cells_and_ties():
    pts = ics.uniform_points(13000, 3, 22)
    ext = np.ascontiguousarray((pts - 0.5) / 1.2 + 0.5)
    g64, _, g32, _ = both(3, 32, ext, unit=True)
    assert_identical(g64, g32)
    lat = ics.jittered_lattice(48, 2, 0.0, np.random.default_rng(0))  # exact cocircular quadruples
    g64, _, g32, st = both(2, 24, lat, unit=True)
    assert_identical(g64, g32)
    assert st["reclip_cells"] > 0  # degenerate predicates are undecided in FP32 and go to FP64


def test_fp32_moving_mesh_steps():
    ic = ics.sedov_3d(n=20000, seed=6)
    res = []
    for prec in ("fp64", "fp32"):
        with Context(dim=3, k=190, buff=0.1, flux="physical", precision=prec) as ctx:
            ctx.sim_init(ic.pos, ic.rho, ic.vel, ic.energy, ic.deposit)
            dts = [ctx.sim_step(0.3) for _ in range(3)]
            res.append((dts,) + ctx.sim_get())
    for a, b in zip(res[0], res[1]):
        assert np.array_equal(np.asarray(a), np.asarray(b))


@pytest.mark.parametrize("sep", [1e-6, 1e-7, 1e-8])
def test_fp32_near_coincident_seeds(sep):
    """Pairs of seeds sep apart (500 pairs among 20,000 uniform points, random
    directions): tiny faces whose global-frame FP64 determinants carry a large
    rounding relative to the face.  The FP32 form must still equal the FP64 form."""
    rng = np.random.default_rng(41)
    pts = ics.uniform_points(20000, 3, 40)
    d = rng.normal(size=(500, 3))
    d *= sep / np.linalg.norm(d, axis=1)[:, None]
    twins = np.clip(pts[:500] + d, 0.0, np.nextafter(1.0, 0.0))
    pts = np.concatenate([pts, twins])
    g64, s64, g32, s32 = both(3, 190, pts, buff=0.1)
    assert_identical(g64, g32)
    assert_same_topology(g64, om.build_mesh(pts, 190, buff=0.1))
