"""GPU KNN parity: identical ordered neighbour lists (ties by index) against the oracle."""
import numpy as np
import pytest

import oracle as om
from proteusgpu_b200 import Context, ics

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dim,k", [(2, 1), (2, 16), (2, 32), (2, 33), (2, 64), (3, 16), (3, 64), (3, 100),
                                   (3, 190), (3, 256)])
def test_knn_uniform(dim, k):
    pts = ics.uniform_points(6000 if dim == 2 else 9000, dim, 40 + k)
    with Context(dim=dim, k=k) as ctx:
        g = ctx.knn(pts)
    assert np.array_equal(g, om.knn(pts, k))


def test_knn_clustered_contrast():
    ic = ics.clustered_3d(n=40000, seed=9)
    with Context(dim=3, k=48) as ctx:
        g = ctx.knn(ic.pos)
    assert np.array_equal(g, om.knn(ic.pos, 48))


def test_knn_fewer_points_than_k():
    pts = ics.uniform_points(10, 3, 3)
    with Context(dim=3, k=16) as ctx:
        g = ctx.knn(pts)
    o = om.knn(pts, 16)
    assert np.array_equal(g, o)
    assert (g[:, 9:] == np.iinfo(np.uint32).max).all()


def test_knn_duplicates_and_ties():
    rng = np.random.default_rng(5)
    base = rng.random((500, 3))
    pts = np.concatenate([base, base[:100]])  # exact duplicates (distance 0)
    with Context(dim=3, k=20) as ctx:
        g = ctx.knn(pts)
    assert np.array_equal(g, om.knn(pts, 20))


def test_knn_sorted_order_is_a_permutation():
    pts = ics.uniform_points(5000, 2, 4)
    with Context(dim=2, k=8) as ctx:
        ctx.knn(pts)
        sp, perm, ng = ctx.knn_sorted()
    assert sorted(perm.tolist()) == list(range(5000))
    assert np.array_equal(sp, pts[perm])
    assert ng >= 1
