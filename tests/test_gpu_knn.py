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


def _dense_blob(n_blob, n_bg, dim, sigma, seed):
    rng = np.random.default_rng(seed)
    blob = 0.5 + sigma * rng.standard_normal((n_blob, dim))
    pts = np.concatenate([np.clip(blob, 0.0, 1.0 - 1e-12), rng.random((n_bg, dim))])
    return np.ascontiguousarray(pts)


@pytest.mark.parametrize("dim,k", [(3, 64), (3, 190), (2, 32)])
def test_knn_refined_bins(dim, k):
    """A blob thousands of times denser than the background: its coarse bins are
    split into sub-bins (up to the deepest level) and queries search at the
    blob's spacing; queries at the blob's edge mix levels."""
    pts = _dense_blob(30000, 8000, dim, 0.002 if dim == 3 else 0.001, 11 + dim)
    with Context(dim=dim, k=k) as ctx:
        g = ctx.knn(pts)
    assert np.array_equal(g, om.knn(pts, k))


def test_knn_refined_lattice_on_box_edges():
    """Unjittered points on the sub-bin grid lines of a refined region (coordinates
    that are exact multiples of the sub-bin side) next to a sparse background."""
    rng = np.random.default_rng(21)
    side = 1.0 / 2048
    g1 = (np.arange(40) * side + 0.25)
    lat = np.stack(np.meshgrid(g1, g1, indexing="ij"), -1).reshape(-1, 2)
    pts = np.ascontiguousarray(np.concatenate([lat, rng.random((3000, 2))]))
    with Context(dim=2, k=24) as ctx:
        g = ctx.knn(pts)
    assert np.array_equal(g, om.knn(pts, 24))


def test_knn_many_duplicates_in_one_bin():
    rng = np.random.default_rng(22)
    base = rng.random((2000, 3))
    pts = np.ascontiguousarray(np.concatenate([base, np.repeat(base[:3], 400, axis=0)]))
    with Context(dim=3, k=32) as ctx:
        g = ctx.knn(pts)
    assert np.array_equal(g, om.knn(pts, 32))


def _knn_thread(pts, k, kt):
    with Context(dim=pts.shape[1], k=k) as ctx:
        ctx.set_tuning(knn_thread=kt)
        return ctx.knn(pts)


@pytest.mark.parametrize("case,k,kt", [("uniform2", 16, 32), ("uniform2", 32, 32), ("uniform2", 48, 64),
                                       ("uniform3", 64, 64), ("uniform3", 100, 64), ("blob3", 64, 64),
                                       ("blob2", 32, 32), ("lattice2", 24, 32), ("dups3", 20, 32),
                                       ("few3", 16, 32)])
def test_knn_thread_per_query(case, k, kt):
    """One thread per query (the small-K kernel) gives the warp kernel's lists: the
    same exact K nearest with ties by index, over refined bins, grid-line points,
    duplicates and fewer points than K."""
    rng = np.random.default_rng(sum(map(ord, case)) + k)
    if case == "uniform2":
        pts = ics.uniform_points(6000, 2, 50 + k)
    elif case == "uniform3":
        pts = ics.uniform_points(9000, 3, 50 + k)
    elif case == "blob3":
        pts = _dense_blob(30000, 8000, 3, 0.002, 14)
    elif case == "blob2":
        pts = _dense_blob(30000, 8000, 2, 0.001, 13)
    elif case == "lattice2":
        g1 = np.arange(40) / 2048 + 0.25
        lat = np.stack(np.meshgrid(g1, g1, indexing="ij"), -1).reshape(-1, 2)
        pts = np.ascontiguousarray(np.concatenate([lat, rng.random((3000, 2))]))
    elif case == "dups3":
        base = rng.random((500, 3))
        pts = np.ascontiguousarray(np.concatenate([base, base[:100]]))
    else:
        pts = ics.uniform_points(10, 3, 3)
    assert np.array_equal(_knn_thread(pts, k, kt), om.knn(pts, k))


def test_knn_sub_bin_beyond_the_deepest_level():
    """Thousands of points inside one deepest-level sub-bin (a pile-up far denser than
    the refinement can split): such sub-bins are sorted by a block, and the lists and
    the sorted order (ids ascending inside the sub-bin) stay the same as for small ones."""
    rng = np.random.default_rng(31)
    pile = 0.4321 + 1e-9 * rng.random((9000, 3))       # > 8192: keys sorted in global scratch
    pile2 = 0.7123 + 1e-9 * rng.random((3000, 3))      # <= 8192: keys sorted in shared memory
    pts = np.ascontiguousarray(np.concatenate([rng.random((20000, 3)), pile, pile2]))
    with Context(dim=3, k=24) as ctx:
        g = ctx.knn(pts)
        sp, perm, _ = ctx.knn_sorted()
        g2 = ctx.knn(pts)
    assert np.array_equal(g, om.knn(pts, 24)) and np.array_equal(g, g2)
    for lo, hi in ((20000, 29000), (29000, 32000)):
        at = np.nonzero((perm >= lo) & (perm < hi))[0]
        assert np.array_equal(at, np.arange(at[0], at[0] + len(at)))  # contiguous: one sub-bin
        assert np.array_equal(perm[at], np.arange(lo, hi))            # ids ascending inside it
    assert np.array_equal(sp, pts[perm])


@pytest.mark.parametrize("kt", [0, 64])
def test_knn_packed_key_ties_are_redone_exactly(kt):
    """A regular lattice puts exact distance ties everywhere: the packed-key search (warp
    kernel, or the thread-per-query kernel with kt) flags those queries and the exact-key
    search redoes them; the lists equal the oracle's, ties by index."""
    g1 = (np.arange(24) + 0.5) / 24
    pts = np.ascontiguousarray(np.stack(np.meshgrid(g1, g1, g1, indexing="ij"), -1).reshape(-1, 3))
    with Context(dim=3, k=40) as ctx:
        ctx.set_tuning(knn_thread=kt)
        g = ctx.knn(pts)
        st = ctx.stats()
    assert st["knn_redone"] > 0
    assert np.array_equal(g, om.knn(pts, 40))
