"""The checker extensions of the oracle (listed-query KNN, listed cells, growing budget)
against the pinned restatement: identical rows and cells."""
import numpy as np

import oracle as om
from proteusgpu_b200 import ics


def test_grid_knn_rows_equal_full_knn():
    for dim, n, k in ((3, 30000, 190), (2, 20000, 16), (3, 5000, 1000)):
        pts = np.random.default_rng(dim + n).random((n, dim))
        full = om.knn(pts, k)
        g = om.Grid(pts)
        q = np.arange(0, n, 3)
        assert np.array_equal(g.knn(q, k), full[q])


def test_grid_knn_clustered_large_budget():
    ic = ics.clustered_3d(n=40000, seed=4)
    ext, _, _ = om.ghosts(ic.pos, 0.15)
    g = om.Grid(ext)
    q = np.arange(0, 40000, 97)
    assert np.array_equal(g.knn(q, 2000), om.knn(ext, 2000)[q])


def test_listed_cells_equal_full_cells():
    ic = ics.sedov_3d(n=20000, seed=6)
    ext, _, _ = om.ghosts(ic.pos, 0.1)
    kl = om.knn(ext, 64)
    full = om.cells(ext, 20000, kl, n_compute=20000)
    ids = np.arange(7, 20000, 13)
    lst = om.cells_list(ext, ids, kl[ids])
    assert np.array_equal(lst.status, full.status[ids]) and np.array_equal(lst.cert_k, full.cert_k[ids])
    assert np.array_equal(lst.volumes, full.volumes[ids])
    for t, i in enumerate(ids):
        a = slice(lst.face_ptr[t], lst.face_ptr[t] + lst.face_counts[t])
        b = slice(full.face_ptr[i], full.face_ptr[i] + full.face_counts[i])
        assert np.array_equal(lst.neighbor[a], full.neighbor[b]) and np.array_equal(lst.area[a], full.area[b])


def test_growing_budget_equals_large_fixed_budget():
    """Cells that need more than K = 32 neighbours: the growing budget certifies them with
    the same result as one pass at K = 512 (the clipping stops where the certificate closes)."""
    ic = ics.sedov_3d(n=20000, seed=6)
    ext, _, _ = om.ghosts(ic.pos, 0.1)
    g = om.Grid(ext)
    ids = np.arange(20000)
    m, ku = om.cells_certified(g, ids, 32, 512)
    ref = om.cells_list(ext, ids, g.knn(ids, 512))
    assert (ku > 32).sum() > 100 and (m.status == om.SUCCESS).all()
    assert np.array_equal(m.status, ref.status) and np.array_equal(m.cert_k, ref.cert_k)
    assert np.array_equal(m.volumes, ref.volumes) and np.array_equal(m.neighbor, ref.neighbor)
    # the hydro-only build with the growing budget gives the same cells
    b = om.build_mesh(ic.pos, 32, buff=0.1, hydro_only=True, expand_k=512)
    s = 1.2 ** 3
    assert np.array_equal(b.status[:20000], m.status)
    assert np.allclose(b.volumes[:20000], s * m.volumes, rtol=1e-15, atol=0)
