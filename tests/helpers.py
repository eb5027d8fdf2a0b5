"""Comparison helpers shared by the parity tests."""
import numpy as np

# Stated per-field tolerances of the CUDA path against the FP64 oracle.
# Topology (statuses, face counts, neighbour ids, face order) is compared bit-exactly.
TOL = {
    "normal": 0.0,        # bit-identical: same plane equation and normalisation
    "area_2d": 0.0,       # bit-identical: same two vertices, same formula
    "area_3d": 1e-11,     # relative; vertex order inside a cell differs -> fan rounding
    "volume_2d": 1e-12,   # relative; same angular order, centroid sum order differs
    "volume_3d": 1e-11,   # relative (small clustered cells: offsets from O(1) coordinates)
    "centroid": 1e-11,    # absolute, unit box
    "hydro": 1e-10,       # relative, after a few steps on the two meshes
}


def rel_err(a, b, floor_frac=1e-9):
    """max |a - b| / max(|b|, floor), floor = floor_frac x median |b|: relative error,
    except for values that are zero up to rounding (degenerate faces of mirror-symmetric
    point sets), where only an absolute error far below the typical magnitude is meaningful."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    if a.size == 0:
        return 0.0
    floor = max(floor_frac * float(np.median(np.abs(b))), 1e-300)
    return float((np.abs(a - b) / np.maximum(np.abs(b), floor)).max())


def status_pairs(g, o):
    """{(gpu status, oracle status): count} over cells where they differ."""
    gs, os_ = np.asarray(g.status), np.asarray(o.status)
    d = np.nonzero(gs != os_)[0]
    pairs = {}
    for i in d:
        pairs[(int(gs[i]), int(os_[i]))] = pairs.get((int(gs[i]), int(os_[i])), 0) + 1
    return pairs


def assert_same_topology(g, o, failure_codes_may_differ=False):
    """Statuses, face counts and ordered neighbour lists equal (cells in input order).

    failure_codes_may_differ: the set of extracted (SUCCESS) cells and their faces must
    still be identical, but a failed cell may carry a different failure code.  Used for
    mirror-symmetric point sets, where coincident planes create vertices with w = 0 and
    the reference's running std::max (cell.cpp:377) then depends on vertex order."""
    assert g.n_seeds == o.n_seeds and g.n_hydro == o.n_hydro
    gs, os_ = np.asarray(g.status), np.asarray(o.status)
    if failure_codes_may_differ:
        assert np.array_equal(gs == 4, os_ == 4), f"extracted cells differ: {status_pairs(g, o)}"
    else:
        assert np.array_equal(gs, os_), f"statuses differ: {status_pairs(g, o)}"
    assert np.array_equal(np.asarray(g.face_counts, np.int64), np.asarray(o.face_counts, np.int64))
    assert g.num_faces == o.num_faces
    assert np.array_equal(np.asarray(g.neighbor), np.asarray(o.neighbor)), "neighbour lists differ"


def faces_of(m, cells):
    """Concatenated face indices of the given cells (each cell's faces in stored order)."""
    fp = np.asarray(m.face_ptr, np.int64)
    fc = np.asarray(m.face_counts, np.int64)
    cells = np.asarray(cells, np.int64)
    if len(cells) == 0:
        return np.zeros(0, np.int64)
    return np.concatenate([np.arange(fp[c], fp[c] + fc[c]) for c in cells])


def cell_faces(m, c):
    s = int(m.face_ptr[c])
    return slice(s, s + int(m.face_counts[c]))
