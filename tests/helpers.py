"""Comparison helpers shared by the parity tests."""
import numpy as np

# Stated per-field tolerances of the CUDA path against the FP64 oracle.
# Topology (statuses, face counts, neighbour ids, face order) is compared bit-exactly.
TOL = {
    "normal": 0.0,        # bit-identical: same plane equation and normalisation
    "area_2d": 0.0,       # bit-identical: same two vertices, same formula
    "area_3d": 1e-12,     # relative; vertex order inside a cell differs -> fan rounding
    "volume_2d": 1e-12,   # relative; same angular order, centroid sum order differs
    "volume_3d": 1e-12,   # relative
    "centroid": 1e-11,    # absolute, unit box
    "hydro": 1e-10,       # relative, after a few steps on the two meshes
}


def rel_err(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    if a.size == 0:
        return 0.0
    return float((np.abs(a - b) / np.maximum(np.abs(b), 1e-300)).max())


def assert_same_topology(g, o, cells=None):
    """Statuses, face counts and ordered neighbour lists equal (cells in input order)."""
    assert g.n_seeds == o.n_seeds and g.n_hydro == o.n_hydro
    if cells is None:
        assert np.array_equal(np.asarray(g.status), np.asarray(o.status)), "statuses differ"
        assert np.array_equal(np.asarray(g.face_counts, np.int64), np.asarray(o.face_counts, np.int64))
        assert g.num_faces == o.num_faces
        assert np.array_equal(np.asarray(g.neighbor), np.asarray(o.neighbor)), "neighbour lists differ"


def cell_faces(m, c):
    s = int(m.face_ptr[c])
    return slice(s, s + int(m.face_counts[c]))
