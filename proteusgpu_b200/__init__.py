"""B200 (sm_100a) implementation of ProteusGPU's per-timestep mesh-and-flux path.

Ghost layer, Morton grid sort, exact KNN, Ray et al. half-space clipping with
the security-radius certificate, extraction, CFL step and HLL flux update with
mesh-point drift, as hand-written CUDA kernels behind the C ABI declared in
include/proteus_gpu.h.  ``Context`` mirrors the reference's knn:: / voronoi:: /
hydro:: entry points.
"""
from .core import Context, Mesh, STATUS_SUCCESS, STATUS_NOT_COMPUTED  # noqa: F401
from . import ics  # noqa: F401

__all__ = ["Context", "Mesh", "ics", "STATUS_SUCCESS", "STATUS_NOT_COMPUTED"]
