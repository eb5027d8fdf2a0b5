"""pgpu_dt_cfl_static -- the CFL step from the caller's device arrays, no allocation --
against pgpu_dt_cfl on the same mesh and primitives, through the C ABI.

Collected last (file name) so that it also runs after every other GPU test has
used the library on the same device.  Device arrays for the call are made with
torch here in the test; the entry point itself allocates nothing.
"""
import ctypes as C

import numpy as np
import pytest

from proteusgpu_b200 import Context, _lib, ics

pytestmark = pytest.mark.gpu

PGPU_ECAPACITY = -4
PGPU_EINVAL = -1
MAX_CELLS = 16777216


def _case(dim):
    rng = np.random.default_rng(11 + dim)
    if dim == 2:
        pts, gamma, k = ics.sod_2d().pos, 1.4, 16
    else:
        pts, gamma, k = ics.uniform_points(20000, 3, 5), 5.0 / 3.0, 190
    n = len(pts)
    rho = rng.uniform(0.5, 2.0, n)
    v = rng.normal(0.0, 0.3, (n, dim))
    P = rng.uniform(0.1, 1.0, n)
    E = P / (gamma - 1.0) + 0.5 * rho * (v * v).sum(1)
    return pts, gamma, k, rho, v, E


def _static_dt(L, dim, gamma, cfl, dev_arrays, n, stream):
    dt = C.c_double(-1.0)
    rho, v, E, vol = (C.c_void_p(t.data_ptr()) for t in dev_arrays)
    rc = L.pgpu_dt_cfl_static(dim, gamma, cfl, rho, v, E, vol, n, C.c_void_p(stream), C.byref(dt))
    assert rc == 0
    return dt.value


@pytest.mark.parametrize("dim", [2, 3])
def test_static_dt_matches_context_dt(dim):
    torch = pytest.importorskip("torch")
    pts, gamma, k, rho, v, E = _case(dim)
    cfl = 0.3
    with Context(dim=dim, k=k, gamma=gamma, buff=0.04 if dim == 2 else 0.1) as ctx:
        mesh = ctx.compute_periodic_mesh(pts)
        ctx.set_prim(rho, v, E)
        want = ctx.dt_cfl(cfl)
    nh = mesh.n_hydro
    assert nh == len(pts) and want > 0.0
    dev = [torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda:0")
           for a in (rho, v, E, mesh.volumes[:nh])]
    torch.cuda.synchronize()
    L = _lib.load()
    stream = torch.cuda.current_stream().cuda_stream
    first = _static_dt(L, dim, gamma, cfl, dev, nh, stream)
    second = _static_dt(L, dim, gamma, cfl, dev, nh, stream)
    # same per-cell formula and an exact minimum: equal to rounding (in practice bit-equal)
    assert abs(first - want) <= 1e-15 * want
    assert abs(second - want) <= 1e-15 * want
    # a different CFL number on the same scratch: no state carried between calls
    assert abs(_static_dt(L, dim, gamma, 0.1, dev, nh, stream) - want / 3.0) <= 1e-14 * want


def test_static_dt_allocates_nothing_at_its_largest_size():
    """Repeated calls at the largest accepted n leave the device's free memory unchanged
    (cudaMemGetInfo before and after), and every call returns the same step."""
    torch = pytest.importorskip("torch")
    n, gamma, cfl = MAX_CELLS, 5.0 / 3.0, 0.3
    g = torch.Generator(device="cuda:0").manual_seed(5)
    rho = torch.rand(n, dtype=torch.float64, device="cuda:0", generator=g) + 0.5
    v = torch.randn(n * 3, dtype=torch.float64, device="cuda:0", generator=g) * 0.3
    E = torch.rand(n, dtype=torch.float64, device="cuda:0", generator=g) + 1.0
    vol = torch.rand(n, dtype=torch.float64, device="cuda:0", generator=g) * 1e-7 + 1e-8
    torch.cuda.synchronize()
    L = _lib.load()
    stream = torch.cuda.current_stream().cuda_stream
    first = _static_dt(L, 3, gamma, cfl, (rho, v, E, vol), n, stream)  # the first call does the set-up
    torch.cuda.synchronize()
    free0, _total = torch.cuda.mem_get_info(0)
    vals = [_static_dt(L, 3, gamma, cfl, (rho, v, E, vol), n, stream) for _ in range(20)]
    torch.cuda.synchronize()
    free1, _total = torch.cuda.mem_get_info(0)
    assert free1 == free0, f"device free memory changed by {free0 - free1} bytes"
    assert all(x == first for x in vals) and first > 0.0


def test_static_dt_rejects_sizes_beyond_its_scratch():
    L = _lib.load()
    dt = C.c_double(-1.0)
    one = (C.c_double * 1)()
    p = C.cast(one, C.c_void_p)
    assert L.pgpu_dt_cfl_static(3, 5.0 / 3.0, 0.3, p, p, p, p, MAX_CELLS + 1, None, C.byref(dt)) == PGPU_ECAPACITY
    assert L.pgpu_dt_cfl_static(4, 5.0 / 3.0, 0.3, p, p, p, p, 1, None, C.byref(dt)) == PGPU_EINVAL
    assert L.pgpu_dt_cfl_static(3, 5.0 / 3.0, 0.3, p, p, p, p, 0, None, C.byref(dt)) == PGPU_EINVAL
    assert dt.value == -1.0
