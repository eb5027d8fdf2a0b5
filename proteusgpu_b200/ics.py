"""Seeded initial conditions for the mesh-and-flux workloads.

The reference reads its initial conditions from HDF5 files written by
``create.py`` / ``create_sod.py`` (datasets ``seedpos`` N x D, ``rho`` N,
``vel`` N x D, ``Energy`` N; src/io/input.cpp:121-309).  h5py is not available
here, so these generators build the same four fields in memory from fixed seeds.
``Energy`` is the total energy per unit volume, as in the reference's
``primvars::E`` (src/global/allvars.h:203-207).

The workload generators (sod_2d, sedov_2d, sedov_3d, kh_2d, clustered_3d and the
instances of batch_2d) draw from a counter-based generator so that the device
can produce the same initial conditions bit for bit (pgpu_ic_generate,
csrc/ics.cu): every random number is a pure function of (seed, stream, index),
and the few transcendental functions used (ln, exp, sin, cos) are evaluated with
the same sequence of IEEE double operations on both sides instead of the
platforms' own libraries:
  * random words: the SplitMix64 output function (Steele, Lea, Flood, "Fast
    splittable pseudorandom number generators", OOPSLA 2014) applied to
    key + (index + 1) * 0x9E3779B97F4A7C15, key = mix(seed * 0x9E37... + stream);
    uniforms are the top 53 bits times 2^-53;
  * normals: Marsaglia's polar method, attempt j of sample i drawing the words
    128 i + 2 j and 128 i + 2 j + 1 of its stream;
  * ln(x) = e ln 2 + 2 atanh((m - 1) / (m + 1)) for x = m 2^e, m in [sqrt(1/2), sqrt(2)),
    atanh by its odd series to t^21; exp(x) = 2^k exp(r), r = x - k ln 2, Taylor
    to r^13; sin and cos by quadrant reduction with pi/2 and Taylor series to r^17.

uniform_points and jittered_lattice (numpy's generator) remain for arbitrary
test point sets and the golden fixtures.  Each generator returns an :class:`IC`
whose arrays are C-contiguous float64.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np


@dataclasses.dataclass
class IC:
    name: str
    dim: int
    pos: np.ndarray          # (N, dim) generating points in [0, 1)^dim
    rho: np.ndarray          # (N,)
    vel: np.ndarray          # (N, dim)
    energy: np.ndarray       # (N,) total energy per unit volume
    gamma: float
    boundary: str = "periodic"      # "periodic" or "reflective"
    # Energy added per cell (not per volume) once the first mesh gives volumes;
    # used by the Sedov blast deposit.  None when there is no deposit.
    deposit: np.ndarray | None = None
    # the generator's arguments (what pgpu_ic_generate needs to make it on the device)
    spec: dict | None = None

    @property
    def n(self) -> int:
        return int(self.pos.shape[0])


def _finish(ic: IC) -> IC:
    for f in ("pos", "rho", "vel", "energy"):
        setattr(ic, f, np.ascontiguousarray(getattr(ic, f), dtype=np.float64))
    if ic.deposit is not None:
        ic.deposit = np.ascontiguousarray(ic.deposit, dtype=np.float64)
    return ic


# ------------------------------------------------------------------ counter-based generator
_M64 = (1 << 64) - 1
_GOLDEN = 0x9E3779B97F4A7C15
_U = np.uint64

# stream ids (shared with csrc/ics.cu)
S_JITTER, S_POS, S_CENTRE, S_SIGMA, S_WHICH, S_GAUSS, S_NOISE = 1, 2, 3, 4, 5, 6, 7

LN2 = 0.6931471805599453
PI = 3.141592653589793
HALF_PI = 1.5707963267948966
SQRT_HALF = 0.7071067811865476


def _mix_int(z: int) -> int:
    z &= _M64
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & _M64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & _M64
    return z ^ (z >> 31)


def stream_key(seed: int, stream: int) -> int:
    """The 64-bit key of one stream of a seed."""
    return _mix_int((seed * _GOLDEN + stream) & _M64)


def _mix(z: np.ndarray) -> np.ndarray:
    with np.errstate(over="ignore"):
        z = (z ^ (z >> _U(30))) * _U(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> _U(27))) * _U(0x94D049BB133111EB)
    return z ^ (z >> _U(31))


def words(key: int, idx) -> np.ndarray:
    """Random 64-bit words number idx of the stream with this key."""
    i = np.asarray(idx, dtype=np.uint64)
    with np.errstate(over="ignore"):
        return _mix(_U(key) + (i + _U(1)) * _U(_GOLDEN))


def unif(key: int, idx) -> np.ndarray:
    """Uniform doubles in [0, 1): the top 53 bits of each word times 2^-53."""
    return (words(key, idx) >> _U(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def log_d(x) -> np.ndarray:
    """ln x for x > 0 (normal numbers), the same operation sequence as the device's."""
    x = np.asarray(x, np.float64)
    m, e = np.frexp(x)
    small = m < SQRT_HALF
    m = np.where(small, m * 2.0, m)
    e = np.where(small, e - 1, e).astype(np.float64)
    t = (m - 1.0) / (m + 1.0)
    t2 = t * t
    s = np.full_like(t, 1.0 / 21.0)
    for k in (19, 17, 15, 13, 11, 9, 7, 5, 3):
        s = s * t2 + 1.0 / k
    s = s * t2 + 1.0
    return e * LN2 + 2.0 * t * s


_EXP_C = [1.0 / math.factorial(j) for j in range(14)]


def exp_d(x) -> np.ndarray:
    """exp x for moderate |x|, the same operation sequence as the device's."""
    x = np.asarray(x, np.float64)
    k = np.rint(x * (1.0 / LN2))
    r = x - k * LN2
    s = np.full_like(r, _EXP_C[13])
    for j in range(12, 0, -1):
        s = s * r + _EXP_C[j]
    s = s * r + 1.0
    return np.ldexp(s, k.astype(np.int64))


_SIN_C = [(-1.0) ** j / math.factorial(2 * j + 1) for j in range(9)]   # r, r^3, ..., r^17
_COS_C = [(-1.0) ** j / math.factorial(2 * j) for j in range(10)]      # 1, r^2, ..., r^18


def _sincos_red(r):
    r2 = r * r
    s = np.full_like(r, _SIN_C[8])
    for j in range(7, -1, -1):
        s = s * r2 + _SIN_C[j]
    s = s * r
    c = np.full_like(r, _COS_C[9])
    for j in range(8, -1, -1):
        c = c * r2 + _COS_C[j]
    return s, c


def sin_d(x) -> np.ndarray:
    """sin x for moderate |x|: x = k pi/2 + r, |r| <= pi/4, series by quadrant."""
    x = np.asarray(x, np.float64)
    k = np.rint(x * (1.0 / HALF_PI))
    r = x - k * HALF_PI
    s, c = _sincos_red(r)
    q = k.astype(np.int64) & 3
    return np.select([q == 0, q == 1, q == 2], [s, c, -s], -c)


def cos_d(x) -> np.ndarray:
    x = np.asarray(x, np.float64)
    k = np.rint(x * (1.0 / HALF_PI))
    r = x - k * HALF_PI
    s, c = _sincos_red(r)
    q = k.astype(np.int64) & 3
    return np.select([q == 0, q == 1, q == 2], [c, -s, -c], s)


def normals(key: int, idx) -> np.ndarray:
    """Standard normal doubles number idx of a stream (Marsaglia's polar method; attempt
    j of sample i uses words 128 i + 2 j and 128 i + 2 j + 1, at most 64 attempts)."""
    idx = np.asarray(idx, dtype=np.uint64).ravel()
    out = np.zeros(len(idx))
    pend = np.arange(len(idx))
    for j in range(64):
        if len(pend) == 0:
            break
        c = idx[pend] * _U(128) + _U(2 * j)
        u = 2.0 * unif(key, c) - 1.0
        v = 2.0 * unif(key, c + _U(1)) - 1.0
        s = u * u + v * v
        ok = (s < 1.0) & (s > 0.0)
        so = s[ok]
        out[pend[ok]] = u[ok] * np.sqrt(-2.0 * log_d(so) / so)
        pend = pend[~ok]
    return out


def _wrap01(p):
    """[0, 1) wrap of a coordinate: fmod, + 1 below zero, and 1.0 (a rounding of a tiny
    negative) to 0."""
    r = np.fmod(p, 1.0)
    r = np.where(r < 0.0, r + 1.0, r)
    return np.where(r >= 1.0, 0.0, r)


def _lattice(n_side: int, dim: int, jitter: float, seed: int) -> np.ndarray:
    """Cell centres of an n_side^dim lattice (x fastest), each moved by U(-jitter, jitter)
    x spacing per axis, clipped into [0, 1)."""
    n = n_side ** dim
    i = np.arange(n, dtype=np.int64)
    h = 1.0 / n_side
    key = stream_key(seed, S_JITTER)
    cols = []
    rest = i
    for a in range(dim):
        ia = rest % n_side
        rest = rest // n_side
        base = (ia.astype(np.float64) + 0.5) * h
        j = (2.0 * unif(key, dim * i + a) - 1.0) * jitter
        cols.append(np.clip(base + j * h, 0.0, np.nextafter(1.0, 0.0)))
    return np.stack(cols, axis=1)


def _uniform(n: int, dim: int, seed: int, stream: int = S_POS) -> np.ndarray:
    i = np.arange(n, dtype=np.int64)
    key = stream_key(seed, stream)
    return np.stack([unif(key, dim * i + a) for a in range(dim)], axis=1)


def blast_deposit(pos: np.ndarray, e_total: float, n_dep: int = 32, sigma: float = 0.01) -> np.ndarray:
    """Energy per cell for a blast of ``e_total`` over the ``n_dep`` points nearest the box
    centre (ties by index), weighted by exp(-r^2 / (2 sigma^2)) and normalised by their
    sum taken nearest first."""
    dim = pos.shape[1]
    d2 = np.zeros(len(pos))
    for a in range(dim):
        d = pos[:, a] - 0.5
        d2 = d2 + d * d
    order = np.lexsort((np.arange(len(d2)), d2))[:n_dep]
    w = exp_d(-d2[order] / (2.0 * sigma * sigma))
    tot = 0.0
    for x in w:
        tot = tot + float(x)
    dep = np.zeros(len(pos))
    dep[order] = e_total * (w / tot)
    return dep


def sod_2d(n_side: int = 100, seed: int = 1, jitter: float = 0.1, gamma: float = 1.4,
           boundary: str = "reflective", split_angle: float = 0.0) -> IC:
    """2D Sod shock tube on a jittered lattice (left rho=1, P=1; right rho=0.125, P=0.1).

    ``split_angle`` rotates the discontinuity about the box centre (0 = split at x=0.5)."""
    spec = sod_2d_spec(n_side, seed, jitter, gamma, split_angle)
    pos = _lattice(n_side, 2, jitter, seed)
    c, s = spec["split_cos"], spec["split_sin"]
    left = ((pos[:, 0] - 0.5) * c + (pos[:, 1] - 0.5) * s) < 0.0
    rho = np.where(left, 1.0, 0.125)
    P = np.where(left, 1.0, 0.1)
    vel = np.zeros_like(pos)
    energy = P / (gamma - 1.0)
    return _finish(IC("sod2d", 2, pos, rho, vel, energy, gamma, boundary, spec=spec))


# The generators' arguments as the device generator takes them (pgpu_ic_spec), without
# generating anything on the host.
def sod_2d_spec(n_side: int = 100, seed: int = 1, jitter: float = 0.1, gamma: float = 1.4,
                split_angle: float = 0.0) -> dict:
    return dict(kind="sod", dim=2, n_side=n_side, seed=seed, jitter=jitter, gamma=gamma,
                split_cos=float(cos_d(split_angle)), split_sin=float(sin_d(split_angle)))


def sedov_spec(dim: int, n: int, seed: int, gamma: float = 5.0 / 3.0, p0: float = 1e-5, e_blast: float = 1.0) -> dict:
    return dict(kind="sedov", dim=dim, n=n, seed=seed, gamma=gamma, p0=p0, e_blast=e_blast)


def kh_2d_spec(n_side: int = 2048, seed: int = 3, gamma: float = 5.0 / 3.0, rho_ratio: float = 2.0) -> dict:
    return dict(kind="kh", dim=2, n_side=n_side, seed=seed, gamma=gamma, rho_ratio=rho_ratio)


def clustered_3d_spec(n: int = 16_777_216, seed: int = 4, n_clumps: int = 64, frac_clumped: float = 0.7,
                      gamma: float = 5.0 / 3.0, p0: float = 1e-5, e_blast: float = 1.0) -> dict:
    return dict(kind="clustered", dim=3, n=n, seed=seed, gamma=gamma, p0=p0, e_blast=e_blast,
                n_clumps=n_clumps, frac_clumped=frac_clumped)


def uniform_points(n: int, dim: int, seed: int) -> np.ndarray:
    """Uniform test points from numpy's generator (test point sets, golden fixtures)."""
    rng = np.random.default_rng(seed)
    return rng.random((n, dim))


def jittered_lattice(n_side: int, dim: int, jitter: float, rng: np.random.Generator) -> np.ndarray:
    """A jittered lattice from numpy's generator (test point sets, golden fixtures)."""
    h = 1.0 / n_side
    axes = [(np.arange(n_side) + 0.5) * h] * dim
    grid = np.stack(np.meshgrid(*axes, indexing="xy"), axis=-1).reshape(-1, dim)
    grid = grid + rng.uniform(-jitter, jitter, size=grid.shape) * h
    return np.clip(grid, 0.0, np.nextafter(1.0, 0.0))


def _sedov_fields(pos, gamma, p0, e_blast):
    n = len(pos)
    return np.ones(n), np.zeros_like(pos), np.full(n, p0 / (gamma - 1.0)), blast_deposit(pos, e_blast)


def sedov_3d(n: int = 1_048_576, seed: int = 2, gamma: float = 5.0 / 3.0, p0: float = 1e-5,
             e_blast: float = 1.0, points: np.ndarray | None = None) -> IC:
    """3D Sedov-Taylor blast: uniform points, rho=1, P=p0, v=0, E deposited near the centre.
    ``points`` replaces the generated positions (no device counterpart then)."""
    pos = _uniform(n, 3, seed) if points is None else np.asarray(points, dtype=np.float64)
    rho, vel, energy, dep = _sedov_fields(pos, gamma, p0, e_blast)
    spec = None if points is not None else sedov_spec(3, n, seed, gamma, p0, e_blast)
    return _finish(IC("sedov3d", 3, pos, rho, vel, energy, gamma, "periodic", dep, spec=spec))


def sedov_2d(n: int, seed: int, gamma: float = 5.0 / 3.0, p0: float = 1e-5, e_blast: float = 1.0) -> IC:
    pos = _uniform(n, 2, seed)
    rho, vel, energy, dep = _sedov_fields(pos, gamma, p0, e_blast)
    spec = sedov_spec(2, n, seed, gamma, p0, e_blast)
    return _finish(IC("sedov2d", 2, pos, rho, vel, energy, gamma, "periodic", dep, spec=spec))


def kh_2d(n_side: int = 2048, seed: int = 3, gamma: float = 5.0 / 3.0, rho_ratio: float = 2.0) -> IC:
    """Kelvin-Helmholtz shear layer on a jittered periodic lattice: rho = rho_ratio, vx = +0.5
    for |y - 0.5| < 0.25, rho = 1, vx = -0.5 elsewhere, P = 2.5, vy = 0.01 sin(4 pi x) plus
    1e-3 white noise."""
    pos = _lattice(n_side, 2, 0.1, seed)
    n = len(pos)
    band = np.abs(pos[:, 1] - 0.5) < 0.25
    rho = np.where(band, rho_ratio, 1.0)
    vx = np.where(band, 0.5, -0.5)
    vy = 0.01 * sin_d((4.0 * PI) * pos[:, 0]) + 1e-3 * normals(stream_key(seed, S_NOISE), np.arange(n))
    vel = np.stack([vx, vy], axis=1)
    P = np.full(n, 2.5)
    energy = P / (gamma - 1.0) + (0.5 * rho) * (vx * vx + vy * vy)
    spec = kh_2d_spec(n_side, seed, gamma, rho_ratio)
    return _finish(IC("kh2d", 2, pos, rho, vel, energy, gamma, "periodic", spec=spec))


def sound_wave_2d(n_side: int, amp: float = 1e-3, seed: int = 1, gamma: float = 5.0 / 3.0) -> IC:
    """A right-moving plane sound wave along x in a periodic box on a jittered lattice:
    rho = 1 + amp s, vx = c amp s, P = 1 + gamma amp s, s = sin(2 pi x), c = sqrt(gamma).
    To first order in amp it travels unchanged at speed c (convergence tests)."""
    pos = jittered_lattice(n_side, 2, 0.1, np.random.default_rng(seed))
    c = math.sqrt(gamma)
    s = np.sin(2.0 * math.pi * pos[:, 0])
    rho = 1.0 + amp * s
    vel = np.stack([c * amp * s, np.zeros(len(pos))], axis=1)
    P = 1.0 + gamma * amp * s
    energy = P / (gamma - 1.0) + 0.5 * rho * vel[:, 0] ** 2
    return _finish(IC("wave2d", 2, pos, rho, vel, energy, gamma, "periodic"))


def clump_params(seed: int, n_clumps: int = 64):
    """Centres (uniform in the box) and widths (log-uniform in [0.005, 0.05]) of the clumps."""
    c = np.arange(n_clumps, dtype=np.int64)
    kc = stream_key(seed, S_CENTRE)
    centres = np.stack([unif(kc, 3 * c + a) for a in range(3)], axis=1)
    lo, hi = log_d(0.005), log_d(0.05)
    sig = exp_d(lo + (hi - lo) * unif(stream_key(seed, S_SIGMA), c))
    return centres, sig


def clustered_3d(n: int = 16_777_216, seed: int = 4, n_clumps: int = 64, frac_clumped: float = 0.7,
                 gamma: float = 5.0 / 3.0, p0: float = 1e-5, e_blast: float = 1.0) -> IC:
    """Clustered 3D Sedov: Gaussian clumps (sigma log-uniform in [0.005, 0.05]) plus a uniform
    background, wrapped periodically into [0,1)^3.  The first round(frac n) points belong to
    clumps (each picks its clump uniformly), the rest are background."""
    centres, sig = clump_params(seed, n_clumps)
    n_cl = int(round(frac_clumped * n))
    i = np.arange(n, dtype=np.int64)
    pos = np.empty((n, 3))
    ic_ = i[:n_cl]
    which = ((words(stream_key(seed, S_WHICH), ic_) >> _U(32)) * _U(n_clumps)) >> _U(32)
    which = which.astype(np.int64)
    kg = stream_key(seed, S_GAUSS)
    for a in range(3):
        g = normals(kg, 3 * ic_ + a)
        pos[:n_cl, a] = _wrap01(centres[which, a] + g * sig[which])
    kb = stream_key(seed, S_POS)
    ib = i[n_cl:]
    for a in range(3):
        pos[n_cl:, a] = unif(kb, 3 * ib + a)
    rho, vel, energy, dep = _sedov_fields(pos, gamma, p0, e_blast)
    spec = clustered_3d_spec(n, seed, n_clumps, frac_clumped, gamma, p0, e_blast)
    return _finish(IC("clustered3d", 3, pos, rho, vel, energy, gamma, "periodic", dep, spec=spec))


@dataclasses.dataclass
class Batch:
    """Independent 2D simulations for a batched run: per-instance ICs plus the
    concatenated arrays pgpu_batch_init takes."""
    instances: list
    buff: np.ndarray

    @property
    def counts(self) -> np.ndarray:
        return np.array([ic.n for ic in self.instances], np.int64)

    @property
    def gamma(self) -> np.ndarray:
        return np.array([ic.gamma for ic in self.instances])

    @property
    def boundary(self) -> list:
        return [ic.boundary for ic in self.instances]

    def concat(self, field: str) -> np.ndarray:
        parts = [getattr(ic, field) if getattr(ic, field) is not None else np.zeros(ic.n) for ic in self.instances]
        return np.ascontiguousarray(np.concatenate(parts))

    @property
    def n(self) -> int:
        return int(self.counts.sum())


def batch_params(n_inst: int = 256, seed: int = 5, n_min: int = 1000, n_max: int = 200_000) -> list:
    """Per-instance parameters of the batched configuration, from the seed's own stream:
    point count log-uniform in [n_min, n_max], kind (Sod tube with a random split angle
    and reflective walls / Sedov blast with E in [0.1, 10] / Kelvin-Helmholtz shear with
    density ratio in [1, 10], periodic), gamma 1.4 or 5/3, instance seed."""
    key = stream_key(seed, 0)
    out = []
    lo_n, hi_n = log_d(float(n_min)), log_d(float(n_max))
    lo_e, hi_e = log_d(0.1), log_d(10.0)
    for b in range(n_inst):
        u = unif(key, 8 * b + np.arange(8))
        n = int(np.rint(exp_d(lo_n + (hi_n - lo_n) * u[0])))
        kind = ("sod", "sedov", "kh")[min(int(u[1] * 3.0), 2)]
        gamma = 1.4 if u[2] < 0.5 else 5.0 / 3.0
        s = int(words(key, 8 * b + 3) >> _U(33))
        p = dict(kind=kind, n=n, gamma=gamma, seed=s)
        if kind == "sod":
            p["split_angle"] = float(u[4] * PI)
        elif kind == "sedov":
            p["e_blast"] = float(exp_d(lo_e + (hi_e - lo_e) * u[5]))
        else:
            p["rho_ratio"] = float(1.0 + 9.0 * u[6])
        out.append(p)
    return out


def batch_2d(n_inst: int = 256, seed: int = 5, n_min: int = 1000, n_max: int = 200_000) -> Batch:
    """Batched configuration: n_inst 2D instances (batch_params); the ghost layer is at least
    four mean spacings wide (0.04 is too thin for the smallest ones)."""
    insts, buffs = [], []
    for p in batch_params(n_inst, seed, n_min, n_max):
        side = max(int(round(math.sqrt(p["n"]))), 8)
        if p["kind"] == "sod":
            ic = sod_2d(n_side=side, seed=p["seed"], gamma=p["gamma"], split_angle=p["split_angle"])
        elif p["kind"] == "sedov":
            ic = sedov_2d(p["n"], p["seed"], gamma=p["gamma"], e_blast=p["e_blast"])
        else:
            ic = kh_2d(n_side=side, seed=p["seed"], gamma=p["gamma"], rho_ratio=p["rho_ratio"])
        insts.append(ic)
        buffs.append(max(0.04, 4.0 / math.sqrt(ic.n)))
    return Batch(insts, np.array(buffs))
