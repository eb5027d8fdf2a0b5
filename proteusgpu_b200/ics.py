"""Seeded initial conditions for the mesh-and-flux workloads.

The reference reads its initial conditions from HDF5 files written by
``create.py`` / ``create_sod.py`` (datasets ``seedpos`` N x D, ``rho`` N,
``vel`` N x D, ``Energy`` N; src/io/input.cpp:121-309).  h5py is not available
here, so these generators build the same four fields in memory from fixed seeds.
``Energy`` is the total energy per unit volume, as in the reference's
``primvars::E`` (src/global/allvars.h:203-207).

Each generator returns an :class:`IC` whose arrays are C-contiguous float64.
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

    @property
    def n(self) -> int:
        return int(self.pos.shape[0])


def _finish(ic: IC) -> IC:
    for f in ("pos", "rho", "vel", "energy"):
        setattr(ic, f, np.ascontiguousarray(getattr(ic, f), dtype=np.float64))
    if ic.deposit is not None:
        ic.deposit = np.ascontiguousarray(ic.deposit, dtype=np.float64)
    return ic


def jittered_lattice(n_side: int, dim: int, jitter: float, rng: np.random.Generator) -> np.ndarray:
    """Cell centres of an n_side^dim lattice, each moved by U(-jitter, jitter) x spacing per axis."""
    h = 1.0 / n_side
    axes = [(np.arange(n_side) + 0.5) * h] * dim
    grid = np.stack(np.meshgrid(*axes, indexing="xy"), axis=-1).reshape(-1, dim)
    grid = grid + rng.uniform(-jitter, jitter, size=grid.shape) * h
    return np.clip(grid, 0.0, np.nextafter(1.0, 0.0))


def sod_2d(n_side: int = 100, seed: int = 1, jitter: float = 0.1, gamma: float = 1.4,
           boundary: str = "reflective", split_angle: float = 0.0) -> IC:
    """2D Sod shock tube on a jittered lattice (left rho=1, P=1; right rho=0.125, P=0.1).

    ``split_angle`` rotates the discontinuity about the box centre (0 = split at x=0.5).
    """
    rng = np.random.default_rng(seed)
    pos = jittered_lattice(n_side, 2, jitter, rng)
    c, s = math.cos(split_angle), math.sin(split_angle)
    left = ((pos[:, 0] - 0.5) * c + (pos[:, 1] - 0.5) * s) < 0.0
    rho = np.where(left, 1.0, 0.125)
    P = np.where(left, 1.0, 0.1)
    vel = np.zeros_like(pos)
    energy = P / (gamma - 1.0)
    return _finish(IC("sod2d", 2, pos, rho, vel, energy, gamma, boundary))


def uniform_points(n: int, dim: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return rng.random((n, dim))


def sedov_deposit(pos: np.ndarray, center, e_total: float, n_dep: int = 32, sigma: float = 0.01) -> np.ndarray:
    """Energy per cell for a blast of ``e_total`` over the ``n_dep`` points nearest ``center``,
    weighted by exp(-r^2 / (2 sigma^2)) and normalised.  Ties in distance break by index."""
    d2 = ((pos - np.asarray(center)[None, :]) ** 2).sum(axis=1)
    order = np.lexsort((np.arange(len(d2)), d2))[:n_dep]
    w = np.exp(-d2[order] / (2.0 * sigma * sigma))
    w = w / w.sum()
    dep = np.zeros(len(pos))
    dep[order] = e_total * w
    return dep


def sedov_3d(n: int = 1_048_576, seed: int = 2, gamma: float = 5.0 / 3.0, p0: float = 1e-5,
             e_blast: float = 1.0, points: np.ndarray | None = None) -> IC:
    """3D Sedov-Taylor blast: uniform points, rho=1, P=p0, v=0, E deposited near the centre."""
    pos = uniform_points(n, 3, seed) if points is None else np.asarray(points, dtype=np.float64)
    n = len(pos)
    rho = np.ones(n)
    vel = np.zeros((n, 3))
    energy = np.full(n, p0 / (gamma - 1.0))
    dep = sedov_deposit(pos, (0.5, 0.5, 0.5), e_blast)
    return _finish(IC("sedov3d", 3, pos, rho, vel, energy, gamma, "periodic", dep))


def sedov_2d(n: int, seed: int, gamma: float = 5.0 / 3.0, p0: float = 1e-5, e_blast: float = 1.0) -> IC:
    pos = uniform_points(n, 2, seed)
    rho = np.ones(n)
    vel = np.zeros((n, 2))
    energy = np.full(n, p0 / (gamma - 1.0))
    dep = sedov_deposit(pos, (0.5, 0.5), e_blast)
    return _finish(IC("sedov2d", 2, pos, rho, vel, energy, gamma, "periodic", dep))


def kh_2d(n_side: int = 2048, seed: int = 3, gamma: float = 5.0 / 3.0, rho_ratio: float = 2.0) -> IC:
    """Kelvin-Helmholtz shear layer on a jittered periodic lattice."""
    rng = np.random.default_rng(seed)
    pos = jittered_lattice(n_side, 2, 0.1, rng)
    band = np.abs(pos[:, 1] - 0.5) < 0.25
    rho = np.where(band, rho_ratio, 1.0)
    vel = np.zeros_like(pos)
    vel[:, 0] = np.where(band, 0.5, -0.5)
    vel[:, 1] = 0.01 * np.sin(4.0 * math.pi * pos[:, 0]) + 1e-3 * rng.standard_normal(len(pos))
    P = np.full(len(pos), 2.5)
    energy = P / (gamma - 1.0) + 0.5 * rho * (vel ** 2).sum(axis=1)
    return _finish(IC("kh2d", 2, pos, rho, vel, energy, gamma, "periodic"))


def clustered_3d(n: int = 16_777_216, seed: int = 4, n_clumps: int = 64, frac_clumped: float = 0.7,
                 gamma: float = 5.0 / 3.0, p0: float = 1e-5, e_blast: float = 1.0) -> IC:
    """Clustered 3D Sedov: Gaussian clumps (sigma log-uniform in [0.005, 0.05]) plus a uniform
    background, wrapped periodically into [0,1)^3."""
    rng = np.random.default_rng(seed)
    n_cl = int(round(frac_clumped * n))
    centres = rng.random((n_clumps, 3))
    sig = np.exp(rng.uniform(math.log(0.005), math.log(0.05), size=n_clumps))
    which = rng.integers(0, n_clumps, size=n_cl)
    pts_cl = centres[which] + rng.standard_normal((n_cl, 3)) * sig[which, None]
    pts_bg = rng.random((n - n_cl, 3))
    pos = np.mod(np.concatenate([pts_cl, pts_bg]), 1.0)
    pos = np.where(pos >= 1.0, 0.0, pos)
    return sedov_3d(points=pos, gamma=gamma, p0=p0, e_blast=e_blast)


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


def batch_2d(n_inst: int = 256, seed: int = 5, n_min: int = 1000, n_max: int = 200_000) -> Batch:
    """Batched configuration: n_inst 2D instances, point counts log-uniform in
    [n_min, n_max]; each draws a Sod tube with a random split angle (reflective
    walls), a Sedov blast with E in [0.1, 10] or a Kelvin-Helmholtz shear with
    density ratio in [1, 10] (periodic), gamma 1.4 or 5/3.  The ghost layer is
    at least four mean spacings wide (0.04 is too thin for the smallest ones)."""
    rng = np.random.default_rng(seed)
    insts, buffs = [], []
    for b in range(n_inst):
        n = int(round(math.exp(rng.uniform(math.log(n_min), math.log(n_max)))))
        kind = int(rng.integers(0, 3))
        gamma = 1.4 if rng.random() < 0.5 else 5.0 / 3.0
        s = int(rng.integers(0, 2**31 - 1))
        if kind == 0:
            side = max(int(round(math.sqrt(n))), 8)
            ic = sod_2d(n_side=side, seed=s, gamma=gamma, split_angle=float(rng.uniform(0.0, math.pi)))
        elif kind == 1:
            ic = sedov_2d(n, s, gamma=gamma, e_blast=float(math.exp(rng.uniform(math.log(0.1), math.log(10.0)))))
        else:
            side = max(int(round(math.sqrt(n))), 8)
            ic = kh_2d(n_side=side, seed=s, gamma=gamma, rho_ratio=float(rng.uniform(1.0, 10.0)))
        insts.append(ic)
        buffs.append(max(0.04, 4.0 / math.sqrt(ic.n)))
    return Batch(insts, np.array(buffs))
