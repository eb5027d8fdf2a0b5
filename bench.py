#!/usr/bin/env python
"""Benchmark of the per-timestep mesh-and-flux path (one JSON line on stdout).

A step is one full moving-mesh step of the clustered 3D Sedov-Taylor workload
(16,777,216 points, 70 % of them in 64 Gaussian clumps): ghost layer, two-level
Morton grid sort, KNN, clipping with the security-radius certificate,
extraction, CFL time step, HLL flux + conserved update + drift.  The metric is hydro cell-updates per second (one
hydro cell advanced one full step) of the learned-K + FP32-clipping form, with
the plain fixed-K (190) FP64 form timed beside it on the same states.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 runs under torchrun: every rank advances its own replica of the workload
(weak scaling, no data-path collective); the timed region is bracketed by a
barrier + synchronize on every rank and the maximum over ranks is reported.
``--impl reference`` times the reference's own CPU implementation (compiled
from its sources into oracle/_ref) on the host cores instead.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Voronoi cell-updates/s per B200: learned-K+FP32 vs plain GPU, at matched L1 err"
UNIT = "cell-updates/s"

# Workloads.  clustered3d_16m is the configuration the metric is quoted on (3D
# clustered Sedov, 16,777,216 points: 70 % in 64 Gaussian clumps, seed 4); the
# others are the uniform 3D Sedov (1M points) and smaller profiling/smoke cases.
CONFIGS = {
    "clustered3d_16m": dict(dim=3, n=16_777_216, seed=4, k=190, buff=0.04, boundary="periodic", cfl=0.3,
                            ic="clustered"),
    "clustered3d_1m": dict(dim=3, n=1_048_576, seed=4, k=190, buff=0.04 * 16 ** (1 / 3), boundary="periodic",
                           cfl=0.3, ic="clustered"),
    "sedov3d_1m": dict(dim=3, n=1_048_576, seed=2, k=190, buff=0.04, boundary="periodic", cfl=0.3),
    "sedov3d_256k": dict(dim=3, n=262_144, seed=2, k=190, buff=0.04 * 4 ** (1 / 3), boundary="periodic", cfl=0.3),
    "sod2d_10k": dict(dim=2, n=10_000, seed=1, k=16, buff=0.04, boundary="reflective", cfl=0.3),
    # 2D Kelvin-Helmholtz shear on a jittered 2048^2 periodic lattice (learned-K configuration)
    "kh2d_4m": dict(dim=2, n=4_194_304, seed=3, k=48, buff=0.04, boundary="periodic", cfl=0.3, ic="kh"),
    # 256 independent 2D simulations (Sod with walls / Sedov / Kelvin-Helmholtz, gamma 1.4 or 5/3),
    # point counts log-uniform in [1e3, 2e5], advanced together
    "batched2d_256": dict(dim=2, n=None, seed=5, k=32, buff=None, boundary="mixed", cfl=0.3, batch=True,
                          n_inst=256),
}

# Algorithmic work per unit, counted with the oracle's
# instrumented restatement of the reference's search and clipping on the workloads'
# distributions: 3D clustered (100,000 cells of the 1,048,576-point clustered set, K=190
# lists), 3D uniform (K=190), 2D jittered lattice (K=16).
#   KNN: candidates per query x flops per squared distance (3D: 8, 2D: 5); the bench
#        uses the candidates the run itself evaluated (the learned budgets' own search)
#   clip: predicates per cell x 45 (det4x4) + vertices created per cell x 59   (3D)
#         predicates per cell x 14 (det3x3) + vertices created per cell x 11   (2D)
#   hydro (flux+update+drift): compulsory HBM bytes per cell-update
WORK = {
    (3, "clustered"): dict(knn_flop_per_cand=8, clip_flop_per_cell=1118.5 * 45 + 71.0 * 59, hydro_bytes_per_cell=683),
    (3, "uniform"): dict(knn_flop_per_cand=8, clip_flop_per_cell=924.7 * 45 + 70.8 * 59, hydro_bytes_per_cell=683),
    (2, "uniform"): dict(knn_flop_per_cand=5, clip_flop_per_cell=34.3 * 14 + 12.0 * 11, hydro_bytes_per_cell=272),
}
STAGES = ["ghosts", "sort", "knn", "clip", "hydro"]


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--config", choices=sorted(CONFIGS), default="clustered3d_16m")
    ap.add_argument("--skip-cpu", action="store_true", help="omit the cpu_baseline leg")
    ap.add_argument("--skip-e2e", action="store_true", help="omit the end-to-end leg")
    ap.add_argument("--skip-forms", action="store_true",
                    help="time only the headline form and the plain baseline (not fp32_clip, learned_fp64)")
    ap.add_argument("--headline-only", action="store_true",
                    help="time only the headline form (profiling runs; no speed-up against the plain form)")
    ap.add_argument("--skip-extras", action="store_true",
                    help="omit the other configurations' short measurements (default run only)")
    ap.add_argument("--skip-oracle", action="store_true",
                    help="omit the oracle checks (sampled cells at full size, density error of a full oracle run)")
    return ap.parse_args()


class Workload:
    """A workload's initial condition as the device generates it: its generator spec
    (pgpu_ic_spec) and sizes, without host arrays."""

    def __init__(self, spec, n, dim, gamma):
        self.spec, self.n, self.dim, self.gamma = spec, n, dim, gamma


def make_workload(cfg):
    """The initial condition of a configuration for the GPU arm: a Workload (generated on
    the device), or the host-generated Batch of a batched configuration."""
    from proteusgpu_b200 import ics
    if cfg.get("batch"):
        return make_ic(cfg)
    if cfg.get("ic") == "clustered":
        spec = ics.clustered_3d_spec(n=cfg["n"], seed=cfg["seed"])
    elif cfg.get("ic") == "kh":
        spec = ics.kh_2d_spec(n_side=int(round(cfg["n"] ** 0.5)), seed=cfg["seed"])
    elif cfg["dim"] == 3:
        spec = ics.sedov_spec(3, cfg["n"], cfg["seed"])
    else:
        spec = ics.sod_2d_spec(n_side=int(round(cfg["n"] ** 0.5)), seed=cfg["seed"])
    n = spec["n_side"] ** spec["dim"] if "n_side" in spec else spec["n"]
    return Workload(spec, n, spec["dim"], spec["gamma"])


def make_ic(cfg):
    from proteusgpu_b200 import ics
    if cfg.get("batch"):
        return ics.batch_2d(cfg["n_inst"], cfg["seed"])
    if cfg.get("ic") == "clustered":
        return ics.clustered_3d(n=cfg["n"], seed=cfg["seed"])
    if cfg.get("ic") == "kh":
        return ics.kh_2d(n_side=int(round(cfg["n"] ** 0.5)), seed=cfg["seed"])
    if cfg["dim"] == 3:
        return ics.sedov_3d(n=cfg["n"], seed=cfg["seed"])
    return ics.sod_2d(n_side=int(round(cfg["n"] ** 0.5)), seed=cfg["seed"])


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


# ---------------------------------------------------------------- clocks
class ClockSampler:
    """Samples SM clocks and throttle reasons with nvidia-smi during the timed region."""
    Q = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id: str | None, enabled: bool = True):
        self.gpu_id, self.proc, self.lines, self.enabled = gpu_id, None, [], enabled

    def __enter__(self):
        if not self.enabled:
            return self
        cmd = ["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits", "-lms", "200"]
        if self.gpu_id:
            cmd += ["-i", self.gpu_id]
        try:
            self.proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 6:
                continue
            try:
                sm.append(float(f[0]))
                mx = float(f[1])
            except ValueError:
                continue
            for nm, v in zip(names, f[2:6]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------- CPU reference
# The reference cannot run the 16.8M-point workload itself: knn::init sizes its neighbour
# lists as len_pts * _K_ * sizeof(int) with int operands (src/knn/knn.cpp:110), which
# overflows beyond 2^31 / 190 = 11.3M extended points (20.9M here), so the allocation fails
# and the run faults.  Its CPU baseline is therefore a bounded sample of the same distribution.
REFERENCE_FULL_SIZE_LIMIT = ("the reference cannot run this workload at full size: src/knn/knn.cpp:110 "
                             "computes len_pts * _K_ in int (20.9M extended points x 190 > 2^31), the "
                             "neighbour-list allocation fails and the process faults")
CPU_SAMPLE_POINTS = 65536


def cpu_reference_step_rate(steps: int, cfg: dict, n_sample: int = CPU_SAMPLE_POINTS, nthreads: int | None = None):
    """Cell-updates/s of the reference's own CPU code (oracle/_ref, compiled from its sources) on a
    bounded sample of the workload: per step and simulation compute_periodic_mesh (KNN + clipping +
    extraction) + dt_CFL + hydro_step.  3D: n_sample points of the same distribution, the ghost layer
    widened so that it spans the same number of mean cells as the workload's buff does at its full
    size (at most 0.15).  Batches: the first instances of the batch up to n_sample points in all, each
    with its own buff and gamma (the reference knows periodic boxes only, so walled instances run
    periodic).  Falls back to the C restatement (oracle/liboracle.so) if _ref is absent."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from proteusgpu_b200 import ics
    nthreads = nthreads or os.cpu_count() or 1
    dim, K = cfg["dim"], cfg["k"]
    if cfg.get("batch"):
        B = ics.batch_2d(cfg["n_inst"], cfg["seed"])
        items, tot = [], 0
        for ic, bf in zip(B.instances, B.buff):
            if tot >= n_sample:
                break
            items.append((ic, float(bf)))
            tot += ic.n
        desc = f"first {len(items)} instances of the batch ({tot} 2D points, periodic), K={K}"
    elif dim == 2:
        # the 2D workloads at n_sample points or fewer (the reference box is periodic only)
        ns = min(cfg["n"], n_sample)
        sub = dict(cfg, n=ns)
        ic = make_ic(sub)
        buff = min(cfg["buff"] * (cfg["n"] / ns) ** (1 / 2), 0.15)
        items, tot = [(ic, buff)], ic.n
        desc = (f"{ic.name}, {ic.n} points{' (the whole workload)' if ns == cfg['n'] else ''}, periodic, "
                f"K={K}, buff {buff:.3f}")
    else:
        clustered = cfg.get("ic") == "clustered"
        ic = ics.clustered_3d(n=n_sample, seed=cfg["seed"]) if clustered else ics.sedov_3d(n=n_sample, seed=2)
        buff = min(cfg["buff"] * (cfg["n"] / n_sample) ** (1 / 3), 0.15)
        items, tot = [(ic, buff)], n_sample
        same = "same clumps, fewer points" if clustered else "uniform in the box, fewer points"
        desc = (f"3D Sedov, {n_sample} {'clustered' if clustered else 'uniform'} points (the workload's "
                f"distribution: {same}), K={K}, buff {buff:.3f}")
    kind = "reference"
    try:
        import refbuild as rb
        rb.load(dim, K)
    except (FileNotFoundError, OSError):
        kind = "port"
    state = [(ic.pos.copy(), ic.rho.copy(), ic.vel.copy(), ic.energy.copy()) for ic, _ in items]
    times = []
    for s in range(steps):
        t0 = time.perf_counter()
        for j, (ic, buff) in enumerate(items):
            x, rho, vel, E = state[j]
            n = ic.n
            if kind == "reference":
                m = rb.periodic_mesh(x, K, buff=buff, gamma=ic.gamma, keep_handle=True, nthreads=nthreads)
                if s == 0 and ic.deposit is not None:
                    E = E + ic.deposit / np.where(m.volumes[:n] > 0, m.volumes[:n], 1.0)
                dt = rb.dt_cfl(dim, K, m.handle, 0.3, rho, vel, E, ic.gamma)
                rho, vel, E = rb.hydro_step(dim, K, m.handle, dt, rho, vel, E, ic.gamma)
                rb.free_handle(dim, K, m.handle)
            else:
                import oracle as om
                m = om.build_mesh(x, K, buff=buff)
                if s == 0 and ic.deposit is not None:
                    E = E + ic.deposit / np.where(m.volumes[:n] > 0, m.volumes[:n], 1.0)
                dt = om.dt_cfl(m, 0.3, ic.gamma, rho, vel, E)
                rho, vel, E, _ = om.hydro_step_ref(m, dt, ic.gamma, rho, vel, E)
            state[j] = (x, rho, vel, E)
        times.append(time.perf_counter() - t0)
    t = float(np.mean(times))
    sample = f"{desc}, {steps} step(s) of compute_periodic_mesh + dt_CFL + hydro_step"
    return tot / t, kind, nthreads, sample, t


# ---------------------------------------------------------------- our arm
# Forms of the step.  The headline is the learned neighbour budget with FP32
# local-frame clipping; the plain FP64 fixed-K method is the baseline it is
# compared with (same mesh bit for bit, same states at every step).
FORMS = {
    "plain_fp64": dict(precision="fp64", kbudget=False),
    "fp32_clip": dict(precision="fp32", kbudget=False),
    "learned_fp64": dict(precision="fp64", kbudget=True),
    "learned_fp32": dict(precision="fp32", kbudget=True),
}
HEADLINE, PLAIN_FORM = "learned_fp32", "plain_fp64"

# DRAM bytes per cell of one k_clip32 launch (read + write / cells), from an ncu capture
# of the clustered 1,048,576-cell case on learned-K lists, used for `traffic`.
CLIP32_DRAM_BYTES_PER_CELL = (669.431296e6 + 774.266112e6) / 1_048_576
# and of one k_flux_update launch on the same case (the hydro stage's dominant kernel)
FLUX_DRAM_BYTES_PER_CELL = (1545.615360e6 + 212.092160e6) / 1_048_576
# and of one k_knn launch on the same case (learned budgets), per query
KNN_DRAM_BYTES_PER_QUERY = (71.634944e6 + 243.834368e6) / 1_048_576


def _barrier(dist):
    if dist:
        dist.barrier()


def compare_states(ref, got):
    """Cells whose state (position, mass, momentum, energy) differs from the reference
    form's after the same steps from the same initial condition, and each field's
    relative L1 difference.  Identical states after a run mean every step's mesh was
    identical too: any face or area difference changes the fluxes."""
    names = ("position", "mass", "momentum", "energy")
    n = len(ref[1])
    differ = np.zeros(n, bool)
    l1 = {}
    for nm, a, b in zip(names, ref, got):
        a = np.asarray(a, np.float64).reshape(n, -1)
        b = np.asarray(b, np.float64).reshape(n, -1)
        neq = (a != b) & ~(np.isnan(a) & np.isnan(b))
        differ |= neq.any(axis=1)
        den = float(np.nansum(np.abs(a)))
        l1[nm] = float(np.nansum(np.abs(a - b))) / den if den > 0 else 0.0
    return {"cells_differing": int(differ.sum()), "l1_rel": l1}


def _max_over_ranks(dist, ms):
    if not dist:
        return ms
    import torch
    t = torch.tensor([ms], device="cuda" if dist.get_backend() == "nccl" else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def _oracle_check_module():
    """oracle/check.py: the checker of the full-size meshes (used after the timed region only)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import check
    return check


def time_form(args, cfg, ic, local_rank, dist, form, want_e2e=False, want_clocks=False, want_state=False,
              want_check=False):
    """Runs one form from the initial condition: W warm-up steps (the learned forms
    train their proposal on them), one step with per-stage CUDA events, then K timed
    steps bracketed by a barrier and synchronize (max over ranks).  want_check: the
    oracle checks the first mesh and, after the timed steps, the mesh of one more step
    on samples of their cells (nothing of it is timed)."""
    import torch
    from proteusgpu_b200 import Context, _lib
    L = _lib.load()
    spec = FORMS[form]
    batch = bool(cfg.get("batch"))
    ctx = Context(dim=cfg["dim"], k=cfg["k"], buff=0.04 if batch else cfg["buff"],
                  boundary="periodic" if batch else cfg["boundary"], flux="physical",
                  gamma=1.4 if batch else ic.gamma, device=local_rank, precision=spec["precision"],
                  predicates="robust" if batch else "reference")
    if spec["kbudget"]:
        # the warm-up steps but the last train the proposal; the last one already uses it.  The
        # class is the smallest whose predicted probability mass reaches the quantile: 0.9 in 3D
        # (16.8M clustered points: mean K 59, 0.30 % misses, 410 ms a step; 0.98: mean K 66,
        # 0.28 %, 418 ms), 0.98 in 2D
        q = 0.9 if cfg["dim"] == 3 else 0.98
        ctx.kbudget_enable(train_steps=max(1, args.warmup - 1), iters_per_step=256, quantile=q, seed=1)
    # the initial condition is generated on the device (pgpu_sim_init_ic / pgpu_batch_init_ic):
    # the same arrays, bit for bit, as proteusgpu_b200/ics.py builds on the host
    if batch:
        ctx.batch_init_ic([b.spec for b in ic.instances], ic.buff, ic.boundary)
    else:
        ctx.sim_init_ic(ic.spec)
    checks = {}
    if want_check:
        t0 = time.perf_counter()
        pos0 = ctx.sim_get()[0]  # the initial positions, which the first mesh was built from
        checks["first_mesh"] = _oracle_check_module().sampled_cells(
            ctx, n_random=20000, n_walked=2000, pos_before=pos0, buff=cfg["buff"], boundary=cfg["boundary"],
            seed=11)
        checks["first_mesh"]["seconds"] = time.perf_counter() - t0
    for _ in range(max(args.warmup, 0)):
        ctx.sim_step(cfg["cfl"], want_dt=False)
    # launch shapes for this workload, timed on mesh builds of the current state (nothing advances)
    tuning = ctx.autotune()
    ctx.enable_timing(True)
    ctx.sim_step(cfg["cfl"], want_dt=False)
    stage = ctx.stage_times()
    ctx.enable_timing(False)
    stats = ctx.stats()
    kb = ctx.kbudget_stats() if spec["kbudget"] else None
    stream = torch.cuda.ExternalStream(ctx.stream)
    torch.cuda.synchronize()
    _barrier(dist)
    uuid = None
    try:
        uuid = "GPU-" + str(torch.cuda.get_device_properties(local_rank).uuid)
    except Exception:
        pass
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    l0 = L.pgpu_launch_count()
    with ClockSampler(uuid, enabled=want_clocks) as clk:
        ev0.record(stream)
        for _ in range(args.steps):
            ctx.sim_step(cfg["cfl"], want_dt=False)
        ev1.record(stream)
        torch.cuda.synchronize()
    ms = _max_over_ranks(dist, ev0.elapsed_time(ev1))
    launches = L.pgpu_launch_count() - l0
    kb_after = ctx.kbudget_stats() if spec["kbudget"] else None
    out = {"ms": ms, "stage": stage, "stats": stats, "launches": launches, "clocks": clk.summary(),
           "kbudget": kb_after or kb, "tuning": tuning}
    if want_state:  # the state after the timed steps, for the comparison between forms
        out["state"] = ctx.sim_get()
    if want_e2e:
        # end to end: the same step through the C ABI with the state in pinned host
        # memory, copied to the device before and back after every step
        x, m_, p_, e_ = ctx.sim_get()
        hp = [torch.from_numpy(a).pin_memory() for a in (x, m_, p_, e_)]
        hn = [t.numpy() for t in hp]
        ke = max(1, min(args.steps, 5))
        ctx.sim_step_host(cfg["cfl"], 0.0, *hn)  # warm the path
        torch.cuda.synchronize()
        _barrier(dist)
        t0 = time.perf_counter()
        for _ in range(ke):
            ctx.sim_step_host(cfg["cfl"], 0.0, *hn)
        torch.cuda.synchronize()
        e_ms = _max_over_ranks(dist, (time.perf_counter() - t0) * 1e3)
        nbytes = int(sum(a.nbytes for a in hn))
        out["e2e"] = {"ms": e_ms, "steps": ke, "bytes": nbytes}
    if want_check:
        # one more step, its mesh checked against the oracle from the positions it started at
        t0 = time.perf_counter()
        x_before = ctx.sim_get()[0]
        ctx.sim_step(cfg["cfl"], want_dt=False)
        checks["after_timed_steps"] = _oracle_check_module().sampled_cells(
            ctx, n_random=20000, n_walked=2000, pos_before=x_before, buff=cfg["buff"], boundary=cfg["boundary"],
            seed=12)
        checks["after_timed_steps"]["seconds"] = time.perf_counter() - t0
        out["checks"] = checks
    if spec["kbudget"]:
        out["weights"] = ctx.kbudget_weights()
    ctx.close()
    return out


def density_check(cfg, form, weights, steps=3, n_max=1_048_576):
    """The density error of a whole run against the oracle's: the workload's distribution
    at min(n, n_max) points (ghost layer spanning the same number of mean cells), `steps`
    moving-mesh steps of the given form (learned forms use the proposal trained on the full
    workload) and of the plain FP64 form on the GPU, and the oracle's own run."""
    from proteusgpu_b200 import Context
    check = _oracle_check_module()
    n = min(cfg["n"], n_max)
    sub = dict(cfg, n=n, buff=min(cfg["buff"] * (cfg["n"] / n) ** (1 / cfg["dim"]), 0.15))
    ic = make_ic(sub)
    t0 = time.perf_counter()

    def gpu(spec, w):
        with Context(dim=sub["dim"], k=sub["k"], buff=sub["buff"], boundary=sub["boundary"], flux="physical",
                     gamma=ic.gamma, precision=spec["precision"]) as ctx:
            if spec["kbudget"] and w is not None:
                ctx.kbudget_enable(train_steps=0, iters_per_step=1, quantile=0.98, seed=1)
                ctx.kbudget_weights(set_to=w)
            ctx.sim_init(ic.pos, ic.rho, ic.vel, ic.energy, ic.deposit)
            dts = [ctx.sim_step(sub["cfl"]) for _ in range(steps)]
            vol = ctx.download_volumes()[: ic.n]
            x, m, p, e = ctx.sim_get()
            kb = ctx.kbudget_stats() if spec["kbudget"] else None
        return (dts, x, m, p, e, vol), kb

    head, kb = gpu(FORMS[form], weights)
    plain, _ = gpu(FORMS[PLAIN_FORM], None)
    t_gpu = time.perf_counter() - t0
    ora = check.oracle_moving_run(ic, sub["k"], sub["buff"], sub["boundary"], steps, cfl=sub["cfl"])
    out = {"workload": f"{sub.get('ic', 'uniform')} 3D Sedov, {n} points (seed {sub['seed']}), buff "
                       f"{sub['buff']:.4f}, {steps} moving-mesh steps from the initial condition",
           "oracle": "om_build_mesh (hydro cells, K then growing budgets) + om_step_moving, FP64",
           form: check.state_errors(head, ora), PLAIN_FORM: check.state_errors(plain, ora),
           "seconds_gpu": t_gpu, "seconds_oracle": time.perf_counter() - t0 - t_gpu}
    if kb:
        out[form]["learned_k"] = {"mean_k": kb["mean_k"], "misses": kb["misses"], "cells": kb["cells"]}
    return out


def run_ours(args, rank, world, local_rank):
    import ctypes
    import torch
    from proteusgpu_b200 import _lib
    cfg = CONFIGS[args.config]
    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local_rank))
    ic = make_workload(cfg)
    n = ic.n
    names = [HEADLINE] if args.headline_only else [PLAIN_FORM, HEADLINE] if args.skip_forms else list(FORMS)
    res = {}
    ref_state = None  # the plain form runs first; every other form is compared with it
    want_check = not args.skip_oracle and world == 1 and not cfg.get("batch") and cfg["dim"] == 3
    for f in names:
        res[f] = time_form(args, cfg, ic, local_rank, dist, f, want_e2e=(f == HEADLINE and not args.skip_e2e),
                           want_clocks=(f == HEADLINE), want_state=PLAIN_FORM in names,
                           want_check=want_check and f == HEADLINE)
        st = res[f].pop("state", None)
        if f == PLAIN_FORM:
            ref_state = st
        elif ref_state is not None and st is not None:
            res[f]["vs_plain"] = compare_states(ref_state, st)
        del st
    oracle_check = None
    if want_check:
        oracle_check = dict(res[HEADLINE].pop("checks"))
        oracle_check["form"] = HEADLINE
        oracle_check["density_run"] = density_check(cfg, HEADLINE, res[HEADLINE].get("weights"))
    extras = None
    if world == 1 and not args.skip_extras and args.config == "clustered3d_16m":
        extras = run_extras(args, local_rank)
    _barrier(dist)
    if dist:
        dist.destroy_process_group()
    if rank != 0:
        return None

    def rate(r):
        return n * args.steps * world / (r["ms"] / 1e3)

    head, base = res[HEADLINE], res.get(PLAIN_FORM)
    value = rate(head)
    forms = {}
    for f, r in res.items():
        forms[f] = {"value": rate(r), "ms_per_step": r["ms"] / args.steps,
                    "stages_ms": dict(zip(STAGES, r["stage"])), "reclip_cells": r["stats"]["reclip_cells"],
                    "clip_split_ms": dict(zip(("main_clip", "fallback", "grid_walk"),
                                              r["stats"]["clip_split_ms"])),
                    "walked_cells": r["stats"]["pruned_cells"],
                    "knn_exact_redone": r["stats"]["knn_redone"],
                    "speedup_vs_plain": rate(r) / rate(base) if base else None,
                    "tuning": {k: r["tuning"][k] for k in ("ppb", "knn_warps", "clip_warps", "clip_thread", "knn_thread",
                                                           "ms_default", "ms_tuned")}}
        if "vs_plain" in r:
            forms[f]["vs_plain"] = r["vs_plain"]
        if r["kbudget"]:
            kb = r["kbudget"]
            forms[f]["learned_k"] = {"mean_k": kb["mean_k"], "plain_k": cfg["k"], "cells": kb["cells"],
                                     "misses": kb["misses"], "miss_rate": kb["misses"] / max(kb["cells"], 1),
                                     "train_steps": kb["steps_trained"], "last_train_loss": kb["last_loss"]}
    e2e = None
    if "e2e" in head:
        e = head["e2e"]
        e2e = {"value": n * e["steps"] * world / (e["ms"] / 1e3), "unit": UNIT, "h2d_bytes_per_step": e["bytes"],
               "d2h_bytes_per_step": e["bytes"], "steps": e["steps"],
               "path": f"pgpu_sim_step_host (C ABI), form {HEADLINE}, pinned host state in/out every step"}

    # roofline of the headline's dominant stage
    D = cfg["dim"]
    W = WORK[(D, "clustered" if cfg.get("ic") == "clustered" else "uniform")]
    stage, stats = head["stage"], head["stats"]
    dom = STAGES[int(np.argmax(stage))]
    fp64, fp32 = ctypes.c_double(), ctypes.c_double()
    L = _lib.load()
    L.pgpu_fp64_peak(local_rank, ctypes.c_float(200.0), ctypes.byref(fp64))
    L.pgpu_fp32_peak(local_rank, ctypes.c_float(200.0), ctypes.byref(fp32))
    hbm, hbm_src = measured_peaks()
    n_query = stats["n_hydro"]
    # the main clip pass (k_clip32 and the FP64 re-clip of its undecided cells), timed by
    # CUDA events on the context's stream; the fallback and the grid walk excluded
    main_ms = stats["clip_split_ms"][0] or stage[3]
    ach = n_query * W["clip_flop_per_cell"] / (main_ms * 1e-3) / 1e12
    roof_clip = {"kernel": "k_clip32 (+ FP64 re-clip of undecided cells)", "bound": "fp32", "achieved": ach,
                 "peak": fp32.value, "unit": "TFLOP/s", "frac": ach / fp32.value,
                 "traffic": CLIP32_DRAM_BYTES_PER_CELL * n_query if D == 3 else None,
                 "traffic_note": "DRAM bytes per launch: ncu capture of the clustered 1,048,576-cell case "
                                 "(learned-K lists) scaled by cells",
                 "timed": "main clip pass (CUDA events): k_clip32 + FP64 re-clip",
                 "peak_source": "FP32 FMA rate measured in this run (pgpu_fp32_peak)",
                 "work": f"{W['clip_flop_per_cell']:.0f} algorithmic flop per cell (the oracle's count on this "
                         f"distribution) x {n_query} cells"}
    cand = stats["knn_candidates"] / max(n_query, 1)
    ach = n_query * cand * W["knn_flop_per_cand"] / (stage[2] * 1e-3) / 1e12
    roof_knn = {"kernel": "k_knn", "bound": "fp64", "achieved": ach, "peak": fp64.value, "unit": "TFLOP/s",
                "frac": ach / fp64.value, "traffic": KNN_DRAM_BYTES_PER_QUERY * n_query if D == 3 else None,
                "traffic_note": "DRAM bytes per launch: ncu capture of the clustered 1,048,576-query case "
                                "(learned budgets) scaled by queries",
                "peak_source": "FP64 FMA rate measured in this run (pgpu_fp64_peak)",
                "work": f"{cand:.1f} candidates per query (this run's) x {W['knn_flop_per_cand']} flop x "
                        f"{n_query} queries"}
    if dom == "clip":
        roof = roof_clip
    elif dom == "knn":
        roof = roof_knn
    else:
        ach = n_query * W["hydro_bytes_per_cell"] / (stage[STAGES.index(dom)] * 1e-3) / 1e9
        roof = {"kernel": dom, "bound": "hbm", "achieved": ach, "peak": hbm, "unit": "GB/s", "frac": ach / hbm,
                "traffic": None, "peak_source": f"MEASURED_PEAKS.json hbm_gbs ({hbm_src})"}
    hyd = n_query * W["hydro_bytes_per_cell"] / (stage[4] * 1e-3) / 1e9
    roof_hydro = {"kernel": "k_prim_dt + k_flux_update", "bound": "hbm", "achieved": hyd, "peak": hbm,
                  "unit": "GB/s", "frac": hyd / hbm,
                  "traffic": FLUX_DRAM_BYTES_PER_CELL * n_query if D == 3 else None,
                  "traffic_note": "k_flux_update DRAM bytes per launch: ncu capture of the clustered 1,048,576-cell "
                                  "case scaled by cells (1,676 B per cell against 683 compulsory)",
                  "work": f"{W['hydro_bytes_per_cell']} compulsory bytes per cell-update"}

    cpu = None
    if not args.skip_cpu and world == 1:
        v, kind, cores, sample, t_step = cpu_reference_step_rate(steps=2, cfg=cfg)
        cpu = {"value": v, "unit": UNIT, "cores": cores, "kind": kind, "sample": sample,
               "s_per_step": t_step}
    if cpu and cfg.get("n") and D == 3 and cfg["n"] > 9_000_000:
        cpu["full_size"] = REFERENCE_FULL_SIZE_LIMIT
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": head["ms"] / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": workload_config(args, cfg, n, world),
        "speedup_vs_plain_gpu": value / rate(base) if base else None,
        # the headline's state after the timed steps against the plain FP64 GPU form's (same IC,
        # same steps): 0 cells differing and 0 L1 error = the same meshes and fluxes every step
        "matched_l1": ({"vs": f"{PLAIN_FORM} (the plain GPU form, not the oracle)", **head["vs_plain"]}
                       if "vs_plain" in head else None),
        # the oracle's checks: sampled cells of the full-size meshes, and the density error of a
        # whole run against the oracle's own run (oracle/check.py; outside the timed region)
        "oracle_check": oracle_check,
        "roofline": roof, "roofline_knn": roof_knn if dom != "knn" else None, "roofline_hydro": roof_hydro,
        "stages_ms": dict(zip(STAGES, stage)),
        "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": head["launches"], "forms": forms,
        "clocks": head["clocks"],
        # the other configurations, one short measurement each with its own oracle check
        "configs": extras,
        "mesh": {"n_ext": stats["n_ext"], "faces": stats["num_faces"], "cert_k_max": stats["cert_k_max"],
                 "failed_cells": stats["failed_cells"], "knn_candidates_per_query":
                     stats["knn_candidates"] / max(stats["n_hydro"], 1)},
        "peaks": {"fp64_tflops": fp64.value, "fp32_tflops": fp32.value, "hbm_gbs": hbm},
    }
    return out


def _form_rate(n, steps, ms):
    return n * steps / (ms / 1e3)


def run_extras(args, local_rank):
    """The other configurations beside the headline workload, each measured briefly with
    the same step (headline form and plain form, CUDA events, inputs resident) and checked
    against the oracle:
      sedov3d_1m     3D Sedov, 1,048,576 uniform points, K = 190: sampled cells of the first
                     mesh and of a mesh after the timed steps
      kh2d_4m        2D Kelvin-Helmholtz, 4,194,304 points: the learned budget trained on the
                     first 50 steps (classes 12-48), then timed; sampled cells
      sod2d_10k      2D Sod with walls, 10,000 points: the whole run to t = 0.2 on the GPU,
                     the oracle's run of the same steps, and the reference's CPU run of it
      batched2d_256  256 2D simulations in one launch per stage: instances against the
                     oracle's solo runs of them
    Each entry also carries the reference CPU rate of its sample (cpu_reference_step_rate)."""
    import types
    check = _oracle_check_module()
    out = {}
    for name in ("sedov3d_1m", "kh2d_4m", "sod2d_10k", "batched2d_256"):
        t0 = time.perf_counter()
        cfg = CONFIGS[name]
        try:
            ic = make_ic(cfg) if name in ("sod2d_10k", "batched2d_256") else make_workload(cfg)
            n = ic.n
            e = {"workload": workload_config(args, cfg, n, 1, name)["workload"], "n_points": n, "k": cfg["k"]}
            if name == "sod2d_10k":
                e.update(_sod_full_run(cfg, ic, local_rank, check))
            else:
                ke = min(max(args.steps, 1), 10)
                res = {}
                for f in (PLAIN_FORM, HEADLINE):
                    # the learned form trains on the first 50 steps of the Kelvin-Helmholtz run; the
                    # plain form runs the same steps, so that both time (and compare) the same states
                    w = 51 if name == "kh2d_4m" else 3
                    a = types.SimpleNamespace(steps=ke, warmup=w)
                    res[f] = time_form(a, cfg, ic, local_rank, None, f, want_state=True,
                                       want_check=(cfg["dim"] == 3 or name == "kh2d_4m") and f == HEADLINE)
                    res[f]["steps_run"] = w + 1 + ke
                h, b = res[HEADLINE], res[PLAIN_FORM]
                e.update({"value": _form_rate(n, ke, h["ms"]), "ms_per_step": h["ms"] / ke,
                          "plain_value": _form_rate(n, ke, b["ms"]),
                          "speedup_vs_plain_gpu": b["ms"] / h["ms"], "steps": ke,
                          "warmup": {f: res[f]["steps_run"] - 1 - ke for f in res},
                          "stages_ms": dict(zip(STAGES, h["stage"])), "launches": h["launches"],
                          "vs_plain": compare_states(b["state"], h["state"])})
                # the autotuner's choice for this workload (bin size, block shapes) and its gain
                e["tuning"] = {k: h["tuning"].get(k) for k in ("ppb", "knn_warps", "clip_warps", "clip_thread",
                                                               "knn_thread", "ms_default", "ms_tuned")}
                if h.get("kbudget"):
                    kb = h["kbudget"]
                    e["learned_k"] = {"mean_k": kb["mean_k"], "plain_k": cfg["k"], "misses": kb["misses"],
                                      "miss_rate": kb["misses"] / max(kb["cells"], 1),
                                      "train_steps": kb["steps_trained"]}
                if "checks" in h:
                    e["oracle"] = h["checks"]
                if name == "batched2d_256":
                    e["oracle"] = _batch_instances_vs_oracle(cfg, ic, h, check)
            v, kind, cores, sample, t_step = cpu_reference_step_rate(
                steps=1 if name != "sod2d_10k" else e.get("steps_to_t_end", 1), cfg=cfg)
            e["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": cores, "kind": kind, "sample": sample}
        except Exception as exc:  # one configuration's failure is reported, not fatal
            e = {"error": f"{type(exc).__name__}: {exc}"}
        e["seconds"] = time.perf_counter() - t0
        out[name] = e
    return out


def _sod_full_run(cfg, ic, local_rank, check):
    """2D Sod to t = 0.2: both forms' whole runs timed (CUDA events; a dt read back per step
    to stop at t_end), and the oracle's run of the same number of steps."""
    import torch
    from proteusgpu_b200 import Context
    t_end = 0.2
    runs = {}
    for f in (PLAIN_FORM, HEADLINE):
        spec = FORMS[f]
        with Context(dim=2, k=cfg["k"], buff=cfg["buff"], boundary=cfg["boundary"], flux="physical",
                     gamma=ic.gamma, device=local_rank, precision=spec["precision"], predicates="robust") as ctx:
            if spec["kbudget"]:
                ctx.kbudget_enable(train_steps=5, iters_per_step=64, quantile=0.98, seed=1)
            ctx.sim_init(ic.pos, ic.rho, ic.vel, ic.energy, ic.deposit)
            stream = torch.cuda.ExternalStream(ctx.stream)
            ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            ev0.record(stream)
            t, steps, dts = 0.0, 0, []
            while t < t_end and steps < 10000:
                dts.append(ctx.sim_step(cfg["cfl"]))
                t += dts[-1]
                steps += 1
            ev1.record(stream)
            torch.cuda.synchronize()
            vol = ctx.download_volumes()[: ic.n]
            x, m, p, e = ctx.sim_get()
            runs[f] = {"ms": ev0.elapsed_time(ev1), "steps": steps, "state": (dts, x, m, p, e, vol)}
    steps = runs[HEADLINE]["steps"]
    ora = check.oracle_moving_run(ic, cfg["k"], cfg["buff"], cfg["boundary"], steps, cfl=cfg["cfl"], robust=True)
    h, b = runs[HEADLINE], runs[PLAIN_FORM]
    return {"value": _form_rate(ic.n, steps, h["ms"]), "ms_per_step": h["ms"] / steps,
            "plain_value": _form_rate(ic.n, b["steps"], b["ms"]), "speedup_vs_plain_gpu":
                (b["ms"] / b["steps"]) / (h["ms"] / steps), "steps_to_t_end": steps, "t_end": t_end,
            "timed": "the whole run from the initial condition to t_end (one dt read back per step)",
            "oracle": {HEADLINE: check.state_errors(h["state"], ora),
                       PLAIN_FORM: check.state_errors(b["state"], ora)}}


def _batch_instances_vs_oracle(cfg, B, h, check, n_check=3):
    """The batch's headline-form state after its steps, instance by instance for the
    n_check smallest instances, against the oracle's solo runs of them (each with its
    own ghost layer, gamma and boundary; robust predicates as the batch uses)."""
    x, m, p, e = h["state"]
    counts = B.counts
    off = np.concatenate([[0], np.cumsum(counts)])
    steps = h["steps_run"]
    out = {"steps": steps, "instances": []}
    for i in np.argsort(counts)[:n_check]:
        ic, bf = B.instances[i], float(B.buff[i])
        dts, xo, mo, po, eo, vo = check.oracle_moving_run(ic, cfg["k"], bf, ic.boundary, steps, cfl=cfg["cfl"],
                                                          robust=True)
        sl = slice(off[i], off[i + 1])
        l1 = lambda a, b: float(np.abs(a - b).sum() / max(np.abs(b).sum(), 1e-300))  # noqa: E731
        out["instances"].append({"instance": int(i), "n": int(counts[i]), "ic": ic.name, "boundary": ic.boundary,
                                 "mass_l1_rel": l1(m[sl], mo), "energy_l1_rel": l1(e[sl], eo),
                                 "position_max_abs": float(np.abs(x[sl] - xo).max()),
                                 "momentum_l1_rel": l1(p[sl], po)})
    return out


def workload_config(args, cfg, n, world, name=None):
    """The `config` object of both arms' lines: the workload, its sizes and the forms."""
    name = name or args.config
    dist_name = "clustered (70% in 64 Gaussian clumps)" if cfg.get("ic") == "clustered" else "uniform"
    if cfg.get("batch"):
        wl = (f"{name}: {cfg['n_inst']} independent 2D simulations (Sod with walls / Sedov / "
              f"Kelvin-Helmholtz, gamma 1.4 or 5/3, seed {cfg['seed']}), {n} points in all, point counts "
              "log-uniform in [1e3, 2e5], one launch per stage")
    elif cfg["dim"] == 3:
        wl = (f"{name}: 3D Sedov-Taylor blast, {cfg['n']} {dist_name} points (seed {cfg['seed']}), "
              f"moving mesh, {cfg['boundary']} box")
    elif cfg.get("ic") == "kh":
        wl = (f"{name}: 2D Kelvin-Helmholtz shear, {n} points on a jittered {int(round(n ** 0.5))}^2 lattice "
              f"(seed {cfg['seed']}), moving mesh, periodic box")
    else:
        wl = (f"{name}: 2D Sod shock tube, {n} points on a jittered lattice (seed {cfg['seed']}), moving mesh, "
              f"{cfg['boundary']} walls")
    return {"workload": wl, "n_points": n, "k": cfg["k"], "buff": cfg["buff"],
            "form": "learned-K (BF16 MLP proposal, plain-K fallback) + FP32 local-frame clipping "
                    "(FP64 re-clip, FP64 extraction, hydro and sums)",
            "baseline_form": f"plain: fixed K={cfg['k']}, FP64 clipping",
            "flux": "physical (outward normal, pair-symmetric area)",
            "l2": (f"inputs larger than L2: per-step KNN lists alone are {n * cfg['k'] * 4 / 2 ** 20:.0f} MiB "
                   "at the plain K" if n * cfg["k"] * 4 > 126 * 2 ** 20 else
                   "a small configuration: its working set fits in L2 (no flush between steps)"),
            "parallelism": f"replicas x{world}"}


def run_reference(args, rank):
    if rank != 0:
        return None
    steps, warm = max(args.steps, 1), max(args.warmup, 0)
    v_all = []
    kind = cores = sample = None
    if warm:
        cpu_reference_step_rate(steps=1, cfg=CONFIGS[args.config])
    for _ in range(steps):
        v, kind, cores, sample, _t = cpu_reference_step_rate(steps=1, cfg=CONFIGS[args.config])
        v_all.append(v)
    v = float(np.mean(v_all))
    cfg = CONFIGS[args.config]
    cpu = {"value": v, "unit": UNIT, "cores": cores, "kind": kind, "sample": sample}
    if cfg.get("n") and cfg["dim"] == 3 and cfg["n"] > 9_000_000:
        cpu["full_size"] = REFERENCE_FULL_SIZE_LIMIT
    return {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": steps,
            "warmup": warm, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": workload_config(args, cfg, make_ic(cfg).n if cfg.get("batch") else cfg["n"], args.gpus),
            "cpu_baseline": cpu,
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        out = run_reference(args, rank)
    else:
        out = run_ours(args, rank, world, local_rank)
    if out is not None:
        print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
