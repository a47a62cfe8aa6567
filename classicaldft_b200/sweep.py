"""Sharded state-point sweeps over several GPUs (one process per GPU).

Two forms.  ``run_sweep``: a list of problems on ONE grid, split in
contiguous shares of equal count.  ``run_uneven_sweep``: problems on
different grids (an isotherm over 48^3, 64^3 and 96^3 boxes), split by cost
(N log N per problem, longest first onto the least-loaded rank), each
rank's problems grouped by grid into batched engines and minimised together
by one group minimisation (one graph launch per FIRE step for all of them).

A sweep is a list of independent problems on one grid (a chemical-potential
scan along a branch, several nucleation state points).  The problems
partition across the ranks of a torch.distributed process group: each rank
minimises its contiguous share in batches (one batched engine per chunk, so
small grids fill the GPU), and a single all-gather at the end collects every
problem's scalars (and, if asked, its profile) on every rank, in global
order.  Nothing is exchanged while the problems iterate; the grid itself is
never split (every one of the ~25 transforms of an evaluation is global).

Used like the reference's per-state-point loop:

    res = run_sweep(model, WhiteBearII(), mus, rho0s, Minimizer(...), batch=16)
    res.grand_potential[i], res.converged[i], res.profiles[i]
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Callable, Optional

import numpy as np

from . import _lib
from .functionals import FMTModel, Model, make_weights

# scalar columns gathered per problem
COLUMNS = ("free_energy", "grand_potential", "rms_force", "iterations", "converged")


def shard(n_items: int, rank: int, world: int) -> range:
    """Contiguous share of rank `rank` among `world` (sizes differ by at most one)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("shard: need 0 <= rank < world")
    base, extra = divmod(n_items, world)
    start = rank * base + min(rank, extra)
    return range(start, start + base + (1 if rank < extra else 0))


def chunks(indices: range, batch: int):
    """Consecutive pieces of at most `batch` indices."""
    if batch < 1:
        raise ValueError("chunks: batch must be >= 1")
    for s in range(0, len(indices), batch):
        yield indices[s:s + batch]


@dataclass
class SweepResult:
    free_energy: np.ndarray
    grand_potential: np.ndarray
    rms_force: np.ndarray
    iterations: np.ndarray
    converged: np.ndarray
    profiles: Optional[np.ndarray] = None   # (n, N) when gathered


def _gpu_solver(model: Model, fmt_model: FMTModel, minimizer, precision, mus, rho0s, mode, masses):
    """The solve step on this rank's GPU: batched FIRE2 per chunk."""
    cache = {}

    def solve(idx):
        B = len(idx)
        if B not in cache:
            cache[B] = make_weights(fmt_model, model, precision, batch=B)
        w = cache[B]
        rho = np.stack([np.asarray(rho0s[i], dtype=np.float64).reshape(-1) for i in idx])
        mu = np.asarray([mus[i] for i in idx], dtype=np.float64)
        if mode == "fixed_mass":
            res = minimizer.fixed_mass_batch(model, w, rho, mu, np.asarray([masses[i] for i in idx]))
        else:
            res = minimizer.grand_potential_batch(model, w, rho, mu)
        sc = np.array([[r.free_energy, r.grand_potential, r.rms_force, r.iterations, float(r.converged)]
                       for r in res])
        prof = np.stack([np.asarray(r.densities[0]).reshape(-1) for r in res])
        return sc, prof

    return solve


def run_sweep(model: Model, fmt_model: FMTModel, mus, initial_densities, minimizer, batch: int = 16,
              precision: int = _lib.FP64, mode: str = "grand_potential", target_masses=None,
              gather_profiles: bool = False, group=None,
              solve: Optional[Callable] = None, device=None) -> SweepResult:
    """Minimise every problem of the sweep, sharded over the process group.

    ``solve(indices) -> (scalars (k, 5), profiles (k, N))`` replaces the GPU
    solve (tests drive the sharding and the gather with a host solver).
    Without an initialised process group the sweep runs on this process only.
    """
    import torch
    import torch.distributed as dist
    n = len(mus)
    if len(initial_densities) != n:
        raise ValueError("run_sweep: one initial density per chemical potential")
    if mode not in ("grand_potential", "fixed_mass"):
        raise ValueError("run_sweep: mode is grand_potential or fixed_mass")
    if mode == "fixed_mass" and (target_masses is None or len(target_masses) != n):
        raise ValueError("run_sweep: fixed_mass needs one target mass per problem")
    distributed = dist.is_available() and dist.is_initialized()
    rank = dist.get_rank(group) if distributed else 0
    world = dist.get_world_size(group) if distributed else 1
    if solve is None:
        solve = _gpu_solver(model, fmt_model, minimizer, precision, mus, initial_densities, mode, target_masses)
    mine = shard(n, rank, world)
    N = model.grid.total_points
    sc = np.zeros((len(mine), len(COLUMNS)))
    prof = np.zeros((len(mine), N)) if gather_profiles else None
    for piece in chunks(mine, batch):
        s, p = solve(piece)
        lo = piece.start - mine.start
        sc[lo:lo + len(piece)] = s
        if gather_profiles:
            prof[lo:lo + len(piece)] = p
    if not distributed:
        allsc, allprof = sc, prof
    else:
        if device is None:
            device = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend(group) == "nccl" \
                else torch.device("cpu")
        cap = shard(n, 0, world).stop  # the largest share (rank 0's)
        width = len(COLUMNS) + (N if gather_profiles else 0)
        buf = torch.zeros((cap, width), dtype=torch.float64, device=device)
        if len(mine):
            buf[:len(mine), :len(COLUMNS)] = torch.from_numpy(sc)
            if gather_profiles:
                buf[:len(mine), len(COLUMNS):] = torch.from_numpy(prof)
        out = [torch.empty_like(buf) for _ in range(world)]
        dist.all_gather(out, buf, group=group)
        rows = [out[r][:len(shard(n, r, world))].cpu().numpy() for r in range(world)]
        full = np.concatenate(rows, axis=0) if rows else np.zeros((0, width))
        allsc = full[:, :len(COLUMNS)]
        allprof = full[:, len(COLUMNS):] if gather_profiles else None
    return SweepResult(free_energy=allsc[:, 0], grand_potential=allsc[:, 1], rms_force=allsc[:, 2],
                       iterations=allsc[:, 3].astype(int), converged=allsc[:, 4] > 0.5, profiles=allprof)


# ----------------------------------------------------------- uneven sweeps


@dataclass
class SweepProblem:
    """One state point of an uneven sweep: its own model (grid, species,
    interactions, kT), chemical potential, initial density and, for
    fixed-mass runs, target mass."""

    model: Model
    chemical_potential: float
    initial_density: object
    target_mass: float = 0.0


def problem_cost(n_points: int) -> float:
    """Relative cost of one problem: the N log2 N of its transforms."""
    return float(n_points) * max(np.log2(max(n_points, 2)), 1.0)


def partition_by_cost(costs, world: int):
    """Longest-processing-time partition: problems in decreasing cost (ties by
    index) each go to the rank with the least total cost so far (ties to the
    lowest rank).  Deterministic, so every rank computes the same split.
    Returns one sorted index list per rank."""
    if world < 1:
        raise ValueError("partition_by_cost: world must be >= 1")
    load = [0.0] * world
    parts = [[] for _ in range(world)]
    for i in sorted(range(len(costs)), key=lambda k: (-costs[k], k)):
        r = min(range(world), key=lambda q: (load[q], q))
        parts[r].append(i)
        load[r] += costs[i]
    return [sorted(p) for p in parts]


def _model_key(model: Model):
    g = model.grid
    return (tuple(g.shape), float(g.dx), tuple(float(s.hard_sphere_diameter) for s in model.species),
            float(model.temperature), tuple(repr(it) for it in model.interactions))


def _gpu_group_solver(problems, fmt_model: FMTModel, minimizer, precision, mode, max_batch):
    """This rank's problems grouped by model into batched engines, minimised
    by one group minimisation."""

    def solve(idx):
        groups = {}
        for i in idx:
            groups.setdefault(_model_key(problems[i].model), []).append(i)
        members, order = [], []
        for members_idx in groups.values():
            for s in range(0, len(members_idx), max_batch):
                part = members_idx[s:s + max_batch]
                model = problems[part[0]].model
                w = make_weights(fmt_model, model, precision, batch=len(part))
                rho = np.stack([np.asarray(problems[i].initial_density, dtype=np.float64).reshape(-1) for i in part])
                mu = np.asarray([problems[i].chemical_potential for i in part])
                mass = np.asarray([problems[i].target_mass for i in part]) if mode == "fixed_mass" else None
                members.append((w, rho, mu, mass))
                order.append(part)
        res = minimizer.minimize_group(members, mode=mode)
        out_sc, out_prof = {}, {}
        for part, rs in zip(order, res):
            for i, r in zip(part, rs):
                out_sc[i] = [r.free_energy, r.grand_potential, r.rms_force, r.iterations, float(r.converged)]
                out_prof[i] = np.asarray(r.densities[0]).reshape(-1)
        sc = np.array([out_sc[i] for i in idx]).reshape(len(idx), len(COLUMNS))
        return sc, [out_prof[i] for i in idx]

    return solve


@dataclass
class UnevenSweepResult:
    free_energy: np.ndarray
    grand_potential: np.ndarray
    rms_force: np.ndarray
    iterations: np.ndarray
    converged: np.ndarray
    rank: np.ndarray                  # the rank that minimised each problem
    profiles: Optional[list] = None   # one flat array per problem when gathered


def run_uneven_sweep(problems, fmt_model: FMTModel, minimizer, precision: int = _lib.FP64,
                     mode: str = "grand_potential", gather_profiles: bool = False, group=None,
                     solve: Optional[Callable] = None, device=None, max_batch: int = 16) -> UnevenSweepResult:
    """Minimise every problem of an uneven sweep, sharded over the process
    group by cost; one all-gather at the end returns every problem's scalars
    (and profiles) in input order on every rank.

    ``solve(indices) -> (scalars (k, 5), [profile_i])`` replaces the GPU
    solve (tests drive the partition and the gather with a host solver)."""
    import torch
    import torch.distributed as dist
    n = len(problems)
    if mode not in ("grand_potential", "fixed_mass"):
        raise ValueError("run_uneven_sweep: mode is grand_potential or fixed_mass")
    distributed = dist.is_available() and dist.is_initialized()
    rank = dist.get_rank(group) if distributed else 0
    world = dist.get_world_size(group) if distributed else 1
    sizes = [int(p.model.grid.total_points) for p in problems]
    parts = partition_by_cost([problem_cost(s) * len(p.model.species) for s, p in zip(sizes, problems)], world)
    if solve is None:
        solve = _gpu_group_solver(problems, fmt_model, minimizer, precision, mode, max_batch)
    mine = parts[rank]
    sc = np.zeros((len(mine), len(COLUMNS)))
    prof = []
    if mine:
        sc, prof = solve(mine)
        sc = np.asarray(sc, dtype=np.float64).reshape(len(mine), len(COLUMNS))
    owner = np.zeros(n, dtype=int)
    for r, part in enumerate(parts):
        owner[part] = r
    if not distributed:
        allsc = np.zeros((n, len(COLUMNS)))
        allsc[mine] = sc
        allprof = [None] * n
        for i, pr in zip(mine, prof):
            allprof[i] = np.asarray(pr)
    else:
        if device is None:
            device = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend(group) == "nccl" \
                else torch.device("cpu")
        cap = max(len(p) for p in parts)
        nmax = max(sizes) if gather_profiles else 0
        width = len(COLUMNS) + nmax
        buf = torch.zeros((max(cap, 1), width), dtype=torch.float64, device=device)
        for k, i in enumerate(mine):
            buf[k, :len(COLUMNS)] = torch.from_numpy(sc[k])
            if gather_profiles:
                buf[k, len(COLUMNS):len(COLUMNS) + sizes[i]] = torch.from_numpy(np.asarray(prof[k], dtype=np.float64))
        out = [torch.empty_like(buf) for _ in range(world)]
        dist.all_gather(out, buf, group=group)
        allsc = np.zeros((n, len(COLUMNS)))
        allprof = [None] * n
        for r, part in enumerate(parts):
            rows = out[r].cpu().numpy()
            for k, i in enumerate(part):
                allsc[i] = rows[k, :len(COLUMNS)]
                if gather_profiles:
                    allprof[i] = rows[k, len(COLUMNS):len(COLUMNS) + sizes[i]].copy()
    return UnevenSweepResult(free_energy=allsc[:, 0], grand_potential=allsc[:, 1], rms_force=allsc[:, 2],
                             iterations=allsc[:, 3].astype(int), converged=allsc[:, 4] > 0.5, rank=owner,
                             profiles=allprof if gather_profiles else None)
