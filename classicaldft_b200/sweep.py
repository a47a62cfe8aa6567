"""Sharded state-point sweeps over several GPUs (one process per GPU).

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
