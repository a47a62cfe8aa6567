"""Worker of the two-rank gloo sweep tests (a host solver stands in for the GPU)."""
import os

import numpy as np


def fake_solve(idx):
    """Deterministic per-problem scalars and profiles: problem i -> i-dependent values."""
    sc = np.array([[10.0 * i, -1.0 * i, 1e-3 * i, 7 + i, float(i % 2 == 0)] for i in idx])
    prof = np.stack([np.full(8, 0.1 * i) for i in idx]) if len(idx) else np.zeros((0, 8))
    return sc, prof


def run(rank, world, port, n, batch, gather_profiles, out_dir):
    import torch.distributed as dist

    from classicaldft_b200 import Grid, Model, Species, WhiteBearII
    from classicaldft_b200.sweep import run_sweep, shard
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        model = Model(Grid(0.5, (1.0, 1.0, 2.0), (2, 2, 2)), [Species("A", 1.0)], [], 1.0)
        seen = []

        def solve(idx):
            seen.extend(list(idx))
            assert len(idx) <= batch
            return fake_solve(idx)
        res = run_sweep(model, WhiteBearII(), list(range(n)), [np.zeros(8)] * n, None, batch=batch,
                        gather_profiles=gather_profiles, solve=solve)
        assert seen == list(shard(n, rank, world))
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"), F=res.free_energy, O=res.grand_potential,
                 it=res.iterations, conv=res.converged,
                 prof=res.profiles if res.profiles is not None else np.zeros(0), seen=np.array(seen))
    finally:
        dist.destroy_process_group()


UNEVEN_SHAPES = [(2, 2, 2), (4, 4, 4), (2, 2, 4), (4, 4, 4), (2, 2, 2), (3, 3, 3), (4, 4, 2)]


def fake_uneven_solve(problems):
    def solve(idx):
        sc = np.array([[10.0 * i, -1.0 * i, 1e-3 * i, 7 + i, float(i % 2 == 0)] for i in idx])
        prof = [np.full(problems[i].model.grid.total_points, 0.1 * i) for i in idx]
        return sc, prof
    return solve


def uneven_problems(n):
    from classicaldft_b200 import Grid, Model, Species
    from classicaldft_b200.sweep import SweepProblem
    out = []
    for i in range(n):
        shape = UNEVEN_SHAPES[i % len(UNEVEN_SHAPES)]
        m = Model(Grid(0.5, tuple(0.5 * s for s in shape), shape), [Species("A", 1.0)], [], 1.0)
        out.append(SweepProblem(m, 0.1 * i, np.zeros(int(np.prod(shape)))))
    return out


def run_uneven(rank, world, port, n, out_dir):
    import torch.distributed as dist

    from classicaldft_b200 import WhiteBearII
    from classicaldft_b200.sweep import run_uneven_sweep
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        problems = uneven_problems(n)
        seen = []
        base = fake_uneven_solve(problems)

        def solve(idx):
            seen.extend(list(idx))
            return base(idx)
        res = run_uneven_sweep(problems, WhiteBearII(), None, gather_profiles=True, solve=solve)
        np.savez(os.path.join(out_dir, f"uneven{rank}.npz"), F=res.free_energy, it=res.iterations,
                 conv=res.converged, rank=res.rank, seen=np.array(seen),
                 prof=np.concatenate(res.profiles), lens=np.array([len(p) for p in res.profiles]))
    finally:
        dist.destroy_process_group()
