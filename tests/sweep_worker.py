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
