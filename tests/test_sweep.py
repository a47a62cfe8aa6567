"""Sharded sweeps (classicaldft_b200.sweep): the partition, and the two-rank
gather over gloo on CPU with a host solver standing in for the GPU; on the
GPU, a sweep against single-problem minimisations."""
import socket

import numpy as np
import pytest

from classicaldft_b200.sweep import chunks, partition_by_cost, problem_cost, shard
from tests.sweep_worker import fake_solve, fake_uneven_solve, uneven_problems


def test_shard_is_a_balanced_contiguous_partition():
    for n in range(0, 13):
        for world in range(1, 5):
            parts = [shard(n, r, world) for r in range(world)]
            assert [i for p in parts for i in p] == list(range(n))
            sizes = [len(p) for p in parts]
            assert max(sizes) - min(sizes) <= 1
            assert sizes == sorted(sizes, reverse=True)
    assert [list(c) for c in chunks(range(3, 10), 3)] == [[3, 4, 5], [6, 7, 8], [9]]
    with pytest.raises(ValueError):
        shard(4, 2, 2)


def _port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


@pytest.mark.parametrize("n,batch,profiles", [(7, 3, True), (1, 4, False), (8, 2, True)])
def test_two_rank_gloo_sweep_gathers_every_problem_in_order(tmp_path, n, batch, profiles):
    import torch.multiprocessing as mp

    from tests import sweep_worker
    mp.spawn(sweep_worker.run, args=(2, _port(), n, batch, profiles, str(tmp_path)), nprocs=2, join=True)
    sc, prof = fake_solve(range(n))
    for r in range(2):
        d = np.load(tmp_path / f"rank{r}.npz")
        np.testing.assert_array_equal(d["F"], sc[:, 0])
        np.testing.assert_array_equal(d["O"], sc[:, 1])
        np.testing.assert_array_equal(d["it"], sc[:, 3].astype(int))
        np.testing.assert_array_equal(d["conv"], sc[:, 4] > 0.5)
        if profiles:
            np.testing.assert_array_equal(d["prof"], prof)


def test_cost_partition_is_deterministic_and_balanced():
    """Longest-processing-time split of an uneven sweep (16 each of 48^3,
    64^3 and 96^3 problems): every problem once, the same split on every
    call, and no rank above 4/3 of the optimum bound (the LPT guarantee)."""
    sizes = [48 ** 3] * 16 + [64 ** 3] * 16 + [96 ** 3] * 16
    costs = [problem_cost(n) for n in sizes]
    for world in (1, 2, 3, 4, 8):
        parts = partition_by_cost(costs, world)
        assert sorted(i for p in parts for i in p) == list(range(len(sizes)))
        assert parts == partition_by_cost(costs, world)
        loads = [sum(costs[i] for i in p) for p in parts]
        bound = max(sum(costs) / world, max(costs))
        assert max(loads) <= (4.0 / 3.0) * bound
    # by count the 96^3 problems would all sit on the last ranks
    by_count = [sum(costs[i] for i in shard(48, r, 4)) for r in range(4)]
    lpt = [sum(costs[i] for i in p) for p in partition_by_cost(costs, 4)]
    assert max(lpt) / min(lpt) < max(by_count) / min(by_count)


def test_two_rank_gloo_uneven_sweep_gathers_every_problem_in_order(tmp_path):
    import torch.multiprocessing as mp

    from tests import sweep_worker
    n = 9
    mp.spawn(sweep_worker.run_uneven, args=(2, _port(), n, str(tmp_path)), nprocs=2, join=True)
    problems = uneven_problems(n)
    sc, prof = fake_uneven_solve(problems)(list(range(n)))
    parts = partition_by_cost([problem_cost(p.model.grid.total_points) for p in problems], 2)
    for r in range(2):
        d = np.load(tmp_path / f"uneven{r}.npz")
        np.testing.assert_array_equal(d["F"], sc[:, 0])
        np.testing.assert_array_equal(d["it"], sc[:, 3].astype(int))
        np.testing.assert_array_equal(d["conv"], sc[:, 4] > 0.5)
        np.testing.assert_array_equal(d["seen"], parts[r])
        np.testing.assert_array_equal(d["lens"], [len(p) for p in prof])
        np.testing.assert_array_equal(d["prof"], np.concatenate(prof))
        for i in range(n):
            assert d["rank"][i] == (0 if i in parts[0] else 1)


@pytest.mark.gpu
def test_gpu_sweep_matches_single_problem_minimisations():
    import classicaldft_b200 as cd
    from classicaldft_b200.sweep import run_sweep
    from tests.parity import Problem, smooth_noise
    shape = (16, 16, 16)
    pr = Problem(shape, 0.25, [1.0], "WhiteBearII", inters=[(0, 0, 1.0, 1.0, 1.8)], kT=1.0)
    rng = np.random.default_rng(6)
    mus = [1.5, 1.0, 0.5, 0.0, -0.5]
    rho0 = [0.4 * (1.0 + 0.05 * smooth_noise(shape, rng)) for _ in mus]
    mz = cd.Minimizer(fire=cd.Fire(dt=0.05, dt_max=0.5, alpha_start=0.01, f_alpha=0.99, force_tolerance=1e-10,
                                   max_steps=4000))
    res = run_sweep(pr.model, pr.fmt, mus, rho0, mz, batch=2, gather_profiles=True)
    for i, mu in enumerate(mus):
        one = mz.grand_potential(pr.model, pr.weights, rho0[i], mu)
        assert res.converged[i] and one.converged
        assert res.grand_potential[i] == pytest.approx(one.grand_potential, rel=1e-12)
        assert np.max(np.abs(res.profiles[i] - one.densities[0])) <= 1e-10
