"""cdft_total_stream: a sequence of host states evaluated with the copies of
one state overlapping the evaluation of the next (two device slots).

Each state's result must equal cdft_total on that state bitwise (the same
kernels on the same inputs), for mixed and FP64 engines, with and without
external fields, for a batched engine, and for more states than slots with
page-locked and pageable host buffers.
"""
import ctypes

import numpy as np
import pytest

import classicaldft_b200 as cd
from tests.parity import Problem, smooth_noise

pytestmark = pytest.mark.gpu
LJ = (1.0, 1.0, 2.5)


def _states(shape, count, seed, S=1):
    rng = np.random.default_rng(seed)
    return [np.stack([0.3 * (1.0 + 0.05 * smooth_noise(shape, rng)).ravel() for _ in range(S)]) for _ in range(count)]


@pytest.mark.parametrize("precision", [cd.MIXED, cd.FP64])
def test_stream_equals_one_call_per_state(precision):
    shape = (64, 32, 32)
    pr = Problem(shape, 0.1, [1.0], "WhiteBearII", inters=[(0, 0) + LJ], kT=0.9, precision=precision)
    states = _states(shape, 5, 11)
    mus = [[0.1 * i - 0.2] for i in range(5)]
    rng = np.random.default_rng(12)
    vexts = [None, [rng.uniform(0.0, 0.5, pr.grid.total_points)], None, None,
             [rng.uniform(0.0, 0.5, pr.grid.total_points)]]
    got = cd.total_stream(pr.model, states, pr.weights, mus, vexts)
    assert len(got) == 5
    for i, st in enumerate(states):
        ref = cd.total(pr.model, st, pr.weights, mus[i], vexts[i])
        assert got[i].free_energy == ref.free_energy, i
        assert got[i].grand_potential == ref.grand_potential, i
        assert got[i].parts == ref.parts, i
        assert np.array_equal(got[i].forces[0], ref.forces[0]), i
    assert cd.total_stream(pr.model, [], pr.weights, []) == []


def test_stream_batched_engine_and_pinned_buffers():
    import torch
    shape = (32, 32, 32)
    pr = Problem(shape, 0.2, [1.0, 0.6], "WhiteBearII", inters=[(0, 0) + LJ, (0, 1, 1.0, 0.8, 2.5)], kT=0.9,
                 precision=cd.MIXED)
    B, S, N = 2, 2, pr.grid.total_points
    w = cd.make_weights(pr.fmt, pr.model, cd.MIXED, batch=B)
    e = w.engine
    count = 3
    rng = np.random.default_rng(13)
    rho = [torch.tensor(np.stack([np.stack(_states(shape, 1, 20 + 7 * i + b, S=2)[0]) for b in range(B)]))
           .pin_memory() for i in range(count)]
    force = [torch.empty(B, S, N, dtype=torch.float64).pin_memory() for _ in range(count)]
    mu = rng.uniform(-0.3, 0.3, (count, B, S))
    sc = e.total_stream_ptrs([r.data_ptr() for r in rho], mu, [f.data_ptr() for f in force])
    assert sc.shape == (count, B, 10)
    for i in range(count):
        s_ref, f_ref = e.total_host(rho[i].numpy(), mu[i])
        assert np.array_equal(sc[i], s_ref), i
        assert np.array_equal(force[i].numpy(), f_ref), i
    # forces may be skipped per state; scalars still come back
    sc2 = e.total_stream_ptrs([r.data_ptr() for r in rho], mu, [None, force[1].data_ptr(), None])
    assert np.array_equal(sc2, sc)
    e.close()


def test_stream_rejects_missing_states():
    shape = (32, 32, 32)
    pr = Problem(shape, 0.2, [1.0], "WhiteBearII", precision=cd.MIXED)
    L = cd.lib()
    arr = (ctypes.c_void_p * 2)(None, None)
    mu = (ctypes.c_double * 2)(0.0, 0.0)
    assert L.cdft_total_stream(pr.weights.engine.handle, 2, arr, None, mu, None, None) == -1
    assert L.cdft_total_stream(pr.weights.engine.handle, -1, arr, None, mu, None, None) == -1
