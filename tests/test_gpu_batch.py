"""Batched engines (cdft_create_batch): B problems of one grid evaluated by one
set of launches, each problem against the FP64 oracle with the tolerances of
the single-problem tests (|dF|/|F| <= 1e-12, forces 1e-11 of their max;
mixed precision 1e-9 against the FP64 engine near uniform density), and
against the same problem evaluated alone by an unbatched engine.
"""
import numpy as np
import pytest

import classicaldft_b200 as cd
from tests.parity import Problem, force_err, rel_err, smooth_noise

pytestmark = pytest.mark.gpu

F_TOL = 1e-12
FORCE_TOL = 1e-11
LJ = (1.0, 1.0, 2.5)


def batch_of(pr, B, S, shape, seed, mean=0.4, amp=0.1):
    rng = np.random.default_rng(seed)
    rho = np.stack([np.stack([mean * (1.0 + amp * smooth_noise(shape, rng)) for _ in range(S)]) for _ in range(B)])
    mu = rng.uniform(-2.0, 2.0, (B, S))
    vext = 0.5 * rng.standard_normal((B, S, pr.N))
    return rho, mu, vext


def batched_weights(pr, B, precision=cd.FP64):
    return cd.make_weights(pr.fmt, pr.model, precision, batch=B)


@pytest.mark.parametrize("model", ["WhiteBearII", "RSLT"])
def test_batch_matches_oracle_and_single_engine(model):
    shape = (24, 24, 24)
    pr = Problem(shape, 0.2, [1.0], model, inters=[(0, 0) + LJ], kT=0.9)
    B = 5
    rho, mu, vext = batch_of(pr, B, 1, shape, 1)
    w = batched_weights(pr, B)
    res = cd.total_batch(pr.model, rho, w, mu, vext)
    assert len(res) == B
    for b in range(B):
        ref = pr.ref([rho[b, 0]], [mu[b, 0]], [vext[b, 0]])
        assert rel_err(res[b].free_energy, ref.free_energy) <= F_TOL
        assert rel_err(res[b].grand_potential, ref.grand_potential) <= F_TOL
        assert force_err(res[b].forces, ref.forces) <= FORCE_TOL
        one = pr.gpu([rho[b, 0]], [mu[b, 0]], [vext[b, 0]])
        assert rel_err(res[b].free_energy, one.free_energy) <= 1e-13
        assert force_err(res[b].forces, one.forces) <= 1e-13


def test_batch_binary_mixture_and_odd_grid():
    """Two species with a cross interaction on a grid with N % 4 != 0 (the
    register-prefetch pointwise kernel)."""
    shape = (15, 18, 21)
    inters = [(0, 0) + LJ, (0, 1, 1.0, 0.8, 2.5)]
    pr = Problem(shape, 0.2, [1.0, 0.6], "esFMT", inters=inters, kT=1.1)
    B = 3
    rho, mu, _ = batch_of(pr, B, 2, shape, 2, 0.25, 0.2)
    w = batched_weights(pr, B)
    res = cd.total_batch(pr.model, rho, w, mu)
    for b in range(B):
        ref = pr.ref(list(rho[b]), list(mu[b]))
        assert rel_err(res[b].free_energy, ref.free_energy) <= F_TOL
        assert rel_err(res[b].grand_potential, ref.grand_potential) <= F_TOL
        assert force_err(res[b].forces, ref.forces) <= FORCE_TOL


def test_batch_mixed_precision_meets_1e9():
    shape = (32, 32, 32)
    pr = Problem(shape, 0.2, [1.0], "WhiteBearII", inters=[(0, 0) + LJ], kT=0.8)
    B = 8
    rng = np.random.default_rng(3)
    rho = 0.35 * (1.0 + 0.01 * rng.uniform(-1.0, 1.0, (B, 1, pr.N)))
    mu = np.linspace(-3.0, 1.0, B)
    w64 = batched_weights(pr, B)
    w32 = batched_weights(pr, B, cd.MIXED)
    r64 = cd.total_batch(pr.model, rho, w64, mu)
    r32 = cd.total_batch(pr.model, rho, w32, mu)
    for b in range(B):
        assert rel_err(r32[b].free_energy, r64[b].free_energy) <= 1e-9
        assert rel_err(r32[b].grand_potential, r64[b].grand_potential) <= 1e-9
        assert force_err(r32[b].forces, r64[b].forces) <= 1e-6


def test_batch_device_api_matches_host_api():
    import torch
    shape = (16, 16, 16)
    pr = Problem(shape, 0.25, [1.0], "WhiteBearI", inters=[(0, 0, 1.0, 1.0, 1.8)], kT=1.0)
    B = 4
    rho, mu, vext = batch_of(pr, B, 1, shape, 4)
    w = batched_weights(pr, B)
    host = cd.total_batch(pr.model, rho, w, mu, vext)
    d_rho = torch.tensor(rho, device="cuda")
    d_v = torch.tensor(vext, device="cuda")
    d_f = torch.empty_like(d_rho)
    d_sc = torch.empty((B, 10), dtype=torch.float64, device="cuda")
    w.engine.total_device(d_rho.data_ptr(), d_v.data_ptr(), mu, d_f.data_ptr(), d_sc.data_ptr(),
                          torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    sc = d_sc.cpu().numpy()
    f = d_f.cpu().numpy()
    for b in range(B):
        assert sc[b, 0] == host[b].free_energy
        assert sc[b, 1] == host[b].grand_potential
        assert np.array_equal(f[b, 0], host[b].forces[0])


def test_batch_engine_rejects_single_problem_drivers():
    pr = Problem((8, 8, 8), 0.25, [1.0], "Rosenfeld")
    w = batched_weights(pr, 2)
    assert w.engine.batch == 2
    with pytest.raises(ValueError, match="batch 1"):
        cd.Minimizer().grand_potential(pr.model, w, 0.3 * np.ones(pr.N), 0.0)
    with pytest.raises(ValueError, match="batch 1"):
        cd.hessian_times_vector(w, 0.3 * np.ones(pr.N), np.ones(pr.N), 0.0, exact=True)


def _fire():
    return cd.Fire(dt=0.05, dt_max=0.5, alpha_start=0.01, f_alpha=0.99, force_tolerance=1e-10, max_steps=4000)


def test_batched_fire_grand_potential_matches_single_problem_runs_and_oracle():
    """Three state points minimised together: each problem converges at its
    own iteration and ends where the single-problem minimiser (and the oracle
    restatement of Minimizer::grand_potential) ends."""
    from oracle import algorithms as oalg
    shape = (16, 16, 16)
    pr = Problem(shape, 0.25, [1.0], "WhiteBearII", inters=[(0, 0, 1.0, 1.0, 1.8)], kT=1.0)
    rng = np.random.default_rng(5)
    B = 3
    rho0 = np.stack([0.4 * (1.0 + 0.05 * smooth_noise(shape, rng)) for _ in range(B)])
    mus = np.array([1.5, 0.5, -1.0])
    wb = batched_weights(pr, B)
    mz = cd.Minimizer(fire=_fire(), param=cd.Unbounded(1e-18))
    res = mz.grand_potential_batch(pr.model, wb, rho0, mus)
    iters = []
    for b in range(B):
        one = mz.grand_potential(pr.model, pr.weights, rho0[b], mus[b])
        assert res[b].converged and one.converged
        assert res[b].iterations == one.iterations
        assert np.max(np.abs(res[b].densities[0] - one.densities[0])) <= 1e-10
        assert res[b].grand_potential == pytest.approx(one.grand_potential, rel=1e-12)
        iters.append(res[b].iterations)
    assert len(set(iters)) > 1  # the problems stop at different steps

    def ofn(r, mu):
        o = pr.ref([r], [mu])
        return o.free_energy, o.grand_potential, o.forces[0]
    ofire = oalg.Fire(dt=0.05, dt_max=0.5, alpha_start=0.01, f_alpha=0.99, force_tolerance=1e-10, max_steps=4000)
    o = oalg.Minimizer(fire=ofire, param=oalg.Unbounded(1e-18)).grand_potential(pr.omodel.grid, ofn, rho0[0], mus[0])
    assert np.max(np.abs(res[0].densities[0] - o.densities[0])) <= 1e-8


def test_batched_fire_fixed_mass_keeps_each_target():
    shape = (16, 16, 16)
    pr = Problem(shape, 0.25, [1.0], "RSLT", inters=[(0, 0, 1.0, 1.0, 1.8)], kT=1.0)
    ix, iy, iz = np.meshgrid(*[np.arange(k) for k in shape], indexing="ij")
    r = np.sqrt(((ix - 8) * 0.25) ** 2 + ((iy - 8) * 0.25) ** 2 + ((iz - 8) * 0.25) ** 2).reshape(-1)
    rho0 = np.stack([np.where(r < r0, 0.6, 0.05) for r0 in (1.0, 1.3)])
    dv = 0.25 ** 3
    masses = rho0.sum(axis=1) * dv
    wb = batched_weights(pr, 2)
    mz = cd.Minimizer(fire=_fire(), param=cd.Unbounded(1e-99))
    res = mz.fixed_mass_batch(pr.model, wb, rho0, [0.3, 0.3], masses)
    for b in range(2):
        one = mz.fixed_mass(pr.model, pr.weights, rho0[b], 0.3, masses[b])
        assert res[b].converged
        assert float(np.sum(res[b].densities[0])) * dv == pytest.approx(masses[b], rel=1e-12)
        assert np.max(np.abs(res[b].densities[0] - one.densities[0])) <= 1e-10
