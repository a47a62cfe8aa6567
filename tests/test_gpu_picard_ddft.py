"""Picard iteration, the split-operator and Crank-Nicolson DDFT steps and the
DDFT run with snapshots / stop / reservoir boundary on the device, against
the oracle's restatement of the reference (picard.hpp:63-124,
minimization.hpp:159-180, dynamics.hpp:410-538, 551-557, 583-693).

Tolerances: Picard densities after the same iteration count agree to 1e-10
in max-norm and Omega to 1e-11 relative; a split-operator step to 1e-11 in
max-norm, a Crank-Nicolson step to 1e-10 (its fixed point stops within
fp_tolerance), both 1e-11 relative in the energy.
"""
import numpy as np
import pytest

import classicaldft_b200 as cd
from oracle import algorithms as oalg
from tests.parity import Problem, smooth_noise

pytestmark = pytest.mark.gpu
SHAPE = (16, 16, 16)
DX = 0.25


def problem(model="WhiteBearII", batch=1):
    pr = Problem(SHAPE, DX, [1.0], model, inters=[(0, 0, 1.0, 1.0, 1.8)], kT=1.0)
    if batch > 1:
        pr.weights = cd.make_weights(pr.fmt, pr.model, cd.FP64, batch=batch)
    return pr


def oracle_fn(pr, mu):
    def fn(dens):
        r = pr.ref(dens, [mu])
        return r.grand_potential, r.forces
    return fn


def cluster(r0=1.2, rin=0.6, rout=0.05):
    ix, iy, iz = np.meshgrid(*[np.arange(k) for k in SHAPE], indexing="ij")
    c = [(k * DX) / 2.0 for k in SHAPE]
    r = np.sqrt((ix * DX - c[0]) ** 2 + (iy * DX - c[1]) ** 2 + (iz * DX - c[2]) ** 2)
    return np.where(r < r0, rin, rout).reshape(-1).astype(np.float64)


def test_picard_fixed_iterations_match_oracle():
    pr = problem()
    rng = np.random.default_rng(11)
    rho0 = 0.4 * (1.0 + 0.05 * smooth_noise(SHAPE, rng))
    mu = 1.5
    g = cd.Picard(mixing=0.1, tolerance=1e-14, max_iterations=40).solve([rho0], pr.weights, mu)
    o = oalg.Picard(mixing=0.1, tolerance=1e-14, max_iterations=40).solve([rho0], oracle_fn(pr, mu), DX ** 3)
    assert g.iterations == o.iterations == 40
    assert g.converged == o.converged  # the reference's flag after max_iterations
    assert np.max(np.abs(g.densities[0] - o.densities[0])) <= 1e-10
    assert g.grand_potential == pytest.approx(o.grand_potential, rel=1e-11)
    assert g.residual == pytest.approx(o.residual, rel=1e-9)


def test_picard_converges_like_oracle():
    pr = problem()
    rng = np.random.default_rng(12)
    rho0 = 0.4 * (1.0 + 0.05 * smooth_noise(SHAPE, rng))
    mu = 1.5
    g = cd.Picard(mixing=0.1, tolerance=1e-7, max_iterations=3000, check_interval=10).solve([rho0], pr.weights, mu)
    o = oalg.Picard(mixing=0.1, tolerance=1e-7, max_iterations=3000).solve([rho0], oracle_fn(pr, mu), DX ** 3)
    assert g.converged and o.converged
    assert g.iterations < 3000
    # a tie at the |dOmega| threshold may move the stop by one iteration, which
    # changes rho by about mixing * force / dV
    assert abs(g.iterations - o.iterations) <= 1
    tol = 1e-10 if g.iterations == o.iterations else 1e-4
    assert np.max(np.abs(g.densities[0] - o.densities[0])) <= tol
    assert g.grand_potential == pytest.approx(o.grand_potential, rel=1e-10 if tol < 1e-9 else 1e-8)


def test_picard_fixed_mass_matches_oracle():
    pr = problem("RSLT")
    rho0 = cluster()
    dv = DX ** 3
    bg = np.full(pr.N, 0.05)
    target = float(np.sum(rho0 - bg)) * dv
    mu = 0.3
    cg = cd.fixed_mass_constraint([target], [bg], dv)
    co = oalg.fixed_mass_constraint([target], [bg], dv)
    g = cd.Picard(mixing=0.05, tolerance=1e-14, max_iterations=30).solve([rho0], pr.weights, mu, cg)
    o = oalg.Picard(mixing=0.05, tolerance=1e-14, max_iterations=30).solve([rho0], oracle_fn(pr, mu), dv, co)
    assert g.iterations == o.iterations
    assert float(np.sum(g.densities[0] - bg)) * dv == pytest.approx(target, rel=1e-12)
    assert np.max(np.abs(g.densities[0] - o.densities[0])) <= 1e-10
    assert g.grand_potential == pytest.approx(o.grand_potential, rel=1e-11)


def test_picard_batch_matches_single_problems():
    B = 3
    pr = problem(batch=B)
    single = problem()
    rng = np.random.default_rng(13)
    rhos = np.stack([0.35 * (1.0 + 0.05 * smooth_noise(SHAPE, rng)) for _ in range(B)])
    mus = np.array([0.8, 1.2, 1.5])
    p = cd.Picard(mixing=0.1, tolerance=1e-6, max_iterations=2000, check_interval=7)
    res = p.solve_batch(rhos, pr.weights, mus)
    for b in range(B):
        one = p.solve([rhos[b]], single.weights, mus[b])
        assert res[b].converged and one.converged
        assert res[b].iterations == one.iterations
        assert np.max(np.abs(res[b].densities[0] - one.densities[0])) <= 1e-12
        assert res[b].grand_potential == pytest.approx(one.grand_potential, rel=1e-12)


@pytest.mark.parametrize("scheme", ["split", "cn"])
def test_split_and_cn_steps_match_oracle(scheme):
    pr = problem()
    rng = np.random.default_rng(14)
    rho = 0.35 * (1.0 + 0.05 * smooth_noise(SHAPE, rng))
    grid = pr.omodel.grid
    k2 = oalg.compute_k_squared(grid)
    cfg_g = cd.StepConfig(dt=1e-3, fp_tolerance=1e-11)
    cfg_o = oalg.StepConfig(dt=1e-3, fp_tolerance=1e-11)
    fn = oracle_fn(pr, 0.0)
    rg, ro = rho.copy(), [rho.copy()]
    for _ in range(3):
        if scheme == "split":
            rg, eg, _ = cd.split_operator_step(rg, pr.weights, cfg_g, 0.0)
            prop = oalg.diffusion_propagator(k2, cfg_o.diffusion_coefficient, cfg_o.dt)
            ro, eo, _ = oalg.split_operator_step(ro, grid, k2, prop, fn, cfg_o)
        else:
            rg, eg, _ = cd.crank_nicholson_step(rg, pr.weights, cfg_g, 0.0)
            ro, eo, _ = oalg.crank_nicholson_step(ro, grid, k2, fn, cfg_o)
        # the CN fixed point stops within fp_tolerance of its limit
        assert np.max(np.abs(rg - ro[0])) <= (1e-11 if scheme == "split" else 1e-10)
        assert eg == pytest.approx(eo, rel=1e-11)
    assert cfg_g.dt == 1e-3
    assert float(np.sum(rg)) == pytest.approx(float(np.sum(rho)), rel=1e-6)


def test_simulation_snapshots_stop_and_oracle():
    pr = problem()
    rng = np.random.default_rng(15)
    rho = 0.35 * (1.0 + 0.02 * smooth_noise(SHAPE, rng))
    step = dict(dt=1e-3, dt_max=4e-3, fp_tolerance=1e-9)
    sim = cd.Simulation(step=cd.StepConfig(**step), n_steps=12, snapshot_interval=4, log_interval=5)
    out = sim.run([rho], pr.weights, 0.0)
    assert [s.step for s in out["snapshots"]] == [0, 4, 8, 12]
    assert np.array_equal(out["snapshots"][0].densities[0], rho)
    assert np.array_equal(out["snapshots"][-1].densities[0], out["densities"][0])
    assert [out["all_times"][i] for i in (0, 5, 10, 12)] == out["times"]
    o = oalg.Simulation(step=oalg.StepConfig(**step), n_steps=12).run([rho], pr.omodel.grid, oracle_fn(pr, 0.0))
    assert np.allclose(out["all_times"], o["times"], rtol=1e-14, atol=0)
    assert np.allclose(out["all_energies"], o["energies"], rtol=1e-11, atol=0)
    assert np.max(np.abs(out["densities"][0] - o["densities"][0])) <= 1e-10
    # a snapshot equals the state of a run that ended there
    short = cd.Simulation(step=cd.StepConfig(**step), n_steps=8, snapshot_interval=0).run([rho], pr.weights, 0.0)
    assert np.max(np.abs(out["snapshots"][2].densities[0] - short["densities"][0])) <= 1e-13
    # the stop condition ends the run after the step it fires on
    seen = []

    def stop(s, t, e):
        seen.append(s)
        return s == 7

    st = cd.Simulation(step=cd.StepConfig(**step), n_steps=12, snapshot_interval=3, stop_condition=stop)
    so = st.run([rho], pr.weights, 0.0)
    assert so["steps"] == 7 and seen == list(range(1, 8))
    assert [s.step for s in so["snapshots"]] == [0, 3, 6]
    seven = cd.Simulation(step=cd.StepConfig(**step), n_steps=7, snapshot_interval=0).run([rho], pr.weights, 0.0)
    assert np.max(np.abs(so["densities"][0] - seven["densities"][0])) <= 1e-13


def test_reservoir_boundary_matches_oracle():
    pr = problem()
    rng = np.random.default_rng(16)
    rho = 0.35 * (1.0 + 0.05 * smooth_noise(SHAPE, rng))
    mask = np.zeros(SHAPE, dtype=bool)
    mask[0, :, :] = True
    mask = mask.reshape(-1)
    res = 0.3
    step = dict(dt=1e-3, dt_max=1e-3, fp_tolerance=1e-9)
    out = cd.Simulation(step=cd.StepConfig(**step), n_steps=5, snapshot_interval=0,
                        boundary=cd.reservoir_boundary(mask, res)).run([rho], pr.weights, 0.0)

    def bnd(dens):
        for r in dens:
            r[mask] = res

    o = oalg.Simulation(step=oalg.StepConfig(**step), n_steps=5, boundary=bnd).run(
        [rho], pr.omodel.grid, oracle_fn(pr, 0.0))
    assert np.all(out["densities"][0][mask] == res)
    assert np.max(np.abs(out["densities"][0] - o["densities"][0])) <= 1e-10
    assert out["mass_initial"] == pytest.approx(o["mass_initial"], rel=1e-13)
    assert out["mass_final"] == pytest.approx(o["mass_final"], rel=1e-12)
