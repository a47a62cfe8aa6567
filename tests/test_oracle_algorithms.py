"""Pins the oracle's FIRE2, minimiser and DDFT restatement (reference known answers)."""
import math

import numpy as np
import pytest

from oracle import algorithms as alg
from oracle.grid import Grid, boundary_mask, fixed_boundary, homogeneous_boundary, make_grid


def quadratic(x):
    """fire.cpp:11-19."""
    return sum(0.5 * float(np.dot(a, a)) for a in x), [-a for a in x]


def test_fire_quadratic_and_multispecies():
    """fire.cpp:21-76."""
    st = alg.Fire().initialize([np.array([1.0, 2.0, 3.0])], quadratic)
    assert st.energy == pytest.approx(7.0) and st.rms_force > 0 and st.iteration == 0 and not st.converged
    cfg = alg.Fire(dt=0.01, force_tolerance=1e-6)
    st = cfg.initialize([np.array([1.0, 2.0, 3.0])], quadratic)
    _, f = quadratic(st.x)
    st2, _ = cfg.step(st, f, quadratic)
    assert st2.energy < st.energy and st2.iteration == 1
    cfg = alg.Fire(dt=0.01, force_tolerance=1e-6, max_steps=5000)
    r = cfg.minimize([np.array([5.0])], quadratic)
    assert r.converged and abs(r.x[0][0]) < 1e-3 and r.energy < 1e-6
    r = cfg.minimize([np.array([3.0, -2.0, 1.0])], quadratic)
    assert r.converged and np.linalg.norm(r.x[0]) < 1e-3
    r = cfg.minimize([np.array([2.0, 1.0]), np.array([-1.0, 3.0])], quadratic)
    assert r.converged and np.linalg.norm(r.x[0]) < 1e-3 and np.linalg.norm(r.x[1]) < 1e-3
    assert alg.Fire(force_tolerance=1e-6).initialize([np.zeros(3)], quadratic).converged


def test_fire_rosenbrock_and_uphill():
    """fire.cpp:80-137."""
    def rb(x):
        xi, yi = x[0]
        e = (1 - xi) ** 2 + 100 * (yi - xi * xi) ** 2
        dfdx = -2 * (1 - xi) - 400 * xi * (yi - xi * xi)
        dfdy = 200 * (yi - xi * xi)
        return e, [np.array([-dfdx, -dfdy])]
    r = alg.Fire(dt=1e-4, dt_max=1e-3, force_tolerance=0.1, max_steps=50000).minimize([np.array([-1.0, 1.0])], rb)
    assert r.energy < rb([np.array([-1.0, 1.0])])[0] * 0.1
    count = [0]

    def alternating(x):
        count[0] += 1
        sign = -1.0 if count[0] % 2 == 0 else 1.0
        return sign * float(np.dot(x[0], x[0])), [sign * (-2.0 * x[0])]
    with pytest.raises(RuntimeError):
        alg.Fire(dt=0.5, dt_max=0.5, n_delay=0, max_uphill=3, force_tolerance=1e-10,
                 max_steps=5000).minimize([np.array([1.0, 1.0])], alternating)


def test_parametrizations():
    """minimization.cpp:14-113."""
    u = alg.Unbounded(1e-18)
    assert np.allclose(alg.to_density(np.zeros(3), u), 1e-18)
    assert np.allclose(alg.to_density(np.array([1.0, 2.0, 3.0]), alg.Unbounded(0.0)), [1, 4, 9])
    x = np.array([0.5, 1.0, 2.5])
    assert np.allclose(alg.from_density(alg.to_density(x, u), u), x, rtol=1e-12)
    assert np.allclose(alg.transform_force(np.ones(3), np.array([1.0, 2.0, 3.0]), alg.Unbounded(0.0)), [2, 4, 6])
    b = alg.Bounded(1e-18, 0.9)
    xb = np.array([0.1, 0.5, 1.0, 5.0])
    assert np.allclose(alg.from_density(alg.to_density(xb, b), b), xb, rtol=1e-10)
    assert alg.to_density(np.array([1e6]), alg.Bounded(0.0, 1.0))[0] == pytest.approx(1.0, rel=1e-6)
    xb = np.array([1.0, 2.0])
    fx = alg.transform_force(np.ones(2), xb, alg.Bounded(0.0, 1.0))
    assert np.allclose(fx, 2.0 * xb / (1 + xb * xb) ** 2, rtol=1e-12)


def test_boundary_masks():
    """minimization.cpp:117-158."""
    g = make_grid(1.0, (3.0, 3.0, 3.0))
    m = boundary_mask(g)
    assert int(m.sum()) == 26
    f = np.arange(27, dtype=np.float64)
    r = homogeneous_boundary(f, m)
    assert r[13] == 13.0 and np.allclose(r[m.astype(bool)], r[0])
    r = fixed_boundary(np.ones(27), m)
    assert r[13] == 1.0 and np.all(r[m.astype(bool)] == 0.0)


GRID8 = Grid(dx=0.5, box_size=(4.0, 4.0, 4.0), shape=(8, 8, 8))


def ideal_forces(dens):
    """dynamics.cpp:17-27."""
    dv = GRID8.cell_volume
    e = 0.0
    out = []
    for d in dens:
        rho = np.clip(d, 1e-18, np.inf)
        e += float(np.sum(rho * (np.log(rho) - 1.0))) * dv
        out.append(np.log(rho) * dv)
    return e, out


def gaussian_blob(amp):
    n = GRID8.shape
    ix, iy, iz = np.meshgrid(*[np.arange(k) for k in n], indexing="ij")
    x = (ix - n[0] / 2.0) * 0.5
    y = (iy - n[1] / 2.0) * 0.5
    z = (iz - n[2] / 2.0) * 0.5
    return (0.5 + amp * np.exp(-(x * x + y * y + z * z))).reshape(-1)


def test_ddft_helpers_and_steps():
    """dynamics.cpp:31-179."""
    k2 = alg.compute_k_squared(GRID8)
    assert k2.size == 8 * 8 * 5 and k2.reshape(-1)[0] == pytest.approx(0.0, abs=1e-14) and np.all(k2 >= 0)
    prop = alg.diffusion_propagator(k2, 1.0, 0.01)
    assert prop.reshape(-1)[0] == pytest.approx(1.0) and np.all(prop > 0) and np.all(prop <= 1 + 1e-14)
    cfg = alg.StepConfig(dt=1e-4)
    rho0 = gaussian_blob(0.1)
    dv = GRID8.cell_volume
    d, _, _ = alg.split_operator_step([rho0], GRID8, k2, alg.diffusion_propagator(k2, 1.0, 1e-4), ideal_forces, cfg)
    assert float(np.sum(d[0])) * dv == pytest.approx(float(np.sum(rho0)) * dv, rel=1e-3)
    d, _, _ = alg.split_operator_step([np.full(512, 0.1)], GRID8, k2, alg.diffusion_propagator(k2, 1.0, 1e-5),
                                      ideal_forces, alg.StepConfig(dt=1e-5))
    assert np.all(d[0] > 0)
    rho = [gaussian_blob(0.3)]
    var0 = np.var(rho[0])
    p3 = alg.diffusion_propagator(k2, 1.0, 1e-3)
    for _ in range(10):
        rho, _, _ = alg.split_operator_step(rho, GRID8, k2, p3, ideal_forces, alg.StepConfig(dt=1e-3))
    assert np.var(rho[0]) < var0
    d, _, _ = alg.crank_nicholson_step([np.full(512, 0.1)], GRID8, k2, ideal_forces, alg.StepConfig(dt=1e-4))
    assert np.all(d[0] > 0)
    d, _, _ = alg.crank_nicholson_step([rho0], GRID8, k2, ideal_forces, alg.StepConfig(dt=1e-4))
    assert float(np.sum(d[0])) == pytest.approx(float(np.sum(rho0)), rel=1e-3)


def test_integrating_factor_ideal_gas_is_exact_diffusion():
    """For the ideal gas R(rho) = div(rho grad ln rho) - lap rho vanishes up to the
    FD discretisation; the IF step then diffuses with the exact FD propagator and
    conserves mass to round-off."""
    rho0 = gaussian_blob(0.1)
    st = alg.IFState(GRID8)
    cfg = alg.StepConfig(dt=1e-3)
    d, e, dt = alg.integrating_factor_step([rho0], GRID8, st, ideal_forces, cfg)
    assert dt == 1e-3
    assert float(np.sum(d[0])) == pytest.approx(float(np.sum(rho0)), rel=1e-12)
    assert np.var(d[0]) < np.var(rho0)


def test_picard_ideal_gas_converges_to_exp_mu():
    """picard.hpp:63-124 on the ideal gas: force / dV = ln rho - mu, so
    ln rho - mu shrinks by (1 - mixing) per iteration and the fixed point is
    exp(mu)."""
    mu = -1.2
    dv = GRID8.cell_volume

    def fn(dens):
        e, f = ideal_forces(dens)
        return e - mu * float(np.sum(dens[0])) * dv, [f[0] - mu * dv]

    rho0 = gaussian_blob(0.2)
    p = alg.Picard(mixing=0.2, tolerance=1e-9, max_iterations=2000)
    r = p.solve([rho0], fn, dv)
    # Omega stops changing (|dOmega| < tol, second order in the error) before
    # the force RMS falls below the tolerance
    assert r.converged and r.residual > 1e-9
    assert np.max(np.abs(r.densities[0] - math.exp(mu))) < 1e-5
    # the loop stops before updating: the residual belongs to the returned state
    f = (np.log(r.densities[0]) - mu) * dv
    assert math.sqrt(float(np.mean(f * f))) == pytest.approx(r.residual, rel=1e-9)
    # one iteration by hand
    r1 = alg.Picard(mixing=0.2, max_iterations=1).solve([rho0], fn, dv)
    assert r1.iterations == 1
    assert np.allclose(r1.densities[0], rho0 * np.exp(-0.2 * (np.log(rho0) - mu)), rtol=1e-14)
    # max_iterations exhausted: omega_prev equals omega, so the reference reports converged
    assert r1.converged


def test_fixed_mass_constraint_rescales_the_excess():
    """minimization.hpp:159-180."""
    dv = GRID8.cell_volume
    bg = np.full(512, 0.05)
    rho = gaussian_blob(0.3)
    target = 1.7
    out = alg.fixed_mass_constraint([target], [bg], dv)([rho])
    assert float(np.sum(out[0] - bg)) * dv == pytest.approx(target, rel=1e-13)
    # a zero excess is left as it is
    same = alg.fixed_mass_constraint([target], [bg], dv)([bg.copy()])
    assert np.array_equal(same[0], bg)
