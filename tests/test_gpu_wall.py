"""The hard-wall minimisation at its own size: 64^3, dx = 0.1, kT = 1, WBII
(d = 1) + cut LJ (WCA, QF), rho = 0.5 (1 + 0.05 G) with smoothed Gaussian
noise, a hard wall at x = 0 (rho = 0 and V_ext = 50 kT on the planes
x < d/2), FIRE grand-potential minimisation at the bulk mu of rho = 0.5.

* FP64 and mixed precision with the FP64 refine engine converge to the same
  profile within 1e-8 in max-norm, Omega within 1e-10 relative;
* the oracle evaluating the converged FP64 profile finds it stationary (the
  functional of the reference, include/dft/functionals/functionals.hpp:64-95,
  with V_ext): the rms of its forces in the minimiser's variable x
  (rho = rho_min + x^2, dOmega/dx = 2 x dOmega/drho) is the convergence
  criterion's, below 1e-11, and max |dOmega/drho| / dV over the fluid is
  below 1e-4 (the largest forces sit in the dilute first layer at the wall,
  where x is small).
The box is periodic (no boundary treatment) and convergence is the rms
force of Fire::step (fire.hpp:162) below 1e-11 (at 1e-10 the two converged
profiles agree only to ~1.5e-8: the tolerance ball of the criterion).
"""
import numpy as np
import pytest

import classicaldft_b200 as cd
from tests.parity import Problem

pytestmark = pytest.mark.gpu


def test_hard_wall_mixed_refined_matches_fp64_and_the_oracle():
    n, dx = 64, 0.1
    pr = Problem((n,) * 3, dx, [1.0], "WhiteBearII", inters=[(0, 0, 1.0, 1.0, 2.5)], kT=1.0)
    prm = Problem((n,) * 3, dx, [1.0], "WhiteBearII", inters=[(0, 0, 1.0, 1.0, 2.5)], kT=1.0, precision=cd.MIXED)
    rng = np.random.default_rng(20261205)
    w = rng.standard_normal((n,) * 3)
    k = [2.0 * np.pi * np.fft.fftfreq(n, d=dx)] * 3
    K2 = k[0][:, None, None] ** 2 + k[1][None, :, None] ** 2 + k[2][None, None, :] ** 2
    g = np.real(np.fft.ifftn(np.fft.fftn(w) * np.exp(-0.5 * 0.25 * K2)))
    rho0 = 0.5 * (1.0 + 0.05 * (g / g.std()).reshape(-1))
    wall = np.repeat(np.arange(n), n * n) * dx < 0.5
    rho0[wall] = 0.0
    vext = np.where(wall, 50.0, 0.0)
    mu = cd.make_bulk_thermodynamics(pr.model.species, pr.weights).chemical_potential([0.5], 0)
    # periodic box: no boundary treatment; convergence on the rms force
    fire = cd.Fire(dt=0.1, dt_max=1.0, alpha_start=0.01, f_alpha=0.99, force_tolerance=1e-11, max_steps=50000)
    kw = dict(use_homogeneous_boundary=False, use_monitor=False)
    a = cd.Minimizer(fire=fire, **kw).grand_potential(pr.model, pr.weights, rho0, mu, external_field=vext)
    b = cd.Minimizer(fire=fire, refine=pr.weights, refine_switch=1e3, **kw).grand_potential(
        prm.model, prm.weights, rho0, mu, external_field=vext)
    assert a.converged and b.converged
    assert np.max(np.abs(a.densities[0] - b.densities[0])) <= 1e-8
    assert b.grand_potential == pytest.approx(a.grand_potential, rel=1e-10)
    # the wall stays empty and the fluid is layered against it
    assert np.max(a.densities[0][wall]) < 1e-12
    ref = pr.ref([a.densities[0]], [mu], [vext])
    x = np.sqrt(np.maximum(a.densities[0] - 1e-18, 0.0))
    assert float(np.sqrt(np.mean((2.0 * x * ref.forces[0]) ** 2))) <= 1.001e-11
    assert np.max(np.abs(ref.forces[0][~wall])) / pr.grid.cell_volume <= 1e-4
    assert ref.grand_potential == pytest.approx(a.grand_potential, rel=1e-12)
