"""The saddle-point path on the GPU: the block Lanczos eigen solver, the
saddle search against the oracle's Search::find, and the mixed-precision
search (FP64 refinement) against the FP64 one.

* Lanczos against the dense fixed-boundary Hessian of the oracle (central
  differences, interior block, 8^3 grid): lowest eigenvalue to 1e-8
  relative, eigenvector |overlap| >= 1 - 1e-8, zero on the faces; block
  sizes 1, 2 and 4 (batched products).
* On a critical nucleus (24^3, dx = 0.5, LJ at kT = 0.8, S = 1.5): the
  reference's Rayleigh-Ritz iteration (exact products) and Lanczos find the
  same negative eigenvalue (1e-3: the Rayleigh-Ritz tolerance is a residual
  of 1e-4).
* Search::find (saddle_point.hpp:367-589) with the reference's own eigen
  solver and finite-difference products against the oracle from the same
  cluster: same outer iterations and FIRE steps, Omega to 1e-9 relative, the
  eigenvalue to 1e-4, the saddle density to 1e-7 in max-norm.
* The mixed-precision search with the FP64 refine engine and Lanczos on
  batched FP64 products against the FP64 search from the same cluster: the
  barrier (Omega at the saddle) to 1e-8 relative.  The two searches take
  different FIRE paths and a nucleus in a periodic box can end anywhere
  along its translation modes, so the profiles are compared by what does
  not depend on the position: the mass to 1e-9 relative and the sorted
  density values to 1e-4 (the position-dependent max-norm is not a
  criterion here).
"""
import numpy as np
import pytest

import classicaldft_b200 as cd
from oracle import algorithms as oalg
from oracle.grid import boundary_mask
from tests.parity import Problem, smooth_noise

pytestmark = pytest.mark.gpu
KT = 0.8
LJ = cd.make_lennard_jones(1.0, 1.0, 3.0)
D = LJ.hard_sphere_diameter(KT, cd.WEEKS_CHANDLER_ANDERSEN)
INTER = [(0, 0, 1.0, 1.0, 3.0)]


def nucleus(n, dx, S=1.5, R0=3.0, cluster_tol=1e-10):
    """The reference's nucleation set-up (tests/integration/algorithms/
    nucleation.cpp:100-160): coexistence from the grid EOS, a step-function
    droplet of the coexisting liquid in vapour at supersaturation S, the
    fixed-mass FIRE cluster, its background density and chemical potential."""
    pr = Problem((n,) * 3, dx, [D], "RSLT", inters=INTER, kT=KT)
    eos = cd.make_bulk_thermodynamics(pr.model.species, pr.weights)
    co = cd.PhaseSearch(rho_max=1.0, rho_scan_step=0.005).find_coexistence(eos)
    rout = S * co.rho_vapor
    mu = eos.chemical_potential([rout], 0)
    x = np.arange(n) * dx - n * dx / 2
    X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
    rho0 = np.where(np.sqrt(X ** 2 + Y ** 2 + Z ** 2).ravel() < R0, co.rho_liquid, rout)
    tm = float(rho0.sum()) * pr.grid.cell_volume
    fire = cd.Fire(dt=0.1, dt_max=1.0, alpha_start=0.01, f_alpha=0.99, force_tolerance=cluster_tol, max_steps=20000)
    cl = cd.Minimizer(fire=fire, param=cd.Unbounded(1e-99)).fixed_mass(pr.model, pr.weights, rho0, mu, tm)
    assert cl.converged
    rc = np.asarray(cl.densities[0])
    bd = boundary_mask(pr.omodel.grid).astype(bool)
    bg = float(rc[bd].mean())
    assert rc.max() > 10.0 * bg  # a droplet, not an evaporated cluster
    return pr, rc, eos.chemical_potential([bg], 0), tm


@pytest.mark.parametrize("block", [1, 2, 4])
def test_lanczos_matches_the_dense_oracle_hessian(block):
    n = 8
    pr = Problem((n,) * 3, 0.5, [D], "RSLT", inters=INTER, kT=KT)
    rho = 0.3 * (1.0 + 0.3 * smooth_noise((n,) * 3, np.random.default_rng(3)))
    H, inner = oalg.dense_fixed_boundary_hessian(pr.omodel.grid, lambda r: pr.ref([r], [0.0]).forces[0], rho)
    w, V = np.linalg.eigh(0.5 * (H + H.T))
    hw = cd.make_weights(pr.fmt, pr.model, cd.FP64, batch=block) if block > 1 else None
    lz = cd.EigenvalueSolver(1e-8, 400, exact_hvp=True, method="lanczos", block=block).solve(
        pr.weights, rho, 0.0, hvp_weights=hw)
    assert lz.converged
    assert abs(lz.eigenvalue - w[0]) <= 1e-8 * abs(w[0])
    e = np.zeros(rho.size)
    e[inner] = V[:, 0]
    assert abs(float(np.dot(lz.eigenvector, e))) >= 1.0 - 1e-8
    faces = boundary_mask(pr.omodel.grid).astype(bool)
    assert np.all(lz.eigenvector[faces] == 0.0)
    assert float(np.linalg.norm(lz.eigenvector)) == pytest.approx(1.0, abs=1e-12)


def test_lanczos_and_rayleigh_ritz_agree_on_a_nucleus():
    pr, rc, mubg, _ = nucleus(24, 0.5)
    rr = cd.EigenvalueSolver(1e-4, 300, exact_hvp=True).solve(pr.weights, rc, mubg)
    lz = cd.EigenvalueSolver(1e-8, 300, exact_hvp=True, method="lanczos").solve(pr.weights, rc, mubg)
    assert lz.converged and lz.eigenvalue < 0.0
    assert lz.eigenvalue == pytest.approx(rr.eigenvalue, rel=1e-3)
    assert abs(float(np.dot(lz.eigenvector, rr.eigenvector))) > 0.999


def test_saddle_search_matches_the_oracle():
    pr, rc, mubg, tm = nucleus(24, 0.5)
    sf = dict(dt=1e-3, dt_max=1.0, alpha_start=0.01, f_alpha=1.0, force_tolerance=1e-10, max_steps=300)
    kw = dict(omega_tolerance=1e-12, tolerance_start=1e-6, max_outer_iterations=3)
    g = cd.Search(fire=cd.Fire(**sf), eigenvalue=cd.EigenvalueSolver(1e-4, 300, 1e-6), **kw).find(
        pr.model, pr.weights, rc, mubg, tm)

    def ofn(rho, mu):
        r = pr.ref([rho], [mu])
        return r.free_energy, r.grand_potential, r.forces[0]

    o = oalg.Search(fire=oalg.Fire(**sf), eigenvalue=oalg.EigenvalueSolver(1e-4, 300, 1e-6), **kw).find(
        pr.omodel.grid, ofn, rc, mubg, tm)
    assert g.outer_iterations == o.outer_iterations
    assert g.fire_steps == o.fire_steps > 0
    assert g.grand_potential == pytest.approx(o.grand_potential, rel=1e-9)
    assert g.eigenvalue < 0.0 and g.eigenvalue == pytest.approx(o.eigenvalue, rel=1e-4)
    assert np.max(np.abs(g.density - o.density)) <= 1e-7
    assert abs(float(np.dot(g.eigenvector, o.eigenvector))) > 0.9999


def test_mixed_saddle_search_with_refinement_matches_fp64():
    """The batched-product Lanczos search in mixed precision with the FP64
    defect-correction engine reaches the FP64 search's barrier within 1e-8."""
    pr64, rc, mubg, tm = nucleus(32, 0.4, cluster_tol=1e-9)
    prm = Problem((32,) * 3, 0.4, [D], "RSLT", inters=INTER, kT=KT, precision=cd.MIXED)
    hw = cd.make_weights(pr64.fmt, pr64.model, cd.FP64, batch=2)
    sf = dict(dt=1e-3, dt_max=1.0, alpha_start=0.01, f_alpha=1.0, force_tolerance=1e-10, max_steps=20000)
    out = {}
    for label, w, kw in (("fp64", pr64.weights, {}), ("mixed", prm.weights, dict(refine=pr64.weights))):
        se = cd.Search(fire=cd.Fire(**sf),
                       eigenvalue=cd.EigenvalueSolver(1e-6, 300, exact_hvp=True, method="lanczos", block=2),
                       omega_tolerance=1e-9, tolerance_start=1e-6, max_outer_iterations=12, hvp_weights=hw, **kw)
        out[label] = se.find(pr64.model, w, rc, mubg, tm)
        assert out[label].converged and out[label].eigenvalue < 0.0
    a, b = out["fp64"], out["mixed"]
    assert a.fire_steps > 0 and b.fire_steps > 0
    assert b.grand_potential == pytest.approx(a.grand_potential, rel=1e-8)
    assert b.eigenvalue == pytest.approx(a.eigenvalue, rel=1e-6)
    assert float(b.density.sum()) == pytest.approx(float(a.density.sum()), rel=1e-9)
    assert np.max(np.abs(np.sort(a.density) - np.sort(b.density))) <= 1e-4
