"""Bulk thermodynamics and the phase search (CPU; the library's host code).

1. The oracle restatement (oracle/bulk.py) is pinned by the reference's own
   tests: tests/unit/functionals/bulk/thermodynamics.cpp (ideal values,
   single-species agreement with the FMT model's own functions, Gibbs-Duhem
   to 1e-12, mean-field terms to 1e-14) and
   tests/integration/functionals/bulk/coexistence.cpp (spinodal and
   coexistence against the legacy solver to 1e-6 at kT = 0.7, 0.8, 0.9;
   equal P and mu at coexistence to 1e-6).
2. The library (cdft_bulk_*) against the oracle: f, mu, P to 1e-13 relative,
   spinodal and coexistence densities to 1e-9 relative (the same bisections
   on the same dP/drho; only round-off differs).
"""
import math

import numpy as np
import pytest

from oracle import bulk as ob
from oracle import fmt as ofmt
from oracle import legacy as oleg
from oracle import potentials as opot

import classicaldft_b200 as cd
from classicaldft_b200 import bulk as cb

MODELS = ["Rosenfeld", "RSLT", "WhiteBearI", "WhiteBearII", "esFMT"]


def oracle_eos(model="Rosenfeld", diameters=(1.0,), inters=(), A=1.0, B=0.0):
    return ob.BulkThermodynamics(list(diameters), ofmt.FMTModel(model, A, B),
                                 [ob.BulkInteraction(i, j, a) for (i, j, a) in inters])


def product_eos(model="Rosenfeld", diameters=(1.0,), inters=(), A=1.0, B=0.0):
    return cb.BulkThermodynamics([cd.Species(f"S{k}", d) for k, d in enumerate(diameters)], cd.FMTModel(model, A, B),
                                 [cb.BulkInteraction(i, j, a) for (i, j, a) in inters])


def lj_a_vdw(kT, rc=2.5):
    return 2.0 * opot.vdw_integral(opot.make_lennard_jones(1.0, 1.0, rc), kT, opot.WCA)


# ------------------------------------------------------ oracle pinning


def test_oracle_ideal_and_hard_sphere_known_answers():
    eos = oracle_eos()
    assert eos.free_energy_density([1.0]) - eos.hard_sphere_free_energy_density([1.0]) == pytest.approx(-1.0,
                                                                                                     abs=1e-14)
    for name in ["Rosenfeld", "RSLT", "WhiteBearI", "WhiteBearII"]:
        e = oracle_eos(name)
        m = ofmt.FMTModel(name)
        assert e.hard_sphere_free_energy_density([0.5]) == pytest.approx(m.free_energy_density(0.5, 1.0), rel=1e-14)
    for name in ["Rosenfeld", "WhiteBearII"]:
        e = oracle_eos(name)
        assert e.hard_sphere_excess_mu([0.4], 0) == pytest.approx(
            ofmt.FMTModel(name).excess_chemical_potential(0.4, 1.0), rel=1e-14)
    assert abs(oracle_eos().hard_sphere_free_energy_density([1e-15])) < 1e-10


def test_oracle_mean_field_terms():
    a = lj_a_vdw(1.0)
    e = oracle_eos(inters=[(0, 0, a)])
    assert e.free_energy_density([0.3]) - oracle_eos().free_energy_density([0.3]) == pytest.approx(
        0.5 * a * 0.09, rel=1e-12)
    assert e.chemical_potential([0.3], 0) - oracle_eos().chemical_potential([0.3], 0) == pytest.approx(a * 0.3,
                                                                                                      rel=1e-12)
    x = oracle_eos(diameters=(1.0, 0.8), inters=[(0, 1, a)])
    x0 = oracle_eos(diameters=(1.0, 0.8))
    assert x.free_energy_density([0.3, 0.2]) - x0.free_energy_density([0.3, 0.2]) == pytest.approx(a * 0.06,
                                                                                                   rel=1e-12)
    assert x.chemical_potential([0.3, 0.2], 0) - x0.chemical_potential([0.3, 0.2], 0) == pytest.approx(
        0.5 * a * 0.2, rel=1e-12)
    assert x.chemical_potential([0.3, 0.2], 1) - x0.chemical_potential([0.3, 0.2], 1) == pytest.approx(
        0.5 * a * 0.3, rel=1e-12)
    assert e.pressure([0.3]) < oracle_eos().pressure([0.3])


def test_oracle_gibbs_duhem_and_limits():
    for e, rho in [(oracle_eos(), [0.3]), (oracle_eos(diameters=(1.0, 0.8)), [0.3, 0.2]),
                   (oracle_eos(inters=[(0, 0, lj_a_vdw(1.0))]), [0.3])]:
        mu = e.chemical_potentials(rho)
        assert e.pressure(rho) == pytest.approx(float(np.dot(rho, mu)) - e.free_energy_density(rho), rel=1e-12)
    e = oracle_eos("WhiteBearII")
    assert e.grand_potential_density([0.4]) == pytest.approx(-e.pressure([0.4]), rel=1e-14)
    assert oracle_eos().pressure([0.4]) > 0.0
    assert oracle_eos().pressure([1e-6]) == pytest.approx(1e-6, rel=1e-4)


@pytest.mark.parametrize("kT", [0.7, 0.8, 0.9])
def test_oracle_phase_search_matches_legacy_solver(kT):
    eos = oracle_eos("WhiteBearII", inters=[(0, 0, lj_a_vdw(kT))])
    ps = ob.PhaseSearch(rho_max=1.0, rho_scan_step=0.005)
    sp = ps.find_spinodal(eos)
    p = lambda r: eos.pressure([r])  # noqa: E731
    c = lambda r: eos.chemical_potential([r], 0)  # noqa: E731
    ls = oleg.legacy_find_spinodal(p, 1.0, 0.005)
    assert sp[0] == pytest.approx(ls[0], rel=1e-6)
    assert sp[1] == pytest.approx(ls[1], rel=1e-6)
    co = ps.find_coexistence(eos)
    lc = oleg.legacy_find_coex(p, c, 1.0, 0.005)
    assert co[0] == pytest.approx(lc[0], rel=1e-6)
    assert co[1] == pytest.approx(lc[1], rel=1e-6)
    if kT == 0.8:
        assert p(co[0]) == pytest.approx(p(co[1]), rel=1e-6)
        assert c(co[0]) == pytest.approx(c(co[1]), rel=1e-6)


# ------------------------------------------------- library vs oracle


@pytest.mark.parametrize("model", MODELS)
def test_library_eos_matches_oracle(model):
    a = lj_a_vdw(0.9)
    cases = [((1.0,), [(0, 0, a)], [0.05]), ((1.0,), [(0, 0, a)], [0.7]),
             ((1.0, 0.6), [(0, 0, a), (0, 1, 0.5 * a), (1, 1, 0.3 * a)], [0.3, 0.25]),
             ((1.0, 0.5, 0.8), [], [0.1, 0.2, 0.15])]
    for diam, inters, rho in cases:
        o = oracle_eos(model, diam, inters, A=1.0, B=0.1)
        g = product_eos(model, diam, inters, A=1.0, B=0.1)
        assert g.free_energy_density(rho) == pytest.approx(o.free_energy_density(rho), rel=1e-13)
        assert g.pressure(rho) == pytest.approx(o.pressure(rho), rel=1e-13)
        np.testing.assert_allclose(g.chemical_potentials(rho), o.chemical_potentials(rho), rtol=1e-13)
        assert g.grand_potential_density(rho) == -g.pressure(rho)


@pytest.mark.parametrize("kT", [0.7, 0.9])
def test_library_phase_search_matches_oracle_and_legacy(kT):
    a = lj_a_vdw(kT)
    o = oracle_eos("WhiteBearII", inters=[(0, 0, a)])
    g = product_eos("WhiteBearII", inters=[(0, 0, a)])
    ops = ob.PhaseSearch(rho_max=1.0, rho_scan_step=0.005)
    gps = cb.PhaseSearch(rho_max=1.0, rho_scan_step=0.005)
    osp, gsp = ops.find_spinodal(o), gps.find_spinodal(g)
    assert gsp.rho_low == pytest.approx(osp[0], rel=1e-9)
    assert gsp.rho_high == pytest.approx(osp[1], rel=1e-9)
    oc, gc = ops.find_coexistence(o), gps.find_coexistence(g)
    assert gc.rho_vapor == pytest.approx(oc[0], rel=1e-9)
    assert gc.rho_liquid == pytest.approx(oc[1], rel=1e-9)
    lc = oleg.legacy_find_coex(lambda r: o.pressure([r]), lambda r: o.chemical_potential([r], 0), 1.0, 0.005)
    assert gc.rho_vapor == pytest.approx(lc[0], rel=1e-6)
    assert gc.rho_liquid == pytest.approx(lc[1], rel=1e-6)


def test_library_density_from_mu_grid_and_failures():
    a = lj_a_vdw(1.0)
    o = oracle_eos("WhiteBearII", inters=[(0, 0, a)])
    g = product_eos("WhiteBearII", inters=[(0, 0, a)])
    rho_true = np.linspace(0.5, 0.85, 8)
    mus = [o.chemical_potential([r], 0) for r in rho_true]
    got = cb.densities_from_chemical_potentials(mus, 0.7, g)
    for r, m, x in zip(rho_true, mus, got):
        ref = ob.density_from_chemical_potential(m, 0.7, o)
        assert x == pytest.approx(ref, rel=1e-12)
        assert x == pytest.approx(r, rel=1e-9)
    # a negative start makes mu(rho) = log(rho) + ... NaN: nullopt in the reference
    assert cb.density_from_chemical_potential(mus[0], -1.0, g) is None
    assert ob.density_from_chemical_potential(mus[0], -1.0, o) is None


def test_no_spinodal_above_the_critical_temperature():
    a = lj_a_vdw(2.0)
    g = product_eos("WhiteBearII", inters=[(0, 0, a)])
    assert cb.PhaseSearch(rho_max=1.0, rho_scan_step=0.005).find_spinodal(g) is None
    assert cb.PhaseSearch(rho_max=1.0, rho_scan_step=0.005).find_coexistence(g) is None
    assert ob.PhaseSearch(rho_max=1.0, rho_scan_step=0.005).find_spinodal(oracle_eos("WhiteBearII",
                                                                                   inters=[(0, 0, a)])) is None


def test_bulk_weights_use_the_continuum_vdw_integral():
    inter = cd.Interaction(0, 0, cd.make_lennard_jones(1.0, 1.0, 2.5))
    bw = cb.make_bulk_weights(cd.WhiteBearII(), [inter], 0.8)
    assert bw[0].a_vdw == pytest.approx(lj_a_vdw(0.8), rel=1e-9)  # quadrature tolerance, as for vdw_integral
    with pytest.raises(ValueError):
        cb.BulkThermodynamics([cd.Species("a", -1.0)], cd.WhiteBearII()).pressure([0.1])
    assert math.isfinite(cb.bulk_thermodynamics([cd.Species("a", 1.0)], cd.WhiteBearII(), [inter], 0.8).pressure(0.3))
