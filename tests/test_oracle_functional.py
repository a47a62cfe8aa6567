"""Pins the oracle's mean-field, ideal, external and total terms (reference known answers)."""
import math

import numpy as np
import pytest

from oracle import fmt, legacy
from oracle.functional import (Model, Species, external_field, hard_sphere, ideal_gas, make_weights,
                               mean_field, total)
from oracle.grid import Grid, make_grid
from oracle.potentials import (BH, LINEAR_F, QUADRATIC_F, WCA, ZERO, GAUSS_E, Interaction, cell_weight,
                               hard_sphere_diameter, make_lennard_jones, vdw_integral)

GRID = Grid(dx=0.1, box_size=(1.6, 1.6, 1.6), shape=(16, 16, 16))
N = 16 ** 3
KT = 1.0
VOL = 1.6 ** 3


def lj():
    return make_lennard_jones(1.0, 1.0, 2.5)


def mf_weights(inters, grid=GRID, kT=KT, nspec=1):
    model = Model(grid, [Species(f"S{i}", 1.0) for i in range(nspec)], inters, kT)
    return model, make_weights(fmt.FMTModel("Rosenfeld"), model)


# ---- tests/unit/functionals/mean_field.cpp --------------------------------

def test_a_vdw_negative_and_schemes_differ():
    """mean_field.cpp:64-70, 234-250, 289-314."""
    avals = {}
    for sch in (QUADRATIC_F, ZERO, LINEAR_F, GAUSS_E):
        _, w = mf_weights([Interaction(0, 0, lj(), WCA, sch)])
        avals[sch] = w.mean_field[0]["a_vdw"]
        assert avals[sch] < 0.0
    assert abs(avals[ZERO] - avals[LINEAR_F]) > 1e-10


def test_a_vdw_matches_continuum_integral():
    """mean_field.cpp:72-88 (epsilon 0.05)."""
    pot = make_lennard_jones(0.5, 1.0, 0.75)
    a_cont = 2.0 * vdw_integral(pot, KT, WCA)
    _, w = mf_weights([Interaction(0, 0, pot, WCA, QUADRATIC_F)])
    assert w.mean_field[0]["a_vdw"] == pytest.approx(a_cont, rel=0.05)


def test_mean_field_uniform():
    """mean_field.cpp:92-179."""
    model, w = mf_weights([Interaction(0, 0, lj())])
    a = w.mean_field[0]["a_vdw"]
    F, f = mean_field(model, [np.full(N, 0.5)], w)
    assert F == pytest.approx(0.5 * a * 0.25 * VOL, rel=1e-6)
    F3, _ = mean_field(model, [np.full(N, 0.3)], w)
    F6, _ = mean_field(model, [np.full(N, 0.6)], w)
    assert F6 / F3 == pytest.approx(4.0, rel=1e-6)
    _, f = mean_field(model, [np.full(N, 0.4)], w)
    assert np.max(np.abs(f[0] - f[0].mean())) < 1e-8
    assert f[0][0] == pytest.approx(a * 0.4 * GRID.cell_volume, rel=1e-6)
    F0, f0 = mean_field(model, [np.zeros(N)], w)
    assert F0 == pytest.approx(0.0, abs=1e-14) and np.max(np.abs(f0[0])) < 1e-14


def test_mean_field_cross_interaction():
    """mean_field.cpp:183-230."""
    model, w = mf_weights([Interaction(0, 1, lj())], nspec=2)
    a = w.mean_field[0]["a_vdw"]
    F, f = mean_field(model, [np.full(N, 0.3), np.full(N, 0.2)], w)
    assert F == pytest.approx(0.5 * a * 0.3 * 0.2 * VOL, rel=1e-6)
    dv = GRID.cell_volume
    assert f[0][0] == pytest.approx(0.5 * a * 0.2 * dv, rel=1e-6)
    assert f[1][0] == pytest.approx(0.5 * a * 0.3 * dv, rel=1e-6)
    for s in range(2):
        assert np.max(np.abs(f[s] - f[s].mean())) < 1e-8


# ---- tests/integration/functionals/mean_field.cpp (legacy) ----------------

@pytest.mark.parametrize("dx", [0.4, 0.2])
def test_qf_cell_weights_match_legacy(dx):
    """mean_field.cpp(integration):22-72 (margin 1e-10)."""
    inter = Interaction(0, 0, make_lennard_jones(1.0, 1.0, 2.5), WCA, QUADRATIC_F)
    lim = 1 + int(2.5 / dx)
    rc = 2.5 + math.sqrt(3.0) * 0.5 * dx
    for ix in range(lim + 2):
        for iy in range(ix + 1):
            for iz in range(iy + 1):
                if (ix * ix + iy * iy + iz * iz) * dx * dx > rc * rc:
                    continue
                ours = float(cell_weight(inter, 1.0, dx, ix, iy, iz))
                ref = legacy.generate_weight_qf(1.0, 1.0, 2.5, ix, iy, iz, dx)
                assert ours == pytest.approx(ref, abs=1e-10)


@pytest.mark.parametrize("dx", [0.5, 0.4])
def test_grid_a_vdw_matches_legacy(dx):
    """mean_field.cpp(integration):74-109 (margin 1e-10); the grid weight of
    interaction_weight_real sums to the same a_vdw on a box wider than 2 r_c."""
    pot = make_lennard_jones(1.0, 1.0, 2.5)
    ref = legacy.compute_a_vdw_qf(1.0, 1.0, 2.5, 1.0, dx)
    lim = 1 + int(2.5 / dx)
    rc = 2.5 + math.sqrt(3.0) * 0.5 * dx
    inter = Interaction(0, 0, pot, WCA, QUADRATIC_F)
    r = np.arange(-(lim + 1), lim + 2)
    SX, SY, SZ = np.meshgrid(r, r, r, indexing="ij")
    keep = (SX * SX + SY * SY + SZ * SZ) * dx * dx <= rc * rc
    w = cell_weight(inter, 1.0, dx, SX[keep], SY[keep], SZ[keep])
    assert float(np.sum(w * dx ** 3)) == pytest.approx(ref, abs=1e-10)
    n = 2 * (lim + 2) + 2
    model = Model(make_grid(dx, (n * dx,) * 3), [Species("A", 1.0)], [inter], 1.0)
    wts = make_weights(fmt.FMTModel("Rosenfeld"), model)
    assert wts.mean_field[0]["a_vdw"] == pytest.approx(ref, abs=1e-10)


def test_lj_factory_and_diameters():
    """potentials.hpp:311-325 values; d_HS(kT=1, WCA) of LJ is close to 1."""
    p = make_lennard_jones(1.0, 1.0, 2.5)
    assert p.r_min == pytest.approx(2 ** (1 / 6))
    assert p.v_min == pytest.approx(-1.0 - p.epsilon_shift)
    d = hard_sphere_diameter(p, 1.0, WCA)
    assert 0.95 < d < 1.05
    dbh = hard_sphere_diameter(p, 1.0, BH)
    assert 0.9 < dbh < 1.05


# ---- ideal / external / total ----------------------------------------------

def test_ideal_gas_and_external_field():
    """ideal_gas.cpp:24-108, external_field.cpp:23-99."""
    g = make_grid(0.1, (1.0, 1.0, 1.0))
    model = Model(g, [Species("A", 1.0)], [], 1.0)
    n = g.total_points
    dv = g.cell_volume
    F, f = ideal_gas(model, [np.full(n, 0.5)], [0.0])
    assert F == pytest.approx(0.5 * (math.log(0.5) - 1.0) * dv * n, abs=1e-10)
    F, f = ideal_gas(model, [np.full(n, 0.3)], [2.0])
    assert f[0][0] == pytest.approx((math.log(0.3) - 2.0) * dv, abs=1e-14)
    F, f = ideal_gas(model, [np.full(n, 0.3), np.full(n, 0.7)], [0.0, 0.0])
    assert F == pytest.approx((0.3 * (math.log(0.3) - 1) + 0.7 * (math.log(0.7) - 1)) * dv * n, abs=1e-10)
    v = np.linspace(0, 1, n)
    F, f = external_field(model, [np.full(n, 0.4)], [v])
    assert F == pytest.approx(float(np.sum(0.4 * v)) * dv, rel=1e-14)
    assert np.allclose(f[0], v * dv)
    F, f = ideal_gas(model, [np.zeros(n)], [0.0])
    assert F == 0.0 and np.all(np.isfinite(f[0]))


def test_total_is_sum_of_parts():
    """functionals.cpp:78-183 (epsilon 1e-12)."""
    inters = [Interaction(0, 0, make_lennard_jones(1.0, 1.0, 2.5))]
    model = Model(GRID, [Species("HS", 1.0)], inters, KT)
    w = make_weights(fmt.FMTModel("Rosenfeld"), model)
    rng = np.random.default_rng(3)
    rho = 0.3 * (1.0 + 0.05 * rng.standard_normal(N))
    v = rng.standard_normal(N)
    res = total(model, [rho], w, [1.5], [v])
    Fi, fi = ideal_gas(model, [rho], [1.5])
    Fe, fe = external_field(model, [rho], [v])
    Fh, fh = hard_sphere(model, [rho], w)
    Fm, fm = mean_field(model, [rho], w)
    assert res.free_energy == pytest.approx(Fi + Fe + Fh + Fm, rel=1e-12)
    assert np.max(np.abs(res.forces[0] - (fi[0] + fe[0] + fh[0] + fm[0]))) < 1e-12
    assert res.grand_potential == pytest.approx(res.free_energy - 1.5 * float(np.sum(rho)) * GRID.cell_volume,
                                                rel=1e-12)
