"""Mean-field cell weights made on the GPU (cdft_create_model) against the
host set-up loop (cdft_interaction_weight) and the oracle's restatement of
mean_field.hpp:42-196.

Tolerances: a_vdw to 1e-13 relative (sums of the same cell weights in a
different order; the device may fuse multiply-adds); the mean-field energy,
F and the forces of an evaluation with device weights to 1e-13 relative of
the evaluation with host weights.
"""
import numpy as np
import pytest

import classicaldft_b200 as cd
from oracle import potentials as op
from oracle.grid import Grid as OGrid
from tests.parity import force_err, rel_err, smooth_noise

pytestmark = pytest.mark.gpu

SCHEMES = ["InterpolationZero", "InterpolationLinearE", "InterpolationLinearF", "InterpolationQuadraticF", "GaussE",
           "GaussF"]
POTS = {
    "lj": (lambda: cd.make_lennard_jones(1.0, 1.0, 2.5), lambda: op.make_lennard_jones(1.0, 1.0, 2.5)),
    "lj_uncut": (lambda: cd.make_lennard_jones(1.0, 1.0), lambda: op.make_lennard_jones(1.0, 1.0)),
    "twf": (lambda: cd.make_ten_wolde_frenkel(1.0, 1.0, 2.0), lambda: op.make_ten_wolde_frenkel(1.0, 1.0, 2.0)),
    "wrdf": (lambda: cd.make_wang_ramirez_dobnikar_frenkel(1.0, 1.0, 2.0),
             lambda: op.make_wang_ramirez_dobnikar_frenkel(1.0, 1.0, 2.0)),
}
SPLITS = {cd.WEEKS_CHANDLER_ANDERSEN: op.WCA, cd.BARKER_HENDERSON: op.BH}


def models(shape, dx, pot, split, scheme, kT=0.8):
    grid = cd.Grid(dx=dx, box_size=tuple(n * dx for n in shape), shape=shape)
    inter = cd.Interaction(0, 0, pot, split, scheme)
    return grid, cd.Model(grid, [cd.Species("a", 1.0)], [inter], kT)


@pytest.mark.parametrize("scheme", SCHEMES)
@pytest.mark.parametrize("pot", list(POTS))
def test_device_weights_match_host_and_oracle(scheme, pot):
    shape, dx, kT = (24, 20, 28), 0.2, 0.8
    for split, osplit in SPLITS.items():
        if pot == "wrdf" and split == cd.BARKER_HENDERSON and scheme != "InterpolationQuadraticF":
            continue  # one WRDF/BH case keeps the matrix short
        grid, model = models(shape, dx, POTS[pot][0](), split, scheme, kT)
        fmt = cd.FMTModel("WhiteBearII")
        wd = cd.make_weights(fmt, model, cd.FP64, weights_on="device")
        wh = cd.make_weights(fmt, model, cd.FP64, weights_on="host")
        og = OGrid(dx=dx, box_size=grid.box_size, shape=shape)
        _, ar = op.interaction_weight_real(op.Interaction(0, 0, POTS[pot][1](), osplit, scheme), og, kT)
        assert wd.a_vdw[0] == pytest.approx(wh.a_vdw[0], rel=1e-13)
        assert wd.a_vdw[0] == pytest.approx(ar, rel=1e-13)
        rng = np.random.default_rng(5)
        rho = 0.4 * (1.0 + 0.2 * smooth_noise(shape, rng))
        gd = cd.total(model, [rho], wd, [-1.0])
        gh = cd.total(model, [rho], wh, [-1.0])
        assert rel_err(gd.parts["mean_field"], gh.parts["mean_field"]) <= 1e-13
        assert rel_err(gd.free_energy, gh.free_energy) <= 1e-13
        assert force_err(gd.forces, gh.forces) <= 1e-13


def test_device_weights_batched_binary_odd_grid():
    shape, dx = (15, 17, 9), 0.25
    grid = cd.Grid(dx=dx, box_size=tuple(n * dx for n in shape), shape=shape)
    inters = [cd.Interaction(0, 0, cd.make_lennard_jones(1.0, 1.0, 2.5)),
              cd.Interaction(0, 1, cd.make_lennard_jones(0.9, 0.8, 2.2)),
              cd.Interaction(1, 1, cd.make_ten_wolde_frenkel(0.8, 0.5, 2.0))]
    model = cd.Model(grid, [cd.Species("a", 1.0), cd.Species("b", 0.8)], inters, 1.1)
    fmt = cd.FMTModel("RSLT")
    wd = cd.make_weights(fmt, model, cd.FP64, batch=2, weights_on="device")
    wh = cd.make_weights(fmt, model, cd.FP64, batch=2, weights_on="host")
    for a, b in zip(wd.a_vdw, wh.a_vdw):
        assert a == pytest.approx(b, rel=1e-13)
    rng = np.random.default_rng(6)
    rho = 0.3 * (1.0 + 0.1 * rng.standard_normal((2, 2, grid.total_points)))
    rd = cd.total_batch(model, rho, wd, [[0.1, 0.2], [0.3, -0.1]])
    rh = cd.total_batch(model, rho, wh, [[0.1, 0.2], [0.3, -0.1]])
    for x, y in zip(rd, rh):
        assert rel_err(x.free_energy, y.free_energy) <= 1e-13
        assert force_err(x.forces, y.forces) <= 1e-13


def test_create_model_rejects_bad_input():
    grid, model = models((16, 16, 16), 0.2, cd.make_lennard_jones(1.0, 1.0, 2.5), cd.WEEKS_CHANDLER_ANDERSEN,
                         "InterpolationQuadraticF", kT=0.8)
    bad = cd.Model(grid, model.species, model.interactions, -1.0)
    with pytest.raises(ValueError, match="temperature"):
        cd.make_weights(cd.FMTModel("WhiteBearII"), bad, cd.FP64)
