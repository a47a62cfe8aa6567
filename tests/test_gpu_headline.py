"""The benchmarked state itself against the FP64 oracle.

The throughput figure is quoted on one configuration: a periodic 128^3 grid,
dx = 0.125 sigma, kT = 0.8, one species with White-Bear-II FMT at the WCA
hard-sphere diameter of a cut LJ potential (sigma = eps = 1, r_c = 2.5, QF
weights), rho = 0.35 (1 + 0.01 U(-1, 1)) with seed 20261204.  Here that state
is evaluated on the fused mixed-precision path (hand-written 128-point plane
and column kernels, the default for this engine) and on the FP64 path, and
both are compared with the oracle's functionals::total
(include/dft/functionals/functionals.hpp:64-95) on the same input:

* mixed:  |dF|/|F| and |dOmega|/|Omega| <= 1e-9, max|dforce| <= 1e-6 max|force|;
* FP64:   |dF|/|F| and |dOmega|/|Omega| <= 1e-12, max|dforce| <= 1e-11 max|force|.
"""
import numpy as np
import pytest

import classicaldft_b200 as cd
from oracle import fmt as ofmt
from oracle import potentials as opot
from oracle.functional import Model as OModel
from oracle.functional import Species as OSpecies
from oracle.functional import make_weights as o_make_weights
from oracle.functional import total as o_total
from oracle.grid import Grid as OGrid
from tests.parity import force_err, rel_err

pytestmark = pytest.mark.gpu

SHAPE, DX, KT, RHO_BAR, SEED = (128, 128, 128), 0.125, 0.8, 0.35, 20261204


@pytest.fixture(scope="module")
def headline():
    rng = np.random.default_rng(SEED)
    rho = RHO_BAR * (1.0 + 0.01 * rng.uniform(-1.0, 1.0, int(np.prod(SHAPE))))
    box = tuple(n * DX for n in SHAPE)
    lj = cd.make_lennard_jones(1.0, 1.0, 2.5)
    d = lj.hard_sphere_diameter(KT, cd.WEEKS_CHANDLER_ANDERSEN)
    model = cd.Model(cd.Grid(dx=DX, box_size=box, shape=SHAPE), [cd.Species("LJ", d)], [cd.Interaction(0, 0, lj)],
                     KT)
    olj = opot.make_lennard_jones(1.0, 1.0, 2.5)
    od = opot.hard_sphere_diameter(olj, KT, opot.WCA)
    assert abs(od - d) <= 1e-13 * d
    omodel = OModel(OGrid(dx=DX, box_size=box, shape=SHAPE), [OSpecies("LJ", od)], [opot.Interaction(0, 0, olj)], KT)
    mu = [-0.37]
    ref = o_total(omodel, [rho], o_make_weights(ofmt.FMTModel("WhiteBearII"), omodel), mu)
    return model, rho, mu, ref


@pytest.mark.parametrize("precision,f_tol,force_tol", [(cd.MIXED, 1e-9, 1e-6), (cd.FP64, 1e-12, 1e-11)])
def test_headline_state_matches_oracle(headline, precision, f_tol, force_tol):
    model, rho, mu, ref = headline
    w = cd.make_weights(cd.WhiteBearII(), model, precision)
    assert w.engine.transforms == ("fused" if precision == cd.MIXED else "cufft")
    res = cd.total(model, [rho], w, mu)
    assert rel_err(res.free_energy, ref.free_energy) <= f_tol
    assert rel_err(res.grand_potential, ref.grand_potential) <= f_tol
    assert force_err(res.forces, ref.forces) <= force_tol
    w.engine.close()


def test_headline_state_every_chunk_count(headline):
    """The autotuner may pick any plane-chunk count: each gives the same
    forces and the oracle's F."""
    model, rho, mu, ref = headline
    w = cd.make_weights(cd.WhiteBearII(), model, cd.MIXED)
    base = None
    for k in (1, 2, 4, 8):
        w.engine.set_plane_chunks(k)
        res = cd.total(model, [rho], w, mu)
        assert rel_err(res.free_energy, ref.free_energy) <= 1e-9
        if base is None:
            base = res.forces[0]
        assert np.array_equal(res.forces[0], base), k
    w.engine.close()


def test_headline_state_every_pointwise_variant(headline):
    """The generic and the one-species pointwise kernels evaluate the same
    expressions, and each meets the oracle's tolerances.  Their FP64 results
    may differ in the last bit (contraction of products into fused multiply-
    adds is the compiler's choice per kernel, and the branch-free kernels 3,
    4 and 5 form 1/eta and 1/(1-eta) from one reciprocal), which can flip the
    FP32 rounding of a derivative channel: against the generic kernel the
    forces agree to 1e-8 of the largest force and F to 1e-13."""
    model, rho, mu, ref = headline
    w = cd.make_weights(cd.WhiteBearII(), model, cd.MIXED)
    assert w.engine.pointwise_variants == [0, 1, 2, 3, 4, 5]
    base = None
    for v in (0, 1, 2, 3, 4, 5):
        w.engine.set_pointwise(v)
        assert w.engine.pointwise == v
        res = cd.total(model, [rho], w, mu)
        assert rel_err(res.free_energy, ref.free_energy) <= 1e-9
        assert force_err(res.forces, ref.forces) <= 1e-6
        if base is None:
            base = res
        assert force_err(res.forces, base.forces) <= 1e-8, v
        assert rel_err(res.free_energy, base.free_energy) <= 1e-13, v
    with pytest.raises(ValueError):
        w.engine.set_pointwise(6)
    assert w.engine.column_tile == 16
    with pytest.raises(ValueError):  # one species: 16-column tiles only
        w.engine.set_column_tile(32)
    w.engine.close()


def test_headline_state_dependent_launch_same_results(headline):
    """Programmatic dependent launch between the passes changes when a pass
    is scheduled, not what it computes: F and forces bitwise equal on and
    off (four plane chunks, the launch order the bench uses)."""
    model, rho, mu, ref = headline
    w = cd.make_weights(cd.WhiteBearII(), model, cd.MIXED)
    w.engine.set_plane_chunks(4)
    assert w.engine.dependent_launch
    on = cd.total(model, [rho], w, mu)
    w.engine.set_dependent_launch(False)
    assert not w.engine.dependent_launch
    off = cd.total(model, [rho], w, mu)
    assert on.free_energy == off.free_energy
    assert np.array_equal(on.forces[0], off.forces[0])
    assert rel_err(on.free_energy, ref.free_energy) <= 1e-9
    w.engine.close()
