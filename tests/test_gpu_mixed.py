"""Mixed-precision evaluation (FP32 FFTs / k-space products, FP64 Phi and sums)
against the FP64 oracle.

Tolerances, from the specification of the mixed path:
  * near-uniform states (the DDFT configuration: 1% noise): |dF|/|F| <= 1e-9,
    max|d force| <= 1e-6 max|force|;
  * strongly inhomogeneous states (walls, 20% smoothed noise): the FP32
    round-off is no longer confined to small fluctuations, |dF|/|F| <= 1e-6.
"""
import numpy as np
import pytest

import classicaldft_b200 as cd
from tests.parity import Problem, force_err, rel_err, smooth_noise

pytestmark = pytest.mark.gpu
LJ = (1.0, 1.0, 2.5)


@pytest.mark.parametrize("model", ["WhiteBearII", "RSLT", "esFMT"])
def test_mixed_near_uniform_meets_1e9(model):
    shape = (64, 64, 64)
    pr = Problem(shape, 0.125, [1.02], model, inters=[(0, 0) + LJ], kT=0.8, precision=cd.MIXED)
    rng = np.random.default_rng(20261204)
    rho = 0.35 * (1.0 + 0.01 * rng.uniform(-1.0, 1.0, pr.N))
    g = pr.gpu([rho], [-1.0])
    r = pr.ref([rho], [-1.0])
    assert rel_err(g.free_energy, r.free_energy) <= 1e-9
    assert rel_err(g.grand_potential, r.grand_potential) <= 1e-9
    assert force_err(g.forces, r.forces) <= 1e-6


def test_mixed_binary_mixture():
    shape = (32, 32, 32)
    inters = [(0, 0) + LJ, (0, 1, 1.0, 0.8, 2.5)]
    pr = Problem(shape, 0.2, [1.0, 0.5], "esFMT", inters=inters, kT=1.0, precision=cd.MIXED)
    rng = np.random.default_rng(7)
    r1 = 0.3 * (1.0 + 0.01 * rng.uniform(-1, 1, pr.N))
    r2 = 0.1 * (1.0 + 0.01 * rng.uniform(-1, 1, pr.N))
    g = pr.gpu([r1, r2], [0.1, 0.2])
    r = pr.ref([r1, r2], [0.1, 0.2])
    assert rel_err(g.free_energy, r.free_energy) <= 1e-9
    assert force_err(g.forces, r.forces) <= 1e-6


def test_mixed_strongly_inhomogeneous():
    shape = (48, 48, 48)
    pr = Problem(shape, 0.1, [1.0], "WhiteBearII", inters=[(0, 0) + LJ], precision=cd.MIXED)
    rng = np.random.default_rng(8)
    rho = 0.5 * (1.0 + 0.2 * smooth_noise(shape, rng))
    v = np.zeros(pr.N)
    v.reshape(shape)[:5] = 30.0
    rho.reshape(shape)[:5] = 1e-10
    g = pr.gpu([rho], [0.5], [v])
    r = pr.ref([rho], [0.5], [v])
    assert rel_err(g.free_energy, r.free_energy) <= 1e-6
    assert force_err(g.forces, r.forces) <= 1e-4
