"""The anchored mixed-precision split (cdft_engine_set_anchor) against the
FP64 engine and the oracle.

The mean split's FP32 round-off scales with the density's own swing: on the
binary FCC solid of the crystal tests (a = 1.55, dx = 0.0484375, large
spheres d = 1 as Gaussian peaks alpha = 50 with 0.8 particles per site,
small spheres d = 0.5 uniform at 0.1, esFMT A = 1 B = 0; 64^3 = 2 x 2 x 2
cells) it gives |dF|/|F| ~ 2e-7.  Anchored at the crystal rho_a, an
evaluation transforms only rho - rho_a in FP32:

* at rho = rho_a: F to 1e-13 of FP64, forces to 1e-12 of their max;
* at rho = rho_a (1 + 0.01 G) (G smoothed unit noise): |dF|/|F| <= 1e-9
  against FP64 and against the oracle (measured 3.5e-10 against 1.2e-7 for
  the mean split), forces to 1e-7 of their max (1.1e-8 against 3.7e-7); the
  F error at least 100 times and the force error at least 10 times below
  the mean split's on the same state;
* one species with an external field (the generic pointwise kernel takes
  over from the one-species kernels), a batched engine, clearing the
  anchor (bitwise the evaluation before it) and the argument checks.
"""
import math

import numpy as np
import pytest

import classicaldft_b200 as cd
from classicaldft_b200 import crystal as cc
from tests.parity import Problem, force_err, rel_err, smooth_noise

pytestmark = pytest.mark.gpu

A_FCC, DX5, ALPHA, OCC = 1.55, 0.0484375, 50.0, 0.8


def fcc_binary(cells=2):
    n = int(round(cells * A_FCC / DX5))
    lat = cc.build_lattice(cc.Structure.FCC, cc.Orientation._001, (cells,) * 3)
    sites = lat.scaled_positions(A_FCC / math.sqrt(2.0))
    grid = cd.Grid(dx=DX5, box_size=(n * DX5,) * 3, shape=(n,) * 3)
    rho1 = cc.gaussian_peaks(grid, sites, ALPHA, OCC * (ALPHA / math.pi) ** 1.5, 0.0).cpu().numpy()
    rho2 = np.full(grid.total_points, 0.1)
    return (n,) * 3, rho1, rho2


def test_anchored_binary_solid_matches_fp64_and_oracle():
    import torch
    shape, r1, r2 = fcc_binary(2)
    p64 = Problem(shape, DX5, [1.0, 0.5], "esFMT", A=1.0, B=0.0, precision=cd.FP64)
    pmx = Problem(shape, DX5, [1.0, 0.5], "esFMT", A=1.0, B=0.0, precision=cd.MIXED)
    e = pmx.weights.engine
    anchor = torch.tensor(np.concatenate([r1, r2]), device="cuda")
    rng = np.random.default_rng(21)
    q1 = r1 * (1.0 + 0.01 * smooth_noise(shape, rng).ravel())
    q2 = r2 * (1.0 + 0.01 * smooth_noise(shape, rng).ravel())
    mu = [0.3, -0.2]
    plain = pmx.gpu([q1, q2], mu)
    e.set_anchor(p64.weights.engine, anchor)
    assert e.anchored
    # at the anchor itself
    a0, f0 = pmx.gpu([r1, r2], mu), p64.gpu([r1, r2], mu)
    assert rel_err(a0.free_energy, f0.free_energy) <= 1e-13
    assert force_err(a0.forces, f0.forces) <= 1e-12
    # near it
    a1, f1 = pmx.gpu([q1, q2], mu), p64.gpu([q1, q2], mu)
    ref = p64.ref([q1, q2], mu)
    e_anc, e_plain = rel_err(a1.free_energy, f1.free_energy), rel_err(plain.free_energy, f1.free_energy)
    print(f"binary FCC 64^3, 1% off the anchor: |dF/F| anchored {e_anc:.2e}, mean split {e_plain:.2e}")
    assert e_anc <= 1e-9
    assert rel_err(a1.free_energy, ref.free_energy) <= 1e-9
    assert rel_err(a1.grand_potential, ref.grand_potential) <= 1e-9
    assert force_err(a1.forces, f1.forces) <= 1e-7
    assert force_err(a1.forces, ref.forces) <= 1e-7
    assert e_anc * 100.0 <= e_plain
    assert force_err(a1.forces, f1.forces) * 10.0 <= force_err(plain.forces, f1.forces)


def test_anchored_one_species_with_field_batch_and_clear():
    import torch
    shape = (32, 32, 32)
    inters = [(0, 0, 1.0, 1.0, 2.5)]
    p64 = Problem(shape, 0.1, [1.0], "WhiteBearII", inters=inters, kT=0.9, precision=cd.FP64)
    pmx = Problem(shape, 0.1, [1.0], "WhiteBearII", inters=inters, kT=0.9, precision=cd.MIXED)
    rng = np.random.default_rng(22)
    ra = 0.4 * (1.0 + 0.3 * smooth_noise(shape, rng)).ravel()
    rb = ra * (1.0 + 0.01 * smooth_noise(shape, rng).ravel())
    v = 0.2 * smooth_noise(shape, rng).ravel()
    e = pmx.weights.engine
    before = pmx.gpu([rb], [0.1], [v])
    e.set_anchor(p64.weights.engine, ra)
    got, want = pmx.gpu([rb], [0.1], [v]), p64.gpu([rb], [0.1], [v])
    ref = p64.ref([rb], [0.1], [v])
    assert rel_err(got.free_energy, want.free_energy) <= 1e-9
    assert rel_err(got.grand_potential, ref.grand_potential) <= 1e-9
    assert force_err(got.forces, want.forces) <= 1e-7
    assert force_err(got.forces, ref.forces) <= 1e-7
    e.clear_anchor()
    assert not e.anchored
    again = pmx.gpu([rb], [0.1], [v])
    assert again.free_energy == before.free_energy
    assert np.array_equal(again.forces[0], before.forces[0])
    # a batched engine: each problem anchored at its own state
    B = 2
    w64b = cd.make_weights(p64.fmt, p64.model, cd.FP64, batch=B)
    wmxb = cd.make_weights(pmx.fmt, pmx.model, cd.MIXED, batch=B)
    anchors = np.stack([ra, 0.9 * ra])
    states = np.stack([rb, 0.9 * rb])
    wmxb.engine.set_anchor(w64b.engine, anchors)
    gb = cd.total_batch(pmx.model, states.reshape(B, 1, -1), wmxb, [0.1, 0.2])
    for b in range(B):
        rb_ref = p64.ref([states[b]], [(0.1, 0.2)[b]])
        assert rel_err(gb[b].free_energy, rb_ref.free_energy) <= 1e-9
        assert force_err(gb[b].forces, rb_ref.forces) <= 1e-7
    # argument checks
    with pytest.raises(ValueError):
        p64.weights.engine.set_anchor(p64.weights.engine, ra)  # an FP64 engine has no split
    with pytest.raises(ValueError):
        e.set_anchor(pmx.weights.engine, ra)  # the anchor engine must be FP64
    other = Problem((32, 32, 16), 0.1, [1.0], "WhiteBearII", inters=inters, kT=0.9, precision=cd.FP64)
    with pytest.raises(ValueError):
        e.set_anchor(other.weights.engine, ra)
    for w in (w64b, wmxb):
        w.engine.close()
