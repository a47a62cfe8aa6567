"""Integrating-factor DDFT of a hard-sphere FCC solid with the anchored
mixed-precision split (Simulation.anchor / anchor_interval), against FP64.

The solid: 64^3, dx = 0.0484375, 2 x 2 x 2 FCC cells (a = 1.55), one Gaussian
peak (alpha = 50) of one particle per site, White-Bear II, no attraction.
100 steps at a fixed dt = 1e-7 (dt_max = dt) with fixed-point tolerance 1e-8,
re-anchored every 10 steps at the state the segment starts from:

* FP64 and the anchored mixed run both keep dt (no restart), and agree to
  1e-9 of the peak density in max-norm and 1e-10 in every logged energy
  (measured 2.3e-11 and 1.5e-12);
* the mean split cannot hold the 1e-8 fixed point on this solid: its dt
  collapses by restarts or its density ends more than 100 times further
  from FP64 than the anchored one (measured: dt 3.3e-9, 6.7e-4).
"""
import math

import numpy as np
import pytest

import classicaldft_b200 as cd
from classicaldft_b200 import crystal as cc
from tests.parity import rel_err

pytestmark = pytest.mark.gpu

A, DX, ALPHA = 1.55, 0.0484375, 50.0


def test_anchored_ddft_of_a_solid_matches_fp64():
    n = 64
    lat = cc.build_lattice(cc.Structure.FCC, cc.Orientation._001, (2, 2, 2))
    sites = lat.scaled_positions(A / math.sqrt(2.0))
    grid = cd.Grid(dx=DX, box_size=(n * DX,) * 3, shape=(n,) * 3)
    rho0 = cc.gaussian_peaks(grid, sites, ALPHA, (ALPHA / math.pi) ** 1.5, 1e-8).cpu().numpy()
    model = cd.Model(grid, [cd.Species("hs", 1.0)], [], 1.0)
    w64 = cd.make_weights(cd.WhiteBearII(), model, cd.FP64)
    wmx = cd.make_weights(cd.WhiteBearII(), model, cd.MIXED)

    def sim(**kw):
        st = cd.StepConfig(dt=1e-7, dt_max=1e-7, fp_tolerance=1e-8, fp_max_iterations=200)
        return cd.Simulation(step=st, n_steps=100, snapshot_interval=50, log_interval=10, **kw)

    a = sim().run([rho0], w64, 0.0)
    b = sim(anchor=w64, anchor_interval=10).run([rho0], wmx, 0.0)
    m = sim().run([rho0], wmx, 0.0)
    assert a["steps"] == b["steps"] == 100
    assert a["dt"] == b["dt"] == 1e-7
    assert not wmx.engine.anchored  # cleared after the run
    peak = float(a["densities"][0].max())
    err_b = float(np.max(np.abs(a["densities"][0] - b["densities"][0])))
    assert err_b <= 1e-9 * peak
    assert len(a["energies"]) == len(b["energies"]) == 11
    for ea, eb in zip(a["energies"], b["energies"]):
        assert rel_err(eb, ea) <= 1e-10
    assert [s.step for s in b["snapshots"]] == [0, 50, 100]
    assert b["all_times"][-1] == pytest.approx(a["all_times"][-1], rel=1e-12)
    err_m = float(np.max(np.abs(a["densities"][0] - m["densities"][0])))
    assert m["dt"] < 1e-7 or err_m > 100.0 * err_b


def test_anchored_ddft_snapshot_interval_must_divide():
    grid = cd.Grid(dx=0.25, box_size=(4.0,) * 3, shape=(16,) * 3)
    model = cd.Model(grid, [cd.Species("hs", 1.0)], [], 1.0)
    w64 = cd.make_weights(cd.WhiteBearII(), model, cd.FP64)
    wmx = cd.make_weights(cd.WhiteBearII(), model, cd.MIXED)
    sim = cd.Simulation(n_steps=10, snapshot_interval=5, anchor=w64, anchor_interval=3)
    with pytest.raises(ValueError, match="multiple of anchor_interval"):
        sim.run([np.full(grid.total_points, 0.3)], wmx, 0.0)
