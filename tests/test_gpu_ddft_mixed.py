"""Integrating-factor DDFT on the device: the fixed-point loop as a
conditional graph node, and mixed precision with FP64 defect correction.

* With step graphs on, every step's fixed-point loop runs on the device (the
  conditional WHILE node of the step's graph) and gives bit-identical
  densities, energies and time steps to the host-driven loop.
* The mixed-precision run with the FP64 refine engine (two FP64 fixed-point
  iterations after convergence, FP64 final energy) against the FP64 run,
  200 steps at 32^3 (dt = 1e-3, fixed): max |drho| <= 1e-9 and
  |dF|/|F| <= 1e-13 at every snapshot; without refinement |dF|/|F| stays
  within 1e-11.
* The refined mixed steps against the oracle's integrating_factor_step
  (dynamics.hpp:333-401) at steps 1 and 10: max |drho| <= 1e-9, energy to
  1e-12 relative.
"""
import numpy as np
import pytest

import classicaldft_b200 as cd
from oracle import algorithms as oalg
from tests.parity import Problem

pytestmark = pytest.mark.gpu
SHAPE, DX = (32, 32, 32), 0.2


def problems():
    kw = dict(inters=[(0, 0, 1.0, 1.0, 2.5)], kT=0.8)
    return (Problem(SHAPE, DX, [1.0], "WhiteBearII", precision=cd.FP64, **kw),
            Problem(SHAPE, DX, [1.0], "WhiteBearII", precision=cd.MIXED, **kw))


def start_density(seed=7):
    rng = np.random.default_rng(seed)
    return 0.35 * (1.0 + 0.01 * rng.uniform(-1.0, 1.0, int(np.prod(SHAPE))))


def test_device_loop_matches_the_host_loop():
    pr64, _ = problems()
    rho0 = start_density()
    out = {}
    try:
        for on in (True, False):
            cd.set_step_graphs(on)
            cfg = cd.StepConfig(dt=2e-2, fp_tolerance=1e-8)  # large enough to restart
            r, trace = rho0.copy(), []
            for _ in range(6):
                r, e, dt = cd.integrating_factor_step(r, pr64.weights, cfg, 0.0)
                info = cd.ddft_last_step(pr64.weights)
                assert info["device_loop"] == on and info["status"] == 1
                trace.append((e, dt, info["fp_iterations"], info["restarts"]))
            out[on] = (r, trace)
    finally:
        cd.set_step_graphs(True)
    assert np.array_equal(out[True][0], out[False][0])
    assert out[True][1] == out[False][1]


@pytest.mark.parametrize("shape", [(64, 64, 64), (128, 64, 64)])
def test_device_loop_with_forked_plane_chunks(shape):
    """A mixed-precision engine whose evaluation forks its middle stages onto
    four plane-chunk streams: the step graph (each part captured on its own
    and embedded as a child graph of the conditional loop) matches the host
    loop bit for bit, with refinement by an FP64 engine."""
    kw = dict(inters=[(0, 0, 1.0, 1.0, 2.5)], kT=0.8)
    prm = Problem(shape, 0.125, [1.0], "WhiteBearII", precision=cd.MIXED, **kw)
    pr64 = Problem(shape, 0.125, [1.0], "WhiteBearII", precision=cd.FP64, **kw)
    assert prm.weights.engine.info["kernels_per_eval"] == 16  # four chunks
    rng = np.random.default_rng(3)
    rho0 = 0.35 * (1.0 + 0.01 * rng.uniform(-1.0, 1.0, int(np.prod(shape))))
    out = {}
    try:
        for on in (True, False):
            cd.set_step_graphs(on)
            cfg = cd.StepConfig(dt=1e-4, fp_tolerance=1e-8)
            r = rho0.copy()
            for _ in range(3):
                r, e, dt = cd.integrating_factor_step(r, prm.weights, cfg, 0.0, refine=pr64.weights)
                assert cd.ddft_last_step(prm.weights)["device_loop"] == on
            out[on] = (r, e, dt)
    finally:
        cd.set_step_graphs(True)
    assert np.array_equal(out[True][0], out[False][0])
    assert out[True][1:] == out[False][1:]


def test_mixed_with_fp64_refinement_tracks_fp64():
    pr64, prm = problems()
    rho0 = start_density()
    runs = {}
    for label, w, ref in (("fp64", pr64.weights, None), ("mixed", prm.weights, None),
                          ("refined", prm.weights, pr64.weights)):
        sim = cd.Simulation(step=cd.StepConfig(dt=1e-3, dt_max=1e-3, fp_tolerance=1e-9), n_steps=200,
                            snapshot_interval=50, log_interval=50, refine=ref)
        runs[label] = sim.run([rho0], w, 0.0)
    assert cd.ddft_last_step(prm.weights)["refine_deviation"] < 1e-9
    for label, f_tol in (("mixed", 1e-11), ("refined", 1e-13)):
        for a, b in zip(runs["fp64"]["snapshots"], runs[label]["snapshots"]):
            assert a.step == b.step
            assert np.max(np.abs(a.densities[0] - b.densities[0])) <= 1e-9, (label, a.step)
            assert abs(a.energy - b.energy) <= f_tol * abs(a.energy), (label, a.step)


def test_refined_mixed_steps_match_the_oracle():
    pr64, prm = problems()
    rho = start_density(11)
    cfg_g = cd.StepConfig(dt=1e-3, fp_tolerance=1e-10)
    cfg_o = oalg.StepConfig(dt=1e-3, fp_tolerance=1e-10)
    st = oalg.IFState(pr64.omodel.grid)

    def ofn(dens):
        r = pr64.ref(dens, [0.0])
        return r.grand_potential, r.forces
    rg, ro = rho.copy(), [rho.copy()]
    for step in range(1, 11):
        rg, eg, dtg = cd.integrating_factor_step(rg, prm.weights, cfg_g, 0.0, refine=pr64.weights)
        ro, eo, dto = oalg.integrating_factor_step(ro, pr64.omodel.grid, st, ofn, cfg_o)
        if step in (1, 10):
            assert dtg == dto
            assert np.max(np.abs(rg - ro[0])) <= 1e-9, step
            assert eg == pytest.approx(eo, rel=1e-12), step
