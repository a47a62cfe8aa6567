"""Uneven-size batching: several batched engines (one per grid size)
minimised together, one graph launch per FIRE step for all of them.

* 3 problems each on 16^3, 24^3 and 32^3 grids (WBII + cut LJ, grand
  potential, different mu): every problem's converged profile equals its
  single-problem minimisation to 1e-10 in max-norm (the bar is 1e-8), Omega
  to 1e-12, and the iteration counts are the same;
* the group with step graphs equals the group launched kernel by kernel, bit
  for bit, and equals each member minimised on its own (batched), bit for bit;
* mixed precision with FP64 refinement per member matches FP64 to 1e-8;
* the uneven sweep driver (cost partition, grouping by grid) on one GPU
  reproduces the single-problem results.
"""
import numpy as np
import pytest

import classicaldft_b200 as cd
from classicaldft_b200.sweep import SweepProblem, run_uneven_sweep
from tests.parity import Problem, smooth_noise

pytestmark = pytest.mark.gpu
SIZES = (16, 24, 32)
PER = 3
FIRE = dict(dt=0.05, dt_max=0.5, alpha_start=0.01, f_alpha=0.99, force_tolerance=1e-10, max_steps=6000)


def setup(precision=cd.FP64):
    rng = np.random.default_rng(12)
    out = []
    for n in SIZES:
        pr = Problem((n,) * 3, 0.25, [1.0], "WhiteBearII", inters=[(0, 0, 1.0, 1.0, 1.8)], kT=1.0,
                     precision=precision)
        rhos = np.stack([0.4 * (1.0 + 0.05 * smooth_noise((n,) * 3, rng)) for _ in range(PER)])
        mus = np.linspace(0.5, 1.5, PER) + 0.1 * SIZES.index(n)
        out.append((pr, rhos, mus))
    return out


def group(mz, probs, precision=cd.FP64, refine=False):
    members = []
    for pr, rhos, mus in probs:
        w = cd.make_weights(pr.fmt, pr.model, precision, batch=PER)
        r = cd.make_weights(pr.fmt, pr.model, cd.FP64, batch=PER) if refine else None
        members.append((w, rhos, mus, None, r))
    return mz.minimize_group(members)


def test_group_matches_single_problem_runs():
    probs = setup()
    mz = cd.Minimizer(fire=cd.Fire(**FIRE))
    res = group(mz, probs)
    for (pr, rhos, mus), rs in zip(probs, res):
        for b in range(PER):
            one = mz.grand_potential(pr.model, pr.weights, rhos[b], mus[b])
            assert rs[b].converged and one.converged
            assert rs[b].iterations == one.iterations
            assert np.max(np.abs(rs[b].densities[0] - one.densities[0])) <= 1e-10
            assert rs[b].grand_potential == pytest.approx(one.grand_potential, rel=1e-12)


def test_group_graphs_and_members_alone_are_bitwise_equal():
    probs = setup()
    mz = cd.Minimizer(fire=cd.Fire(**FIRE))
    try:
        cd.set_step_graphs(False)
        direct = group(mz, probs)
    finally:
        cd.set_step_graphs(True)
    graphed = group(mz, probs)
    for (pr, rhos, mus), a, b in zip(probs, graphed, direct):
        w = cd.make_weights(pr.fmt, pr.model, cd.FP64, batch=PER)
        alone = mz.grand_potential_batch(pr.model, w, rhos, mus)
        for k in range(PER):
            assert np.array_equal(a[k].densities[0], b[k].densities[0])
            assert np.array_equal(a[k].densities[0], alone[k].densities[0])
            assert a[k].iterations == b[k].iterations == alone[k].iterations
            assert a[k].grand_potential == alone[k].grand_potential


def test_mixed_group_with_refinement_matches_fp64():
    probs = setup()
    probs_m = setup(cd.MIXED)
    # the rms-force convergence test (the energy monitor leaves soft modes
    # unresolved at the 1e-8 level)
    tight = dict(FIRE, force_tolerance=1e-12, max_steps=20000)
    f64 = group(cd.Minimizer(fire=cd.Fire(**tight), use_monitor=False), probs)
    mix = group(cd.Minimizer(fire=cd.Fire(**tight), refine_switch=1e3, use_monitor=False), probs_m,
                precision=cd.MIXED, refine=True)
    for a, b in zip(f64, mix):
        for k in range(PER):
            assert a[k].converged and b[k].converged
            assert np.max(np.abs(a[k].densities[0] - b[k].densities[0])) <= 1e-8
            assert b[k].grand_potential == pytest.approx(a[k].grand_potential, rel=1e-10)


def test_uneven_sweep_on_one_gpu():
    probs = setup()
    mz = cd.Minimizer(fire=cd.Fire(**FIRE))
    problems = [SweepProblem(pr.model, float(mus[b]), rhos[b]) for pr, rhos, mus in probs for b in range(PER)]
    res = run_uneven_sweep(problems, cd.WhiteBearII(), mz, gather_profiles=True)
    k = 0
    for pr, rhos, mus in probs:
        for b in range(PER):
            one = mz.grand_potential(pr.model, pr.weights, rhos[b], mus[b])
            assert res.converged[k]
            assert res.grand_potential[k] == pytest.approx(one.grand_potential, rel=1e-12)
            assert np.max(np.abs(res.profiles[k] - one.densities[0])) <= 1e-10
            k += 1
