"""Crystal density profiles on the GPU: the Gaussian-peak initialiser
(cdft_gaussian_peaks) against the oracle's direct sum, and the binary
hard-sphere FCC solid under esFMT (A=1, B=0): a = 1.55, dx = 0.0484375,
large spheres (d = 1) as Gaussian peaks (alpha = 50, 0.8 particles per site)
on build_lattice(FCC, 001) sites, small spheres (d = 0.5) uniform at 0.1.

Tolerances: the initialiser to 1e-13 of the peak height; the FP64 engine
against the oracle at 64^3 (2 x 2 x 2 cells) as every FP64 parity test,
|dF|/|F| <= 1e-12 and max|d force| <= 1e-11 max|force|; the mixed engine on
this strongly inhomogeneous state |dF|/|F| <= 1e-6, max|d force| <=
1e-4 max|force|, both against the oracle at 64^3 and against the FP64
engine at 256^3 (8 x 8 x 8 cells).
"""
import math

import numpy as np
import pytest

import classicaldft_b200 as cd
from classicaldft_b200 import crystal as cc
from oracle import crystal as oc
from tests.parity import Problem, force_err, rel_err

pytestmark = pytest.mark.gpu

A_FCC = 1.55
DX5 = 0.0484375
ALPHA = 50.0
OCC = 0.8


def test_gaussian_peaks_match_oracle():
    shape = (32, 24, 40)
    dx = 0.1
    box = np.array(shape) * dx
    lat = cc.build_lattice(cc.Structure.FCC, cc.Orientation._001, (2, 2, 3))
    sites = lat.scaled_positions(box) + 0.013  # off-grid sites, some past the box edge
    grid = cd.Grid(dx=dx, box_size=tuple(box), shape=shape)
    amp = (30.0 / math.pi) ** 1.5
    g = cc.gaussian_peaks(grid, sites, 30.0, amp, 0.02).cpu().numpy()
    o = oc.gaussian_peaks(shape, dx, sites, 30.0, amp, 0.02)
    assert np.max(np.abs(g - o)) <= 1e-13 * amp
    # one particle per site (the sum is spectrally accurate on a periodic grid)
    assert (float(np.sum(g - 0.02)) * dx ** 3) == pytest.approx(len(sites), rel=1e-9)


def test_gaussian_peaks_rejects_small_box():
    grid = cd.Grid(dx=0.1, box_size=(0.8, 3.2, 3.2), shape=(8, 32, 32))
    with pytest.raises(ValueError, match="twice the cut radius"):
        cc.gaussian_peaks(grid, np.zeros((1, 3)), 30.0)


def fcc_solid(cells):
    n = int(round(cells * A_FCC / DX5))
    shape = (n, n, n)
    lat = cc.build_lattice(cc.Structure.FCC, cc.Orientation._001, (cells,) * 3)
    sites = lat.scaled_positions(A_FCC / math.sqrt(2.0))  # unit nearest-neighbour distance -> a / sqrt(2)
    grid = cd.Grid(dx=DX5, box_size=(n * DX5,) * 3, shape=shape)
    rho1 = cc.gaussian_peaks(grid, sites, ALPHA, OCC * (ALPHA / math.pi) ** 1.5, 0.0)
    rho2 = np.full(grid.total_points, 0.1)
    return shape, rho1, rho2


def test_fcc_solid_64_matches_oracle():
    shape, rho1, rho2 = fcc_solid(2)
    assert shape == (64, 64, 64)
    r1 = rho1.cpu().numpy()
    ref = None
    for precision, f_tol, force_tol in ((cd.FP64, 1e-12, 1e-11), (cd.MIXED, 1e-6, 1e-4)):
        pr = Problem(shape, DX5, [1.0, 0.5], "esFMT", A=1.0, B=0.0, precision=precision)
        if ref is None:
            ref = pr.ref([r1, rho2], [0.0, 0.0])
        g = pr.gpu([r1, rho2], [0.0, 0.0])
        assert rel_err(g.free_energy, ref.free_energy) <= f_tol
        assert force_err(g.forces, ref.forces) <= force_tol


def test_fcc_solid_256_mixed_vs_fp64():
    shape, rho1, rho2 = fcc_solid(8)
    assert shape == (256, 256, 256)
    r1 = rho1.cpu().numpy()
    del rho1
    grid = cd.Grid(dx=DX5, box_size=(256 * DX5,) * 3, shape=shape)
    model = cd.Model(grid, [cd.Species("large", 1.0), cd.Species("small", 0.5)], [], 1.0)
    fmt = cd.FMTModel("esFMT", 1.0, 0.0)
    out = {}
    for name, precision in (("fp64", cd.FP64), ("mixed", cd.MIXED)):
        w = cd.make_weights(fmt, model, precision)
        out[name] = cd.total(model, [r1, rho2], w, [0.0, 0.0])
        del w
    f64, fmx = out["fp64"], out["mixed"]
    e = rel_err(fmx.free_energy, f64.free_energy)
    fe = force_err(fmx.forces, f64.forces)
    print(f"256^3 FCC binary esFMT: mixed vs FP64 |dF/F| = {e:.3e}, force error = {fe:.3e}")
    assert math.isfinite(f64.free_energy)
    assert e <= 1e-6
    assert fe <= 1e-4
