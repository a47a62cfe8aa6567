"""Helpers shared by the parity tests: build the same problem for the GPU
engine (the product) and for the oracle (the checker)."""
from __future__ import annotations

import numpy as np

import classicaldft_b200 as cd
from oracle import fmt as ofmt
from oracle import potentials as opot
from oracle.functional import Model as OModel
from oracle.functional import Species as OSpecies
from oracle.functional import make_weights as o_make_weights
from oracle.functional import total as o_total
from oracle.grid import Grid as OGrid

_SPLIT = {cd.WEEKS_CHANDLER_ANDERSEN: opot.WCA, cd.BARKER_HENDERSON: opot.BH}


class Problem:
    """One functional (grid, species, FMT model, LJ interactions) built twice."""

    def __init__(self, shape, dx, diameters, model="WhiteBearII", A=1.0, B=0.0, inters=(), kT=1.0,
                 precision=cd.FP64, scheme="InterpolationQuadraticF"):
        box = tuple(n * dx for n in shape)
        self.grid = cd.Grid(dx=dx, box_size=box, shape=tuple(shape))
        self.N = self.grid.total_points
        self.S = len(diameters)
        species = [cd.Species(f"S{i}", d) for i, d in enumerate(diameters)]
        ci = [cd.Interaction(i, j, cd.make_lennard_jones(s, e, rc), cd.WEEKS_CHANDLER_ANDERSEN, scheme)
              for (i, j, s, e, rc) in inters]
        self.model = cd.Model(self.grid, species, ci, kT)
        self.fmt = cd.FMTModel(model, A, B)
        self.weights = cd.make_weights(self.fmt, self.model, precision)
        og = OGrid(dx=dx, box_size=box, shape=tuple(shape))
        oi = [opot.Interaction(i, j, opot.make_lennard_jones(s, e, rc), opot.WCA, scheme)
              for (i, j, s, e, rc) in inters]
        self.omodel = OModel(og, [OSpecies(f"S{i}", d) for i, d in enumerate(diameters)], oi, kT)
        self.oweights = o_make_weights(ofmt.FMTModel(model, A, B), self.omodel)

    def gpu(self, rhos, mus=None, vexts=None):
        return cd.total(self.model, rhos, self.weights, mus, vexts)

    def ref(self, rhos, mus=None, vexts=None):
        return o_total(self.omodel, list(rhos), self.oweights, mus, vexts)


def smooth_noise(shape, rng, width_cells=2.0):
    """Unit-variance white noise smoothed by a Gaussian of the given width (cells)."""
    w = rng.standard_normal(shape)
    k = [np.fft.fftfreq(n) for n in shape]
    K2 = k[0][:, None, None] ** 2 + k[1][None, :, None] ** 2 + k[2][None, None, :] ** 2
    g = np.exp(-2.0 * (np.pi * width_cells) ** 2 * K2)
    f = np.real(np.fft.ifftn(np.fft.fftn(w) * g))
    return (f / f.std()).reshape(-1)


def rel_err(a, b):
    return abs(a - b) / max(abs(b), 1e-300)


def force_err(fa, fb):
    """max |fa - fb| / max |fb| over all species."""
    num = max(float(np.max(np.abs(np.asarray(x) - np.asarray(y)))) for x, y in zip(fa, fb))
    den = max(float(np.max(np.abs(np.asarray(y)))) for y in fb)
    return num / max(den, 1e-300)
