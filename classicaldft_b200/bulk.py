"""Bulk (uniform-fluid) thermodynamics and the phase search, mirroring
include/dft/functionals/bulk/{thermodynamics,coexistence}.hpp.

Every quantity is computed by the engine library (``cdft_bulk_*``), which
evaluates the same FMT Phi as the GPU kernels at the uniform measures.
Typical use, as in the reference:

    eos = make_bulk_thermodynamics(model.species, weights)   # grid a_vdw
    coex = PhaseSearch(rho_max=1.0, rho_scan_step=0.005).find_coexistence(eos)
    rho_l = density_from_chemical_potential(mu, 0.7, eos)
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from . import _lib
from .functionals import FMTModel, Interaction, Species, Weights, WEEKS_CHANDLER_ANDERSEN


@dataclass
class BulkInteraction:
    """thermodynamics.hpp:187-191."""

    species_i: int
    species_j: int
    a_vdw: float


@dataclass
class BulkThermodynamics:
    """thermodynamics.hpp:201-254: the equation of state of the uniform fluid."""

    species: list
    fmt_model: FMTModel
    interactions: list = field(default_factory=list)

    def _c(self):
        m = _lib.CBulkModel()
        m.n_species = len(self.species)
        if not 1 <= m.n_species <= 4:
            raise ValueError("BulkThermodynamics: 1 to 4 species")
        for s, sp in enumerate(self.species):
            m.diameters[s] = sp.hard_sphere_diameter
        m.fmt_model = _lib.MODEL_IDS[self.fmt_model.name]
        m.esfmt_A, m.esfmt_B = self.fmt_model.A, self.fmt_model.B
        m.n_interactions = len(self.interactions)
        if m.n_interactions > 8:
            raise ValueError("BulkThermodynamics: at most 8 interactions")
        for k, it in enumerate(self.interactions):
            m.interactions[k] = _lib.CBulkInteraction(it.species_i, it.species_j, it.a_vdw)
        return m

    def _rho(self, rho):
        r = np.ascontiguousarray(np.atleast_1d(np.asarray(rho, dtype=np.float64)))
        if r.size != len(self.species):
            raise ValueError(f"expected {len(self.species)} densities")
        return r

    def free_energy_density(self, rho) -> float:
        r = self._rho(rho)
        f = ctypes.c_double()
        _lib.check(_lib.lib().cdft_bulk_free_energy_density(ctypes.byref(self._c()), r.ctypes.data_as(_lib.c_double_p),
                                                            ctypes.byref(f)))
        return f.value

    def chemical_potentials(self, rho) -> np.ndarray:
        r = self._rho(rho)
        mu = np.empty(r.size)
        _lib.check(_lib.lib().cdft_bulk_chemical_potentials(ctypes.byref(self._c()), r.ctypes.data_as(_lib.c_double_p),
                                                            mu.ctypes.data_as(_lib.c_double_p)))
        return mu

    def chemical_potential(self, rho, species_idx: int = 0) -> float:
        return float(self.chemical_potentials(rho)[species_idx])

    def pressure(self, rho) -> float:
        r = self._rho(rho)
        p = ctypes.c_double()
        _lib.check(_lib.lib().cdft_bulk_pressure(ctypes.byref(self._c()), r.ctypes.data_as(_lib.c_double_p),
                                                 ctypes.byref(p)))
        return p.value

    def grand_potential_density(self, rho) -> float:
        return -self.pressure(rho)


def make_bulk_thermodynamics(species, weights: Weights) -> BulkThermodynamics:
    """thermodynamics.hpp:258-271 from GPU Weights: the grid a_vdw of the
    mean-field weights (Functional::bulk(), functional.hpp:48-50)."""
    m = _lib.CBulkModel()
    _lib.check(_lib.lib().cdft_engine_bulk_model(weights.engine.handle, ctypes.byref(m)))
    inters = [BulkInteraction(m.interactions[k].species_i, m.interactions[k].species_j, m.interactions[k].a_vdw)
              for k in range(m.n_interactions)]
    return BulkThermodynamics(list(species), weights.fmt_model, inters)


def make_bulk_weights(fmt_model: FMTModel, interactions, kT: float) -> list:
    """functionals.hpp:38-53: the continuum a_vdw = 2 vdw_integral of each interaction."""
    out = []
    for it in interactions:
        split = getattr(it, "split", WEEKS_CHANDLER_ANDERSEN)
        out.append(BulkInteraction(it.species_i, it.species_j, 2.0 * it.potential.vdw_integral(kT, split)))
    return out


def bulk_thermodynamics(species, fmt_model: FMTModel, interactions, kT: float) -> BulkThermodynamics:
    """make_bulk_thermodynamics(species, make_bulk_weights(fmt_model, interactions, kT))."""
    return BulkThermodynamics(list(species), fmt_model, make_bulk_weights(fmt_model, interactions, kT))


@dataclass
class Newton:
    """solvers/newton.hpp:34-38 (the settings PhaseSearch uses)."""

    max_iterations: int = 200
    tolerance: float = 1e-10


@dataclass
class Spinodal:
    rho_low: float
    rho_high: float


@dataclass
class Coexistence:
    rho_vapor: float
    rho_liquid: float


def density_from_chemical_potential(target_mu: float, initial_guess: float, eos: BulkThermodynamics,
                                    solver: Newton = None) -> Optional[float]:
    """coexistence.hpp:35-49: None where Newton fails or ends at rho <= 0."""
    r = densities_from_chemical_potentials([target_mu], [initial_guess], eos, solver)
    return None if np.isnan(r[0]) else float(r[0])


def densities_from_chemical_potentials(mus, guesses, eos: BulkThermodynamics, solver: Newton = None) -> np.ndarray:
    """density_from_chemical_potential over a grid of targets (NaN where it fails)."""
    solver = solver or Newton()
    mu = np.ascontiguousarray(np.atleast_1d(np.asarray(mus, dtype=np.float64)))
    g = np.ascontiguousarray(np.broadcast_to(np.asarray(guesses, dtype=np.float64), mu.shape))
    rho = np.empty(mu.size)
    found = (ctypes.c_int * max(1, mu.size))()
    _lib.check(_lib.lib().cdft_bulk_density_from_mu(
        ctypes.byref(eos._c()), mu.size, mu.ctypes.data_as(_lib.c_double_p), g.ctypes.data_as(_lib.c_double_p),
        solver.max_iterations, solver.tolerance, rho.ctypes.data_as(_lib.c_double_p), found))
    rho[[not found[i] for i in range(mu.size)]] = np.nan
    return rho


@dataclass
class PhaseSearch:
    """coexistence.hpp:25-33."""

    rho_max: float = 1.0
    rho_scan_step: float = 0.01
    newton: Newton = field(default_factory=Newton)

    def find_spinodal(self, eos: BulkThermodynamics) -> Optional[Spinodal]:
        out = (ctypes.c_double * 2)()
        found = ctypes.c_int()
        _lib.check(_lib.lib().cdft_bulk_spinodal(ctypes.byref(eos._c()), self.rho_max, self.rho_scan_step, out,
                                                 ctypes.byref(found)))
        return Spinodal(out[0], out[1]) if found.value else None

    def find_coexistence(self, eos: BulkThermodynamics) -> Optional[Coexistence]:
        out = (ctypes.c_double * 2)()
        found = ctypes.c_int()
        _lib.check(_lib.lib().cdft_bulk_coexistence(ctypes.byref(eos._c()), self.rho_max, self.rho_scan_step,
                                                    self.newton.max_iterations, self.newton.tolerance, out,
                                                    ctypes.byref(found)))
        return Coexistence(out[0], out[1]) if found.value else None


__all__ = ["BulkInteraction", "BulkThermodynamics", "make_bulk_thermodynamics", "make_bulk_weights",
           "bulk_thermodynamics", "Newton", "Spinodal", "Coexistence", "density_from_chemical_potential",
           "densities_from_chemical_potentials", "PhaseSearch", "Species", "Interaction"]
