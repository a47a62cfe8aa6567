"""The free-energy functional F[rho] and dF/drho (oracle, test infrastructure only).

Restates include/dft/functionals/{hard_sphere,mean_field,ideal_gas,
external_field,functionals,functional}.hpp.  Densities, external fields and
forces are flat FP64 arrays of N = nx*ny*nz points (z fastest).  Forces are
dOmega/drho * dV, as in the reference (functionals.hpp:55-63).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from . import fmt as fmtm
from .grid import Grid, c2r, r2c
from .potentials import Interaction, generate_interaction_weight

PI = math.pi


@dataclass
class Species:
    """types.hpp:25-28."""

    name: str
    hard_sphere_diameter: float


@dataclass
class Model:
    """physics/model.hpp:15-20."""

    grid: Grid
    species: list
    interactions: list = field(default_factory=list)
    temperature: float = 1.0


@dataclass
class Weights:
    """functionals.hpp:19-23: FMT model + per-species FMT weights + MF weights."""

    fmt_model: fmtm.FMTModel
    fmt: list
    mean_field: list  # list of dicts {i, j, weight (k-space), a_vdw}


def make_weights(fmt_model: fmtm.FMTModel, model: Model) -> Weights:
    """functionals.hpp:27-33."""
    fw = [fmtm.generate_weights(sp.hard_sphere_diameter, model.grid) for sp in model.species]
    mf = []
    for inter in model.interactions:
        wk, a = generate_interaction_weight(inter, model.grid, model.temperature)
        mf.append({"i": inter.species_i, "j": inter.species_j, "weight": wk, "a_vdw": a})
    return Weights(fmt_model=fmt_model, fmt=fw, mean_field=mf)


def convolve(weight_k, rho_k, shape):
    """convolution.hpp:13-26: n = c2r(w .* rho_k) (1/N already inside w)."""
    return c2r(weight_k * rho_k, shape).reshape(-1)


def back_convolve(weight_k, derivative, shape, conjugate=False):
    """convolution.hpp:31-49: w .* r2c(d), conj(w) for parity-odd weights."""
    dk = r2c(np.asarray(derivative).reshape(shape))
    return (np.conj(weight_k) if conjugate else weight_k) * dk


def _convolve_weights(ws, rho_k, shape):
    """hard_sphere.hpp:50-67 (all 11 channels, as the reference does)."""
    wd = {
        "eta": convolve(ws["w3"], rho_k, shape),
        "n2": convolve(ws["w2"], rho_k, shape),
        "nv2": [convolve(ws["wv2"][a], rho_k, shape) for a in range(3)],
        "nT": {p: convolve(ws["wT"][p], rho_k, shape) for p in fmtm.TENSOR_PAIRS},
    }
    return wd


def _total_measures(wds, species):
    """hard_sphere.hpp:73-97 and :184-197: species-summed measures at every point."""
    n = wds[0]["eta"].shape[0]
    tot = {"eta": np.zeros(n), "n0": np.zeros(n), "n1": np.zeros(n), "n2": np.zeros(n),
           "v0": np.zeros((3, n)), "v1": np.zeros((3, n)), "T": np.zeros((3, 3, n))}
    for wd, sp in zip(wds, species):
        R = 0.5 * sp.hard_sphere_diameter
        four_pi_R = 4.0 * PI * R
        tot["eta"] += wd["eta"]
        tot["n2"] += wd["n2"]
        tot["n1"] += wd["n2"] / four_pi_R
        tot["n0"] += wd["n2"] / (four_pi_R * R)
        for a in range(3):
            tot["v1"][a] += wd["nv2"][a]
            tot["v0"][a] += wd["nv2"][a] / four_pi_R
        for (i, j) in fmtm.TENSOR_PAIRS:
            tot["T"][i, j] += wd["nT"][(i, j)]
            if i != j:
                tot["T"][j, i] += wd["nT"][(i, j)]
    return tot


def hard_sphere_measures(model: Model, rhos, weights: Weights):
    """Species-summed FMT measures (with inner products) for densities ``rhos``."""
    shape = model.grid.shape
    rho_k = [r2c(np.asarray(r, dtype=np.float64).reshape(shape)) for r in rhos]
    wds = [_convolve_weights(weights.fmt[s], rho_k[s], shape) for s in range(len(rhos))]
    m = _total_measures(wds, model.species)
    m["products"] = fmtm.inner_products(m)
    return m


def hard_sphere_pointwise(fmt_model, m):
    """hard_sphere.hpp:174-224: Phi and dPhi at every point, zero where eta < 1e-30."""
    skip = m["eta"] < 1e-30
    with np.errstate(all="ignore"):
        phi = fmt_model.phi(m)
        dm = fmt_model.d_phi(m)
    phi = np.where(skip, 0.0, phi)
    for key in ("d_eta", "d_n0", "d_n1", "d_n2"):
        dm[key] = np.where(skip, 0.0, dm[key])
    for key in ("d_v0", "d_v1", "d_T"):
        dm[key] = np.where(skip, 0.0, dm[key])
    return phi, dm, skip


def hard_sphere(model: Model, rhos, weights: Weights):
    """hard_sphere.hpp:263-298: (F_hs, [force_s])."""
    grid = model.grid
    shape = grid.shape
    dv = grid.cell_volume
    m = hard_sphere_measures(model, rhos, weights)
    phi, dm, _ = hard_sphere_pointwise(weights.fmt_model, m)
    free_energy = float(np.sum(phi) * dv)
    forces = []
    for s, sp in enumerate(model.species):           # :226-257
        R = 0.5 * sp.hard_sphere_diameter
        four_pi_R = 4.0 * PI * R
        ws = weights.fmt[s]
        fk = back_convolve(ws["w3"], dm["d_eta"], shape)
        fk = fk + back_convolve(ws["w2"], dm["d_n2"] + dm["d_n1"] / four_pi_R + dm["d_n0"] / (four_pi_R * R), shape)
        for a in range(3):
            fk = fk + back_convolve(ws["wv2"][a], dm["d_v1"][a] + dm["d_v0"][a] / four_pi_R, shape, True)
        for (i, j) in fmtm.TENSOR_PAIRS:
            sym = 1.0 if i == j else 2.0
            fk = fk + back_convolve(ws["wT"][(i, j)], sym * dm["d_T"][i, j], shape)
        forces.append(c2r(fk, shape).reshape(-1) * dv)
    return free_energy, forces


def mean_field(model: Model, rhos, weights: Weights):
    """mean_field.hpp:234-281: (F_mf, [force_s])."""
    grid = model.grid
    shape = grid.shape
    dv = grid.cell_volume
    n = grid.total_points
    rho_k = [r2c(np.asarray(r, dtype=np.float64).reshape(shape)) for r in rhos]
    forces = [np.zeros(n) for _ in rhos]
    F = 0.0
    for iw in weights.mean_field:
        i, j = iw["i"], iw["j"]
        conv_j = convolve(iw["weight"], rho_k[j], shape)
        if i == j:
            F += 0.5 * float(np.dot(rhos[i].reshape(-1), conv_j)) * dv
            forces[i] = forces[i] + conv_j * dv
        else:
            F += 0.5 * float(np.dot(rhos[i].reshape(-1), conv_j)) * dv
            forces[i] = forces[i] + 0.5 * conv_j * dv
            conv_i = convolve(iw["weight"], rho_k[i], shape)
            forces[j] = forces[j] + 0.5 * conv_i * dv
    return F, forces


def ideal_gas(model: Model, rhos, mus):
    """ideal_gas.hpp:18-37."""
    dv = model.grid.cell_volume
    F = 0.0
    forces = []
    for rho, mu in zip(rhos, mus):
        rho = np.asarray(rho, dtype=np.float64).reshape(-1)
        log_rho = np.log(np.clip(rho, 1e-300, np.inf))
        F += float(np.dot(rho, log_rho - 1.0)) * dv
        forces.append((log_rho - mu) * dv)
    return F, forces


def external_field(model: Model, rhos, vexts):
    """external_field.hpp:16-30."""
    dv = model.grid.cell_volume
    F = 0.0
    forces = []
    for rho, v in zip(rhos, vexts):
        rho = np.asarray(rho, dtype=np.float64).reshape(-1)
        v = np.zeros_like(rho) if v is None else np.asarray(v, dtype=np.float64).reshape(-1)
        F += float(np.dot(rho, v)) * dv
        forces.append(v * dv)
    return F, forces


@dataclass
class Result:
    """functionals/types.hpp:18-23."""

    free_energy: float
    grand_potential: float
    forces: list
    parts: dict = field(default_factory=dict)


def total(model: Model, rhos, weights: Weights, mus=None, vexts=None) -> Result:
    """functionals.hpp:64-95: F = F_id + F_ext + F_hs + F_mf, Omega = F - sum mu N."""
    S = len(rhos)
    rhos = [np.asarray(r, dtype=np.float64).reshape(-1) for r in rhos]
    mus = [0.0] * S if mus is None else list(mus)
    vexts = [None] * S if vexts is None else list(vexts)
    dv = model.grid.cell_volume
    n = model.grid.total_points
    forces = [np.zeros(n) for _ in range(S)]
    parts = {}
    F = 0.0
    for name, (Fc, fc) in (("ideal", ideal_gas(model, rhos, mus)),
                           ("external", external_field(model, rhos, vexts)),
                           ("hard_sphere", hard_sphere(model, rhos, weights))):
        parts[name] = Fc
        F += Fc
        forces = [a + b for a, b in zip(forces, fc)]
    if weights.mean_field:
        Fc, fc = mean_field(model, rhos, weights)
        parts["mean_field"] = Fc
        F += Fc
        forces = [a + b for a, b in zip(forces, fc)]
    muN = 0.0
    for rho, mu in zip(rhos, mus):
        muN += mu * float(np.sum(rho)) * dv
    return Result(free_energy=F, grand_potential=F - muN, forces=forces, parts=parts)


class Functional:
    """functional.hpp:22-107: model + weights with the evaluate / callback facade."""

    def __init__(self, fmt_model: fmtm.FMTModel, model: Model):
        self.model = model
        self.weights = make_weights(fmt_model, model)

    def evaluate(self, rho, chemical_potential=0.0) -> Result:
        """functional.hpp:33-36: single-species profile, V_ext dropped (init.hpp:28-44)."""
        S = len(self.model.species)
        rhos = [np.asarray(rho, dtype=np.float64).reshape(-1)]
        rhos += [np.zeros(self.model.grid.total_points) for _ in range(1, S)]
        mus = [chemical_potential] + [0.0] * (S - 1)
        return total(self.model, rhos, self.weights, mus)

    def grand_potential_callback(self, chemical_potential):
        """functional.hpp:62-73."""
        def fn(densities):
            r = total(self.model, densities, self.weights, [chemical_potential] * len(densities))
            return r.grand_potential, r.forces
        return fn
