"""Bulk (uniform-fluid) thermodynamics and phase search (oracle, test
infrastructure only).

Restates include/dft/functionals/bulk/thermodynamics.hpp:14-273 (ideal,
hard-sphere and mean-field free energy density, chemical potentials,
pressure), functionals.hpp:38-53 (make_bulk_weights: a_vdw = 2 x the vdW
integral), bulk/coexistence.hpp:13-195 (PhaseSearch: spinodal scan with
central-difference dP/drho and bisection, coexistence by bracketing
P_v - P_l along the vapour branch with Newton inversion of mu(rho)) and the
1-D use of algorithms/solvers/newton.hpp:34-70 with the central-difference
Jacobian of solvers/jacobian.hpp:17-40.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from .fmt import PI, FMTModel, make_uniform_measures, inner_products
from . import potentials as opot


@dataclass
class BulkInteraction:
    species_i: int
    species_j: int
    a_vdw: float


@dataclass
class BulkThermodynamics:
    """thermodynamics.hpp:201-254."""

    diameters: list
    fmt_model: FMTModel
    interactions: list = field(default_factory=list)

    def _measures(self, rho):
        tot = None
        for r, d in zip(rho, self.diameters):
            m = make_uniform_measures(float(r), d)
            if tot is None:
                tot = {k: (np.array(v, dtype=np.float64) if k != "products" else None) for k, v in m.items()}
            else:
                for k in ("eta", "n0", "n1", "n2", "T"):
                    tot[k] = tot[k] + m[k]
        tot["products"] = inner_products(tot)
        return tot

    def hard_sphere_free_energy_density(self, rho):
        """thermodynamics.hpp:37-53."""
        return float(self.fmt_model.phi(self._measures(rho)))

    def hard_sphere_excess_mu(self, rho, s):
        """thermodynamics.hpp:55-92."""
        dm = self.fmt_model.d_phi(self._measures(rho))
        d = self.diameters[s]
        r = 0.5 * d
        mu = (float(dm["d_eta"]) * (PI / 6.0) * d * d * d + float(dm["d_n2"]) * PI * d * d
              + float(dm["d_n1"]) * r + float(dm["d_n0"]))
        if self.fmt_model.needs_tensor:
            dt = PI * d * d / 3.0
            for j in range(3):
                mu += float(dm["d_T"][j, j]) * dt
        return mu

    def free_energy_density(self, rho):
        rho = np.atleast_1d(np.asarray(rho, dtype=np.float64))
        f = 0.0
        for r in rho:  # ideal (thermodynamics.hpp:19-27)
            if r > 0.0:
                f += r * (math.log(r) - 1.0)
        f += self.hard_sphere_free_energy_density(rho)
        for it in self.interactions:
            i, j = it.species_i, it.species_j
            f += (0.5 if i == j else 1.0) * it.a_vdw * rho[i] * rho[j]
        return f

    def chemical_potential(self, rho, s):
        rho = np.atleast_1d(np.asarray(rho, dtype=np.float64))
        mu = math.log(rho[s]) if rho[s] > 0.0 else (-math.inf if rho[s] == 0.0 else math.nan)
        mu += self.hard_sphere_excess_mu(rho, s)
        for it in self.interactions:
            i, j = it.species_i, it.species_j
            if i == s and j == s:
                mu += it.a_vdw * rho[j]
            elif i == s:
                mu += 0.5 * it.a_vdw * rho[j]
            elif j == s:
                mu += 0.5 * it.a_vdw * rho[i]
        return mu

    def chemical_potentials(self, rho):
        rho = np.atleast_1d(np.asarray(rho, dtype=np.float64))
        return np.array([self.chemical_potential(rho, s) for s in range(rho.size)])

    def pressure(self, rho):
        rho = np.atleast_1d(np.asarray(rho, dtype=np.float64))
        p = -self.free_energy_density(rho)
        for s in range(rho.size):
            p += rho[s] * self.chemical_potential(rho, s)
        return p

    def grand_potential_density(self, rho):
        return -self.pressure(rho)


def make_bulk_thermodynamics(diameters, fmt_model, interactions, kT):
    """functionals.hpp:38-53 + thermodynamics.hpp:258-271: a_vdw = 2 vdw_integral."""
    inters = [BulkInteraction(it.species_i, it.species_j, 2.0 * opot.vdw_integral(it.potential, kT, it.split))
              for it in interactions]
    return BulkThermodynamics(list(diameters), fmt_model, inters)


# ------------------------------------------------------------ phase search


def newton_1d(x, f, max_iterations=200, tolerance=1e-10, eps=1e-7):
    """newton.hpp:38-70 in one dimension with jacobian.hpp:17-40."""
    for k in range(max_iterations):
        fk = f(x)
        if abs(fk) < tolerance:
            return x, k, abs(fk), True
        J = (f(x + eps) - f(x - eps)) / (2.0 * eps)
        if not (J != 0.0) or not math.isfinite(J):
            return x, k, abs(fk), False
        x = x - fk / J
    fn = abs(f(x))
    return x, max_iterations, fn, fn < tolerance


def density_from_chemical_potential(target_mu, initial_guess, eos, max_iterations=200, tolerance=1e-10):
    """coexistence.hpp:35-49."""
    x, _, _, ok = newton_1d(initial_guess, lambda r: eos.chemical_potential([r], 0) - target_mu,
                            max_iterations, tolerance)
    if not ok or not (x > 0.0):
        return None
    return x


def dp_drho(rho, eos, h=1e-7):
    """coexistence.hpp:53-57."""
    return (eos.pressure([rho + h]) - eos.pressure([rho - h])) / (2.0 * h)


def bisect_dp_drho(lo, hi, eos):
    """coexistence.hpp:59-73."""
    f_lo = dp_drho(lo, eos)
    for _ in range(60):
        mid = 0.5 * (lo + hi)
        f_mid = dp_drho(mid, eos)
        if (f_lo > 0.0) == (f_mid > 0.0):
            lo, f_lo = mid, f_mid
        else:
            hi = mid
    return 0.5 * (lo + hi)


@dataclass
class PhaseSearch:
    """coexistence.hpp:25-33."""

    rho_max: float = 1.0
    rho_scan_step: float = 0.01
    newton_max_iterations: int = 200
    newton_tolerance: float = 1e-10

    def find_spinodal(self, eos):
        """coexistence.hpp:77-113: (rho_low, rho_high) or None."""
        step = self.rho_scan_step
        prev_dp = dp_drho(step, eos)
        found_low = found_high = False
        low = high = (0.0, 0.0)
        prev_rho = step
        rho = 2.0 * step
        while rho < self.rho_max:
            curr = dp_drho(rho, eos)
            if prev_dp > 0.0 and curr <= 0.0 and not found_low:
                low, found_low = (prev_rho, rho), True
            elif prev_dp < 0.0 and curr >= 0.0 and found_low:
                high, found_high = (prev_rho, rho), True
                break
            prev_dp = curr
            prev_rho = rho
            rho += step
        if not (found_low and found_high):
            return None
        return bisect_dp_drho(*low, eos), bisect_dp_drho(*high, eos)

    def find_coexistence(self, eos):
        """coexistence.hpp:115-191: (rho_vapor, rho_liquid) or None."""
        sp = self.find_spinodal(eos)
        if sp is None:
            return None
        rs1, rs2 = sp

        def liquid(rv):
            mu_v = eos.chemical_potential([rv], 0)
            return density_from_chemical_potential(mu_v, rs2 * 1.2, eos, self.newton_max_iterations,
                                                   self.newton_tolerance)

        def delta_p(rv):
            rl = liquid(rv)
            if rl is None or rl <= rs2:
                return None
            return eos.pressure([rv]) - eos.pressure([rl])

        rho_v = rs1
        dp_prev = delta_p(rho_v)
        if dp_prev is None:
            return None
        bracketed = False
        lo = hi = rho_v
        while rho_v > 1e-12:
            rho_v /= 1.1
            dp = delta_p(rho_v)
            if dp is None:
                continue
            if (dp < 0.0) != (dp_prev < 0.0):
                lo, hi = rho_v, rho_v * 1.1
                bracketed = True
                break
            dp_prev = dp
        if not bracketed:
            return None
        dp_lo = delta_p(lo)
        if dp_lo is None:
            return None
        for _ in range(60):
            mid = 0.5 * (lo + hi)
            dp_mid = delta_p(mid)
            if dp_mid is None:
                hi = mid
                continue
            if (dp_lo > 0.0) == (dp_mid > 0.0):
                lo, dp_lo = mid, dp_mid
            else:
                hi = mid
        rv = 0.5 * (lo + hi)
        rl = liquid(rv)
        if rl is None:
            return None
        return rv, rl
