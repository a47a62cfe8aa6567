"""Pair potentials and mean-field interaction weights (oracle, test infrastructure only).

Restates include/dft/physics/potentials.hpp (LJ, tWF, WRDF, WCA/BH split,
hard-sphere diameter, van der Waals integral) and the real-space cell
weights of include/dft/functionals/mean_field.hpp:42-196.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np
from scipy import integrate

from .grid import Grid, r2c

WCA = "WeeksChandlerAndersen"
BH = "BarkerHenderson"
MAX_POTENTIAL_VALUE = 1e50


@dataclass
class LennardJones:
    """potentials.hpp:57-116, built by make_lennard_jones (:311-325)."""

    sigma: float = 1.0
    epsilon: float = 1.0
    r_cutoff: float = -1.0
    epsilon_shift: float = 0.0
    r_min: float = 0.0
    v_min: float = 0.0
    r_zero: float = 0.0
    name: str = "LennardJones"

    def raw(self, r):
        with np.errstate(divide="ignore", invalid="ignore", over="ignore"):
            y = self.sigma / np.asarray(r, dtype=np.float64)
            y6 = y * y * y * y * y * y
            return 4.0 * self.epsilon * (y6 * y6 - y6)

    def hard_core_diameter(self):
        return 0.0

    def split_point(self, scheme):
        return self.r_zero if scheme == BH else self.r_min

    def repulsive(self, r, scheme):
        r = np.asarray(r, dtype=np.float64)
        v = self.raw(r) - self.epsilon_shift
        if scheme == BH:
            return np.where(r < self.r_zero, v, 0.0)
        return np.where(r < self.r_min, v - self.v_min, 0.0)

    def attractive(self, r, scheme):
        r = np.asarray(r, dtype=np.float64)
        rc = self.r_cutoff if self.r_cutoff > 0.0 else 1e30
        v = self.raw(r) - self.epsilon_shift
        if scheme == BH:
            val = np.where(r >= self.r_zero, v, 0.0)
        else:
            val = np.where(r >= self.r_min, v, self.v_min)
        return np.where(r >= rc, 0.0, val)


def make_lennard_jones(sigma: float, epsilon: float, r_cutoff: float = -1.0) -> LennardJones:
    """potentials.hpp:311-325."""
    def vr(r):
        y = sigma / r
        y6 = y * y * y * y * y * y
        return 4.0 * epsilon * (y6 * y6 - y6)

    lj = LennardJones(sigma=sigma, epsilon=epsilon, r_cutoff=r_cutoff)
    lj.epsilon_shift = vr(r_cutoff) if r_cutoff > 0.0 else 0.0
    lj.r_min = math.pow(2.0, 1.0 / 6.0) * sigma
    lj.v_min = vr(lj.r_min) - lj.epsilon_shift
    lj.r_zero = sigma * math.pow(0.5 * math.sqrt(1.0 + lj.epsilon_shift / epsilon) + 0.5, -1.0 / 6.0)
    return lj


@dataclass
class TenWoldeFrenkel:
    """potentials.hpp:122-182, built by make_ten_wolde_frenkel (:327-346)."""

    sigma: float = 1.0
    epsilon: float = 1.0
    r_cutoff: float = -1.0
    alpha: float = 50.0
    epsilon_shift: float = 0.0
    r_min: float = 0.0
    v_min: float = 0.0
    r_zero: float = 0.0
    name: str = "TenWoldeFrenkel"

    def raw(self, r):
        r = np.asarray(r, dtype=np.float64)
        with np.errstate(divide="ignore", invalid="ignore", over="ignore"):
            s = r / self.sigma
            y = 1.0 / (s * s - 1.0)
            y3 = y * y * y
            v = (4.0 * self.epsilon / (self.alpha * self.alpha)) * (y3 * y3 - self.alpha * y3)
        return np.where(r < self.sigma, MAX_POTENTIAL_VALUE, v)

    def hard_core_diameter(self):
        return self.sigma

    def split_point(self, scheme):
        return self.r_zero if scheme == BH else self.r_min

    def repulsive(self, r, scheme):
        r = np.asarray(r, dtype=np.float64)
        v = self.raw(r) - self.epsilon_shift
        if scheme == BH:
            return np.where(r < self.r_zero, v, 0.0)
        return np.where(r < self.r_min, v - self.v_min, 0.0)

    def attractive(self, r, scheme):
        r = np.asarray(r, dtype=np.float64)
        rc = self.r_cutoff if self.r_cutoff > 0.0 else 1e30
        v = self.raw(r) - self.epsilon_shift
        if scheme == BH:
            val = np.where(r >= self.r_zero, v, 0.0)
        else:
            val = np.where(r >= self.r_min, v, self.v_min)
        return np.where(r >= rc, 0.0, val)


def make_ten_wolde_frenkel(sigma, epsilon, r_cutoff=-1.0, alpha=50.0) -> TenWoldeFrenkel:
    """potentials.hpp:327-346."""
    def vr(r):
        if r < sigma:
            return MAX_POTENTIAL_VALUE
        s = r / sigma
        y = 1.0 / (s * s - 1.0)
        y3 = y * y * y
        return (4.0 * epsilon / (alpha * alpha)) * (y3 * y3 - alpha * y3)

    t = TenWoldeFrenkel(sigma=sigma, epsilon=epsilon, r_cutoff=r_cutoff, alpha=alpha)
    t.epsilon_shift = vr(r_cutoff) if r_cutoff > 0.0 else 0.0
    t.r_min = sigma * math.sqrt(1.0 + math.pow(2.0 / alpha, 1.0 / 3.0))
    t.v_min = vr(t.r_min) - t.epsilon_shift
    t.r_zero = sigma * math.sqrt(1.0 + math.pow(25.0 * math.sqrt(1.0 + t.epsilon_shift) + 25.0, -1.0 / 3.0))
    return t


@dataclass
class WangRamirezDobnikarFrenkel:
    """potentials.hpp:188-243, built by make_wang_ramirez_dobnikar_frenkel (:348-368)."""

    sigma: float = 1.0
    epsilon: float = 1.0
    r_cutoff: float = 3.0
    epsilon_effective: float = 0.0
    r_min: float = 0.0
    v_min: float = 0.0
    name: str = "WangRamirezDobnikarFrenkel"

    def raw(self, r):
        r = np.asarray(r, dtype=np.float64)
        with np.errstate(divide="ignore", invalid="ignore", over="ignore"):
            y = self.sigma / r
            z = self.r_cutoff / r
            v = self.epsilon_effective * (y * y - 1.0) * (z * z - 1.0) * (z * z - 1.0)
        return np.where(r >= self.r_cutoff, 0.0, v)

    def hard_core_diameter(self):
        return 0.0

    def split_point(self, scheme):
        return self.r_min

    def repulsive(self, r, scheme):
        r = np.asarray(r, dtype=np.float64)
        v = self.raw(r)
        if scheme == BH:
            return np.where(r < self.r_min, v, 0.0)
        return np.where(r < self.r_min, v - self.v_min, 0.0)

    def attractive(self, r, scheme):
        r = np.asarray(r, dtype=np.float64)
        v = self.raw(r)
        if scheme == BH:
            val = np.where(r >= self.r_min, v, 0.0)
        else:
            val = np.where(r >= self.r_min, v, self.v_min)
        return np.where(r >= self.r_cutoff, 0.0, val)


def make_wang_ramirez_dobnikar_frenkel(sigma, epsilon, r_cutoff=3.0):
    """potentials.hpp:348-368."""
    rc_s = r_cutoff / sigma
    eps_eff = epsilon * 2.0 * rc_s * rc_s * math.pow(2.0 * (rc_s * rc_s - 1.0) / 3.0, -3.0)
    w = WangRamirezDobnikarFrenkel(sigma=sigma, epsilon=epsilon, r_cutoff=r_cutoff, epsilon_effective=eps_eff)
    w.r_min = r_cutoff * math.pow((1.0 + 2.0 * rc_s * rc_s) / 3.0, -0.5)
    w.v_min = float(w.raw(w.r_min))
    return w


def hard_sphere_diameter(pot, kT: float, scheme: str = WCA) -> float:
    """potentials.hpp:28-37: d = d_core + int_{d_core}^{r_split} (1 - exp(-v_rep/kT)) dr."""
    d_core = pot.hard_core_diameter()
    r_split = pot.split_point(scheme)

    def kernel(r):
        with np.errstate(over="ignore"):
            return float(1.0 - np.exp(-pot.repulsive(r, scheme) / kT))

    val, _ = integrate.quad(kernel, d_core, r_split, epsabs=1e-10, epsrel=1e-10, limit=1000)
    return d_core + val


def vdw_integral(pot, kT: float, scheme: str = WCA) -> float:
    """potentials.hpp:39-50: (2 pi / kT) int r^2 v_att(r) dr."""
    if pot.r_cutoff <= 0.0:
        return 0.0
    r_lower = pot.split_point(scheme) if scheme == BH else 0.0
    val, _ = integrate.quad(lambda r: float(r * r * pot.attractive(r, scheme)), r_lower, pot.r_cutoff,
                            epsabs=1e-10, epsrel=1e-10, limit=1000)
    return (2.0 * math.pi / kT) * val


# ------------------------------------------------------- cell weights

ZERO = "InterpolationZero"
LINEAR_E = "InterpolationLinearE"
LINEAR_F = "InterpolationLinearF"
QUADRATIC_F = "InterpolationQuadraticF"
GAUSS_E = "GaussE"
GAUSS_F = "GaussF"


@dataclass
class Interaction:
    """interactions.hpp:23-30."""

    species_i: int
    species_j: int
    potential: object
    split: str = WCA
    weight_scheme: str = QUADRATIC_F


def cell_weight(inter: Interaction, kT: float, dx: float, sx, sy, sz):
    """mean_field.hpp:42-134: cell weight(s) at integer displacement(s) (sx, sy, sz)."""
    pot = inter.potential
    split = inter.split
    sx = np.asarray(sx, dtype=np.int64)
    sy = np.asarray(sy, dtype=np.int64)
    sz = np.asarray(sz, dtype=np.int64)
    scheme = inter.weight_scheme
    if scheme == ZERO:                                   # :42-54
        r2 = (sx * sx + sy * sy + sz * sz).astype(np.float64) * dx * dx
        return pot.attractive(np.sqrt(r2), split) / kT
    if scheme in (LINEAR_E, LINEAR_F, GAUSS_E, GAUSS_F):  # :59-81
        total = np.zeros(np.broadcast(sx, sy, sz).shape)
        for di in (0, 1):
            for dj in (0, 1):
                for dk in (0, 1):
                    x = (sx.astype(np.float64) - 0.5 + di) * dx
                    y = (sy.astype(np.float64) - 0.5 + dj) * dx
                    z = (sz.astype(np.float64) - 0.5 + dk) * dx
                    total = total + pot.attractive(np.sqrt(x * x + y * y + z * z), split) / kT
        return total / 8.0
    if scheme == QUADRATIC_F:                            # :87-112
        vv = (1.0 / 3.0, 1.0 / 3.0, 1.0 / 3.0)
        pt = (-0.5, 0.0, 0.5)
        total = np.zeros(np.broadcast(sx, sy, sz).shape)
        for i in range(3):
            for j in range(3):
                for k in range(3):
                    rx = (sx.astype(np.float64) + pt[i]) * dx
                    ry = (sy.astype(np.float64) + pt[j]) * dx
                    rz = (sz.astype(np.float64) + pt[k]) * dx
                    r = np.sqrt(rx * rx + ry * ry + rz * rz)
                    total = total + vv[i] * vv[j] * vv[k] * pot.attractive(r, split) / kT
        return total
    raise ValueError(f"unknown weight scheme {scheme}")


def interaction_weight_real(inter: Interaction, grid: Grid, kT: float):
    """mean_field.hpp:146-196 (before the FFT): real-space weight x dV/N and a_vdw."""
    nx, ny, nz = grid.shape
    dx = grid.dx
    dv = grid.cell_volume
    inv_n = 1.0 / float(grid.total_points)
    r_cut = inter.potential.r_cutoff
    margin = math.sqrt(3.0) * 0.5 * dx
    r_skip = r_cut + margin
    r_skip_sq = r_skip * r_skip

    def sgn(n):
        i = np.arange(n)
        return np.where(i <= n // 2, i, i - n)

    SX = sgn(nx)[:, None, None]
    SY = sgn(ny)[None, :, None]
    SZ = sgn(nz)[None, None, :]
    SX, SY, SZ = np.broadcast_arrays(SX, SY, SZ)
    dist2 = (SX * SX + SY * SY + SZ * SZ).astype(np.float64) * dx * dx
    keep = np.ones(grid.shape, dtype=bool)
    if r_cut > 0.0:
        keep = ~(dist2 > r_skip_sq)
    real = np.zeros(grid.shape, dtype=np.float64)
    with np.errstate(divide="ignore", invalid="ignore", over="ignore"):
        w = cell_weight(inter, kT, dx, SX[keep], SY[keep], SZ[keep])
    real[keep] = w * dv * inv_n
    a_vdw = float(np.sum(w * dv))
    return real, a_vdw


def generate_interaction_weight(inter: Interaction, grid: Grid, kT: float):
    """mean_field.hpp:146-196: (k-space weight, a_vdw)."""
    real, a_vdw = interaction_weight_real(inter, grid, kT)
    return r2c(real), a_vdw
