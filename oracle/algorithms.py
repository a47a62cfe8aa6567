"""FIRE2, density minimisation, DDFT and saddle-point search (oracle, test infrastructure only).

Restates include/dft/algorithms/{fire,minimization,dynamics,saddle_point,picard}.hpp.
Vectors are flat FP64 NumPy arrays; multi-species state is a list of them.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field, replace

import numpy as np

from .grid import Grid, boundary_mask, c2r, fixed_boundary, homogeneous_boundary, r2c, wavevectors

# ================================================================= FIRE2


@dataclass
class FireState:
    """fire.hpp:15-26."""

    x: list
    v: list
    dt: float
    alpha: float
    n_positive: int = 0
    n_negative: int = 0
    energy: float = 0.0
    rms_force: float = 0.0
    iteration: int = 0
    converged: bool = False


@dataclass
class Fire:
    """fire.hpp:33-58 (parameters and defaults)."""

    dt: float = 1e-3
    dt_max: float = 1e-2
    dt_min: float = 1e-8
    alpha_start: float = 0.1
    f_inc: float = 1.1
    f_dec: float = 0.5
    f_alpha: float = 0.99
    n_delay: int = 5
    max_uphill: int = 20
    force_tolerance: float = 0.1
    max_steps: int = 10000

    def initialize(self, x0, compute) -> FireState:
        """fire.hpp:60-84."""
        energy, forces = compute(x0)
        total_dof = 0.0
        sum_f2 = 0.0
        v = []
        for s in range(len(x0)):
            v.append(np.zeros_like(x0[s]))
            sum_f2 += float(np.dot(forces[s], forces[s]))
            total_dof += float(forces[s].size)
        rms = math.sqrt(sum_f2 / total_dof)
        return FireState(x=[np.array(a, dtype=np.float64) for a in x0], v=v, dt=self.dt, alpha=self.alpha_start,
                         energy=energy, rms_force=rms, converged=rms < self.force_tolerance)

    def step(self, st: FireState, forces, compute):
        """fire.hpp:86-165."""
        st = replace(st, x=[a.copy() for a in st.x], v=[a.copy() for a in st.v])
        power = 0.0
        for s in range(len(st.x)):
            power += float(np.dot(st.v[s], forces[s]))
        if power > 0.0 or st.iteration == 0:
            st.n_positive += 1
            st.n_negative = 0
            if st.n_positive > self.n_delay:
                st.dt = min(st.dt * self.f_inc, self.dt_max)
                st.alpha *= self.f_alpha
        else:
            st.n_positive = 0
            st.n_negative += 1
            if st.n_negative > self.max_uphill:
                raise RuntimeError("fire::step: exceeded max uphill steps")
            for s in range(len(st.x)):
                st.x[s] = st.x[s] - 0.5 * st.dt * st.v[s]
                st.v[s] = np.zeros_like(st.v[s])
            if st.iteration > self.n_delay:
                st.dt = max(st.dt * self.f_dec, self.dt_min)
                st.alpha = self.alpha_start
        for s in range(len(st.x)):
            st.v[s] = st.v[s] + st.dt * forces[s]
        v_norm = 0.0
        f_norm = 0.0
        for s in range(len(st.x)):
            v_norm += float(np.dot(st.v[s], st.v[s]))
            f_norm += float(np.dot(forces[s], forces[s]))
        v_norm = math.sqrt(v_norm)
        f_norm = math.sqrt(f_norm)
        if f_norm > 0.0:
            ratio = v_norm / f_norm
            for s in range(len(st.x)):
                st.v[s] = (1.0 - st.alpha) * st.v[s] + st.alpha * ratio * forces[s]
        for s in range(len(st.x)):
            st.x[s] = st.x[s] + st.dt * st.v[s]
        energy, new_forces = compute(st.x)
        st.energy = energy
        total_dof = 0.0
        sum_f2 = 0.0
        for s in range(len(st.x)):
            sum_f2 += float(np.dot(new_forces[s], new_forces[s]))
            total_dof += float(new_forces[s].size)
        st.rms_force = math.sqrt(sum_f2 / total_dof)
        st.iteration += 1
        st.converged = st.rms_force < self.force_tolerance
        return st, new_forces

    def minimize(self, x0, compute) -> FireState:
        """fire.hpp:167-178."""
        st = self.initialize(x0, compute)
        _, forces = compute(st.x)
        for _ in range(self.max_steps):
            if st.converged:
                break
            st, forces = self.step(st, forces, compute)
        return st


# ============================================================ minimisation


@dataclass
class Unbounded:
    """minimization.hpp:27-29: rho = rho_min + x^2."""

    rho_min: float = 1e-18


@dataclass
class Bounded:
    """minimization.hpp:34-37: rho = rho_min + range x^2/(1+x^2)."""

    rho_min: float = 1e-18
    rho_max: float = 1.0


def to_density(x, p):
    """minimization.hpp:45-60."""
    if isinstance(p, Unbounded):
        return p.rho_min + x * x
    rng = p.rho_max - p.rho_min
    x2 = x * x
    return p.rho_min + rng * x2 / (1.0 + x2)


def from_density(rho, p):
    """minimization.hpp:63-78."""
    if isinstance(p, Unbounded):
        return np.sqrt(np.clip(rho - p.rho_min, 0.0, np.inf))
    rng = p.rho_max - p.rho_min
    delta = np.clip(rho - p.rho_min, 0.0, rng * (1.0 - 1e-14))
    return np.sqrt(delta / (rng - delta))


def transform_force(f_rho, x, p):
    """minimization.hpp:82-99: f_x = f_rho * drho/dx."""
    if isinstance(p, Unbounded):
        return f_rho * (2.0 * x)
    rng = p.rho_max - p.rho_min
    x2 = x * x
    denom = (1.0 + x2) * (1.0 + x2)
    return f_rho * (2.0 * rng * x / denom)


def convergence_monitor(vv, old_energy, new_energy, dt, volume):
    """minimization.hpp:106-111."""
    new_vv = vv * 0.9 + 0.1 * (abs(new_energy - old_energy) / dt)
    return new_vv, abs(new_vv / volume)


@dataclass
class MinResult:
    """minimization.hpp:114-121."""

    densities: list
    free_energy: float
    grand_potential: float
    rms_force: float
    iterations: int
    converged: bool


@dataclass
class Minimizer:
    """minimization.hpp:123-147, 182-354.

    ``total_fn(rho, mu) -> (free_energy, grand_potential, force)`` evaluates the
    functional for a single-species profile (the reference calls
    functionals::total on init::from_profile(model, rho)).
    """

    fire: Fire = field(default_factory=Fire)
    param: object = field(default_factory=Unbounded)
    use_homogeneous_boundary: bool = True

    def fixed_mass(self, grid: Grid, total_fn, initial_density, chemical_potential, target_mass):
        dv = grid.cell_volume
        bdry = boundary_mask(grid)

        def compute(x_param):
            rho = to_density(x_param[0], self.param)
            mass = float(np.sum(rho)) * dv
            if mass > 0.0:
                rho = rho * (target_mass / mass)
            _, omega, grad = total_fn(rho, 0.0)
            if self.use_homogeneous_boundary:
                grad = homogeneous_boundary(grad, bdry)
            lam = float(np.dot(grad, rho)) / target_mass
            grad = grad - lam * dv
            f = transform_force(grad, x_param[0], self.param)
            return omega, [-f]

        x0 = from_density(np.asarray(initial_density, dtype=np.float64), self.param)
        volume = float(x0.size) * dv
        st = self.fire.initialize([x0], compute)
        _, forces = compute(st.x)
        vv = 1.0
        converged = False
        for _ in range(self.fire.max_steps):
            if converged:
                break
            old = st.energy
            st, forces = self.fire.step(st, forces, compute)
            vv, monitor = convergence_monitor(vv, old, st.energy, st.dt, volume)
            converged = monitor < self.fire.force_tolerance
            st.converged = converged
        rho_final = to_density(st.x[0], self.param)
        fm = float(np.sum(rho_final)) * dv
        if fm > 0.0:
            rho_final = rho_final * (target_mass / fm)
        F, omega, _ = total_fn(rho_final, chemical_potential)
        return MinResult([rho_final], F, omega, st.rms_force, st.iteration, st.converged)

    def grand_potential(self, grid: Grid, total_fn, initial_density, chemical_potential):
        bdry = boundary_mask(grid)

        def compute(x_param):
            rho = to_density(x_param[0], self.param)
            _, omega, grad = total_fn(rho, chemical_potential)
            if self.use_homogeneous_boundary:
                grad = homogeneous_boundary(grad, bdry)
            f = transform_force(grad, x_param[0], self.param)
            return omega, [-f]

        x0 = from_density(np.asarray(initial_density, dtype=np.float64), self.param)
        volume = float(x0.size) * grid.cell_volume
        st = self.fire.initialize([x0], compute)
        _, forces = compute(st.x)
        vv = 1.0
        converged = False
        for _ in range(self.fire.max_steps):
            if converged:
                break
            old = st.energy
            st, forces = self.fire.step(st, forces, compute)
            vv, monitor = convergence_monitor(vv, old, st.energy, st.dt, volume)
            converged = monitor < self.fire.force_tolerance
            st.converged = converged
        rho_final = to_density(st.x[0], self.param)
        F, omega, _ = total_fn(rho_final, chemical_potential)
        return MinResult([rho_final], F, omega, st.rms_force, st.iteration, st.converged)


# ================================================================== DDFT


@dataclass
class StepConfig:
    """dynamics.hpp:26-33."""

    dt: float = 1e-4
    diffusion_coefficient: float = 1.0
    min_density: float = 1e-18
    dt_max: float = 1.0
    fp_tolerance: float = 1e-4
    fp_max_iterations: int = 100


class IFState:
    """dynamics.hpp:70-129: FD-Laplacian eigenvalues and exp(lambda dt) factors."""

    def __init__(self, grid: Grid):
        nx, ny, nz = grid.shape
        self.shape = grid.shape
        self.dx = grid.dx
        Dx = 1.0 / (grid.dx * grid.dx)
        self.lam_x = 2.0 * Dx * (np.cos(2.0 * np.pi * np.arange(nx) / nx) - 1.0)
        self.lam_y = 2.0 * Dx * (np.cos(2.0 * np.pi * np.arange(ny) / ny) - 1.0)
        self.lam_z = 2.0 * Dx * (np.cos(2.0 * np.pi * np.arange(nz // 2 + 1) / nz) - 1.0)
        self.dt = 0.0
        self.fx = self.fy = self.fz = None

    def update_timestep(self, dt):
        if abs(self.dt - dt) < 1e-30:
            return
        self.dt = dt
        self.fx = np.exp(self.lam_x * dt)
        self.fy = np.exp(self.lam_y * dt)
        self.fz = np.exp(self.lam_z * dt)


def divergence_flux(rho, x, shape, dx):
    """dynamics.hpp:135-170: div(rho grad x) with the 7-point flux stencil."""
    D = 0.5 / (dx * dx)
    r = rho.reshape(shape)
    f = x.reshape(shape)
    g = np.zeros(shape)
    for ax in range(3):
        rp = np.roll(r, -1, axis=ax)
        rm = np.roll(r, 1, axis=ax)
        fp = np.roll(f, -1, axis=ax)
        fm = np.roll(f, 1, axis=ax)
        g = g + D * ((rp + r) * (fp - f) - (r + rm) * (f - fm))
    return g.reshape(-1)


def laplacian(rho, shape, dx):
    """dynamics.hpp:174-206 (the term subtracted): 3-point FD Laplacian."""
    D = 1.0 / (dx * dx)
    r = rho.reshape(shape)
    out = np.zeros(shape)
    for ax in range(3):
        out = out + D * (np.roll(r, -1, axis=ax) + np.roll(r, 1, axis=ax) - 2.0 * r)
    return out.reshape(-1)


def excess_rhs_real(rho, forces, dv, shape, dx):
    """dynamics.hpp:233-242: R = div(rho grad(force/dV)) - lap(rho)."""
    return divergence_flux(rho, forces / dv, shape, dx) - laplacian(rho, shape, dx)


def apply_propagator(st: IFState, rho0_k, r0_k, r1_k, d1):
    """dynamics.hpp:247-304: returns (new d1, max |d1_new - d1_old|)."""
    nx, ny, nz = st.shape
    lam = st.lam_x[:, None, None] + st.lam_y[None, :, None] + st.lam_z[None, None, :]
    ex = st.fx[:, None, None] * st.fy[None, :, None] * st.fz[None, None, :]
    dt = st.dt
    with np.errstate(divide="ignore", invalid="ignore"):
        U1 = (ex - 1.0) / lam
        U2 = (ex - 1.0 - dt * lam) / (lam * lam * dt)
    U1[0, 0, 0] = dt
    U2[0, 0, 0] = dt / 2.0
    work = ex * rho0_k + U1 * r0_k + U2 * (r1_k - r0_k)
    n = nx * ny * nz
    new = c2r(work, st.shape).reshape(-1) * (1.0 / n)
    dev = float(np.max(np.abs(d1 - new)))
    return new, dev


def integrating_factor_step(densities, grid: Grid, st: IFState, compute, config: StepConfig):
    """dynamics.hpp:333-401 (config.dt is updated in place on restarts)."""
    shape = grid.shape
    dv = grid.cell_volume
    energy, forces = compute(densities)
    r0_k = r2c(excess_rhs_real(densities[0], forces[0], dv, shape, grid.dx).reshape(shape))
    rho0_k = r2c(densities[0].reshape(shape))
    while True:
        restart = False
        st.update_timestep(config.dt)
        d1 = densities[0].copy()
        deviation = 1e30
        for it in range(config.fp_max_iterations):
            _, f1 = compute([d1])
            r1_k = r2c(excess_rhs_real(d1, f1[0], dv, shape, grid.dx).reshape(shape))
            old = deviation
            d1, deviation = apply_propagator(st, rho0_k, r0_k, r1_k, d1)
            if d1.min() < 0.0 or (it > 0 and deviation > old):
                restart = True
                break
            if deviation < config.fp_tolerance:
                break
        if not restart and deviation > config.fp_tolerance:
            restart = True
        if restart:
            config.dt /= 10.0
            continue
        break
    e_final, _ = compute([d1])
    return [d1], e_final, config.dt


def compute_k_squared(grid: Grid):
    """dynamics.hpp:310-318."""
    kx, ky, kz = wavevectors(grid)
    return (kx * kx + ky * ky + kz * kz)


def diffusion_propagator(k2, D, dt):
    """dynamics.hpp:320-322."""
    return np.exp(-D * k2 * dt)


def split_operator_step(densities, grid: Grid, k2, prop, compute, config: StepConfig):
    """dynamics.hpp:410-465 (Strang splitting)."""
    shape = grid.shape
    n = grid.total_points
    dv = grid.cell_volume
    half = np.sqrt(prop)
    rho_star = c2r(r2c(densities[0].reshape(shape)) * half, shape).reshape(-1) * (1.0 / n)
    rho_star = np.clip(rho_star, config.min_density, np.inf)
    _, forces = compute([rho_star])
    rhs = excess_rhs_real(rho_star, forces[0], dv, shape, grid.dx)
    rho_dstar = np.clip(rho_star + config.dt * rhs, config.min_density, np.inf)
    d1 = c2r(r2c(rho_dstar.reshape(shape)) * half, shape).reshape(-1) * (1.0 / n)
    d1 = np.clip(d1, config.min_density, np.inf)
    e_final, _ = compute([d1])
    return [d1], e_final, config.dt


def crank_nicholson_step(densities, grid: Grid, k2, compute, config: StepConfig):
    """dynamics.hpp:472-538."""
    shape = grid.shape
    n = grid.total_points
    dv = grid.cell_volume
    D = config.diffusion_coefficient
    dt = config.dt
    a = D * k2 * dt * 0.5
    cn_minus = 1.0 - a
    cn_plus_inv = 1.0 / (1.0 + a)
    rho0_k = r2c(densities[0].reshape(shape))
    _, f0 = compute(densities)
    r0_k = r2c(excess_rhs_real(densities[0], f0[0], dv, shape, grid.dx).reshape(shape))
    d1 = densities[0].copy()
    for _ in range(config.fp_max_iterations):
        _, f1 = compute([d1])
        r1_k = r2c(excess_rhs_real(d1, f1[0], dv, shape, grid.dx).reshape(shape))
        wk = (cn_minus * rho0_k + (dt * 0.5) * (r0_k + r1_k)) * cn_plus_inv
        d1_new = np.clip(c2r(wk, shape).reshape(-1) * (1.0 / n), config.min_density, np.inf)
        dev = float(np.max(np.abs(d1_new - d1)))
        d1 = d1_new
        if dev < config.fp_tolerance:
            break
    e_final, _ = compute([d1])
    return [d1], e_final, dt


@dataclass
class Simulation:
    """dynamics.hpp:564-693: integrating-factor DDFT with adaptive dt."""

    step: StepConfig = field(default_factory=StepConfig)
    n_steps: int = 1000
    snapshot_interval: int = 100
    boundary: object = None

    def run(self, densities, grid: Grid, force_fn):
        dv = grid.cell_volume
        densities = [np.array(d, dtype=np.float64).reshape(-1) for d in densities]
        if self.boundary:
            self.boundary(densities)
        mass_initial = sum(float(np.sum(r)) * dv for r in densities)
        st = IFState(grid)
        cfg = replace(self.step)
        e0, _ = force_fn(densities)
        times = [0.0]
        energies = [e0]
        successes = 0
        time = 0.0
        for step in range(1, self.n_steps + 1):
            dt_before = cfg.dt
            densities, e_step, dt_used = integrating_factor_step(densities, grid, st, force_fn, cfg)
            time += dt_used
            if self.boundary:
                self.boundary(densities)
            if dt_used < dt_before:
                successes = 0
            else:
                successes += 1
            if successes >= 5 and cfg.dt < cfg.dt_max:
                cfg.dt = min(2.0 * cfg.dt, cfg.dt_max)
                successes = 0
            times.append(time)
            energies.append(e_step)
        mass_final = sum(float(np.sum(r)) * dv for r in densities)
        return {"densities": densities, "times": times, "energies": energies,
                "mass_initial": mass_initial, "mass_final": mass_final, "dt": cfg.dt}


# ========================================================== saddle point


def hessian_times_vector(force_fn, rho, forces_at_rho, v, eps=1e-6):
    """saddle_point.hpp:30-39: FD Hessian-vector product."""
    _, fs = force_fn(rho + eps * v)
    return (fs - forces_at_rho) / eps


@dataclass
class EigenvalueResult:
    eigenvector: np.ndarray
    eigenvalue: float
    iterations: int
    converged: bool


@dataclass
class EigenvalueSolver:
    """saddle_point.hpp:158-276: smallest Hessian eigenpair (3-vector Rayleigh-Ritz).

    ``hvp(v) -> H v`` may be given to replace the FD product (an exact HVP).
    """

    tolerance: float = 1e-4
    max_iterations: int = 300
    hessian_eps: float = 1e-6
    seed: int = 42

    def solve(self, force_fn, rho, initial_guess=None, hvp=None):
        _, forces = force_fn(rho)
        n = rho.size
        if hvp is None:
            def hvp(vec):
                return hessian_times_vector(force_fn, rho, forces, vec, self.hessian_eps)
        if initial_guess is not None and initial_guess.size == n:
            v = np.array(initial_guess, dtype=np.float64)
        else:
            v = np.random.default_rng(self.seed).standard_normal(n)
        v = v / np.linalg.norm(v)
        hv = hvp(v)
        lam = float(np.dot(v, hv))
        p_raw = None
        converged = False
        it = 0
        while it < self.max_iterations:
            residual = hv - lam * v
            res_norm = float(np.linalg.norm(residual))
            if res_norm < self.tolerance:
                converged = True
                break
            q0 = v
            q1 = residual - float(np.dot(residual, q0)) * q0
            q1n = float(np.linalg.norm(q1))
            if q1n < 1e-30:
                break
            q1 = q1 / q1n
            hq0 = hv
            hq1 = hvp(q1)
            dim = 2
            q2 = hq2 = None
            if p_raw is not None:
                q2 = p_raw - float(np.dot(p_raw, q0)) * q0 - float(np.dot(p_raw, q1)) * q1
                q2n = float(np.linalg.norm(q2))
                if q2n > 1e-10:
                    q2 = q2 / q2n
                    hq2 = hvp(q2)
                    dim = 3
            H = np.zeros((dim, dim))
            H[0, 0] = np.dot(q0, hq0)
            H[0, 1] = H[1, 0] = np.dot(q0, hq1)
            H[1, 1] = np.dot(q1, hq1)
            if dim == 3:
                H[0, 2] = H[2, 0] = np.dot(q0, hq2)
                H[1, 2] = H[2, 1] = np.dot(q1, hq2)
                H[2, 2] = np.dot(q2, hq2)
            _, vecs = np.linalg.eigh(H)
            c = vecs[:, 0]
            v_new = c[0] * q0 + c[1] * q1
            if dim == 3:
                v_new = v_new + c[2] * q2
            p_raw = v_new - v
            v = v_new / np.linalg.norm(v_new)
            hv = hvp(v)
            lam = float(np.dot(v, hv))
            it += 1
        return EigenvalueResult(v, lam, it, converged)


@dataclass
class SaddleResult:
    """saddle_point.hpp:313-320."""

    density: np.ndarray
    eigenvector: np.ndarray
    grand_potential: float
    eigenvalue: float
    outer_iterations: int
    converged: bool
    fire_steps: int = 0


@dataclass
class Search:
    """saddle_point.hpp:324-589: eigenvector following at fixed mass.

    ``total_fn(rho, mu) -> (free_energy, grand_potential, force)`` evaluates the
    functional for a single-species profile.  Each outer iteration draws its
    random eigen start from seed ``eigenvalue.seed + outer`` (the reference
    draws from Armadillo's global generator)."""

    fire: Fire = field(default_factory=lambda: Fire(dt=1e-3, dt_max=1.0, alpha_start=0.01, f_alpha=1.0,
                                                    force_tolerance=1e-4, max_steps=100000))
    eigenvalue: EigenvalueSolver = field(default_factory=lambda: EigenvalueSolver(1e-4, 300, 1e-6))
    param: object = field(default_factory=lambda: Unbounded(1e-18))
    omega_tolerance: float = 1e-5
    tolerance_start: float = 1e-3
    tolerance_factor: float = 10.0
    max_outer_iterations: int = 20
    eigenvalue_clear_count: int = 2

    def find(self, grid: Grid, total_fn, initial_density, chemical_potential, target_mass):
        dv = grid.cell_volume
        bdry = boundary_mask(grid).astype(bool)
        inner = ~bdry

        def eig_force_fn(rho):  # saddle_point.hpp:377-384
            _, omega, f = total_fn(rho, chemical_potential)
            return omega, fixed_boundary(f, bdry)

        rho = np.array(initial_density, dtype=np.float64)
        eigvec = None
        omega = 0.0
        ev = 0.0
        converged = False
        ftol = self.tolerance_start
        steps = 0
        outer = 0
        while outer < self.max_outer_iterations:
            omega_old = omega
            guess = eigvec if (outer >= self.eigenvalue_clear_count and eigvec is not None) else None
            er = replace(self.eigenvalue, seed=self.eigenvalue.seed + outer).solve(eig_force_fn, rho, guess)
            eigvec = er.eigenvector
            ev = er.eigenvalue
            # direction in parameter space (saddle_point.hpp:424-430)
            x_cur = from_density(rho, self.param)
            dir_alias = transform_force(eigvec, x_cur, self.param)
            dn = float(np.linalg.norm(dir_alias))
            if dn > 1e-30:
                dir_alias = dir_alias / dn
            # boundary mass (saddle_point.hpp:432-443)
            nb = int(bdry.sum())
            m_boundary = (float(rho[bdry].sum()) / nb if nb > 0 else 0.0) * dv * nb
            m_t_int = target_mass - m_boundary

            def compute(x_param):  # saddle_point.hpp:445-492
                rho_l = to_density(x_param[0], self.param)
                m_int = float(rho_l[inner].sum()) * dv
                if m_int > 0.0 and m_t_int > 0.0:
                    rho_l = rho_l.copy()
                    rho_l[inner] *= m_t_int / m_int
                _, om, grad = total_fn(rho_l, chemical_potential)
                grad = fixed_boundary(grad, bdry)
                mu_l = float(np.dot(grad[inner], rho_l[inner]))
                if m_t_int > 0.0:
                    mu_l /= m_t_int
                grad = np.where(bdry, 0.0, grad - mu_l * dv)
                f = transform_force(grad, x_param[0], self.param)
                f = f - float(np.dot(dir_alias, f)) * dir_alias
                return om, [-f]

            # FIRE2 at fixed mass, projected (saddle_point.hpp:496-530)
            fire_cfg = replace(self.fire, force_tolerance=max(ftol, self.fire.force_tolerance))
            ftol /= self.tolerance_factor
            st = fire_cfg.initialize([from_density(rho, self.param)], compute)
            _, forces0 = compute(st.x)
            for _ in range(fire_cfg.max_steps):
                if st.converged:
                    break
                st, forces0 = fire_cfg.step(st, forces0, compute)
            steps += st.iteration
            # final density (saddle_point.hpp:533-549) and Omega (:551-554)
            rho = to_density(st.x[0], self.param)
            fm = float(rho[inner].sum()) * dv
            if fm > 0.0 and m_t_int > 0.0:
                rho = rho.copy()
                rho[inner] *= m_t_int / fm
            _, omega, _ = total_fn(rho, chemical_potential)
            if outer > 0 and abs(omega - omega_old) < self.omega_tolerance:
                converged = True
                break
            outer += 1
        return SaddleResult(rho, eigvec, omega, ev, outer + 1, converged, steps)


def dense_fixed_boundary_hessian(grid: Grid, force_fn, rho, h=1e-5):
    """The interior block of the fixed-boundary Hessian by central
    differences of the force (small grids only): H[:, j] =
    (f(rho + h e_j) - f(rho - h e_j)) / 2h restricted to interior rows and
    columns.  Returns (H, interior indices)."""
    inner = np.nonzero(~boundary_mask(grid).astype(bool))[0]
    H = np.empty((inner.size, inner.size))
    for c, j in enumerate(inner):
        e = np.zeros_like(rho)
        e[j] = h
        H[:, c] = ((force_fn(rho + e) - force_fn(rho - e)) / (2.0 * h))[inner]
    return H, inner


# ================================================================= Picard


def fixed_mass_constraint(target_masses, backgrounds, cell_volume, min_density=1e-30):
    """minimization.hpp:159-180: rescale the excess over the background of
    each species to its target mass (skipped when the mass is ~0)."""

    def apply(densities):
        out = [np.array(r, dtype=np.float64) for r in densities]
        for s in range(min(len(out), len(target_masses))):
            excess = out[s] - backgrounds[s]
            mass = float(np.sum(excess)) * cell_volume
            if abs(mass) > 1e-30:
                out[s] = np.maximum(backgrounds[s] + (target_masses[s] / mass) * excess, min_density)
        return out

    return apply


@dataclass
class PicardResult:
    """picard.hpp:23-29."""

    densities: list
    grand_potential: float
    residual: float
    iterations: int
    converged: bool


@dataclass
class Picard:
    """picard.hpp:31-124: log-space Picard iteration."""

    mixing: float = 0.01
    min_density: float = 1e-30
    tolerance: float = 1e-6
    max_iterations: int = 5000

    def solve(self, densities, compute, cell_volume, constraint=None):
        densities = [np.array(r, dtype=np.float64).reshape(-1) for r in densities]
        residual = 0.0
        omega = 0.0
        omega_prev = float(np.finfo(np.float64).max)
        it = 0
        while it < self.max_iterations:
            omega, forces = compute(densities)
            sum_f2 = sum(float(np.dot(f, f)) for f in forces)
            dof = float(sum(f.size for f in forces))
            residual = math.sqrt(sum_f2 / dof)
            if residual < self.tolerance or (it > 0 and abs(omega - omega_prev) < self.tolerance):
                break
            omega_prev = omega
            densities = [np.maximum(r * np.exp(-self.mixing * f / cell_volume), self.min_density)
                         for r, f in zip(densities, forces)]
            if constraint is not None:
                densities = constraint(densities)
            it += 1
        converged = residual < self.tolerance or (it > 0 and abs(omega - omega_prev) < self.tolerance)
        return PicardResult(densities, omega, residual, it, converged)
