"""Host-side mirror of the reference's algorithms, running on the GPU engine.

FIRE2 minimisation (fire.hpp, minimization.hpp), DDFT (dynamics.hpp) and the
saddle-point search (saddle_point.hpp) keep the reference's names,
parameters and defaults; their state lives in HBM and the steps run as
device kernels of libcdft_b200.so.  Densities are exchanged as NumPy arrays
(host) or torch CUDA tensors (device, no copy).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from .functionals import Model, Weights


def _torch():
    import torch
    return torch


def _dev(x):
    """(tensor on the current CUDA device, was_host) for a numpy array or tensor."""
    torch = _torch()
    if isinstance(x, torch.Tensor):
        if not x.is_cuda or x.dtype != torch.float64 or not x.is_contiguous():
            raise ValueError("device vectors must be contiguous float64 CUDA tensors")
        return x, False
    return torch.tensor(np.ascontiguousarray(x, dtype=np.float64).reshape(-1), device="cuda"), True


def _stream():
    return _torch().cuda.current_stream().cuda_stream


# ---------------------------------------------------------------- FIRE


@dataclass
class Fire:
    """fire.hpp:33-44: FIRE2 parameters (same defaults)."""

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

    def c(self):
        return _lib.CFireParams(self.dt, self.dt_max, self.dt_min, self.alpha_start, self.f_inc, self.f_dec,
                                self.f_alpha, self.n_delay, self.max_uphill, self.force_tolerance, self.max_steps)


@dataclass
class Unbounded:
    """minimization.hpp:27-29: rho = rho_min + x^2."""

    rho_min: float = 1e-18


@dataclass
class Bounded:
    """minimization.hpp:34-37: rho = rho_min + (rho_max - rho_min) x^2/(1+x^2)."""

    rho_min: float = 1e-18
    rho_max: float = 1.0


@dataclass
class MinimizationResult:
    """minimization.hpp:114-121."""

    densities: list
    free_energy: float
    grand_potential: float
    rms_force: float
    iterations: int
    converged: bool


def set_step_graphs(on: bool):
    """Process-wide: the FIRE minimisers capture one step (FIRE update and
    evaluation) as a CUDA graph and replay it every step (default on;
    results are identical either way)."""
    _lib.check(_lib.lib().cdft_set_step_graphs(1 if on else 0))


def step_graphs() -> bool:
    on = ctypes.c_int()
    _lib.check(_lib.lib().cdft_step_graphs(ctypes.byref(on)))
    return bool(on.value)


@dataclass
class Minimizer:
    """minimization.hpp:123-147 on the device.

    ``refine``: optional FP64 Weights of the same model; when given, the
    minimiser switches to them (defect correction) once the energy monitor
    falls below ``refine_switch`` x tolerance.
    """

    fire: Fire = field(default_factory=Fire)
    param: object = field(default_factory=Unbounded)
    use_homogeneous_boundary: bool = True
    check_interval: int = 25
    refine: Weights = None
    refine_switch: float = 10.0
    # convergence test: the reference Minimizer's energy monitor
    # (minimization.hpp:431-434), or with False the rms force of Fire::step
    # (fire.hpp:162) against fire.force_tolerance
    use_monitor: bool = True

    def _config(self, mode, mu, target_mass=0.0, boundary_mass=0.0, use_monitor=None):
        if use_monitor is None:
            use_monitor = self.use_monitor
        cfg = _lib.CMinimizerConfig()
        cfg.fire = self.fire.c()
        cfg.mode = mode
        if isinstance(self.param, Bounded):
            cfg.parametrization, cfg.rho_min, cfg.rho_max = 1, self.param.rho_min, self.param.rho_max
        else:
            cfg.parametrization, cfg.rho_min, cfg.rho_max = 0, self.param.rho_min, 1.0
        cfg.homogeneous_boundary = 1 if self.use_homogeneous_boundary else 0
        cfg.chemical_potential = mu
        cfg.target_mass = target_mass
        cfg.boundary_mass = boundary_mass
        cfg.use_monitor = 1 if use_monitor else 0
        cfg.check_interval = self.check_interval
        return cfg

    def _run(self, weights: Weights, rho, mode, mu, target_mass=0.0, boundary_mass=0.0, direction=None,
             use_monitor=None, external_field=None):
        torch = _torch()
        d, host = _dev(rho)
        if not host:
            d = d.clone()
        cfg = self._config(mode, mu, target_mass, boundary_mass, use_monitor)
        vx = None
        if external_field is not None:
            vx, _ = _dev(np.asarray(external_field, dtype=np.float64).reshape(-1)
                         if not hasattr(external_field, "data_ptr") else external_field)
            vx = vx.to(torch.float64).contiguous()
            cfg.external_field = vx.data_ptr()
        res = _lib.CMinimizerResult()
        dirp = None
        if direction is not None:
            dd, _ = _dev(direction)
            dirp = dd.data_ptr()
        ref = self.refine.engine.handle if self.refine is not None else None
        st = _lib.lib().cdft_minimize(weights.engine.handle, ctypes.byref(cfg), d.data_ptr(), dirp, ref,
                                      self.refine_switch, ctypes.byref(res), _stream())
        torch.cuda.synchronize()
        if st != _lib.CDFT_OK:
            msg = _lib.lib().cdft_last_error().decode()
            if res.uphill_error:
                raise RuntimeError(msg)
            _lib.check(st)
        out = d.cpu().numpy() if host else d
        return MinimizationResult([out], res.free_energy, res.grand_potential, res.rms_force, res.iterations,
                                  bool(res.converged))

    def grand_potential(self, model: Model, weights: Weights, initial_density, chemical_potential,
                        external_field=None):
        """minimization.hpp:280-354.  ``external_field`` (N values, or None):
        V_ext / kT of every evaluation (a wall; the reference's Minimizer has
        no field, its profile states drop V_ext)."""
        return self._run(weights, initial_density, 0, chemical_potential, external_field=external_field)

    def fixed_mass(self, model: Model, weights: Weights, initial_density, chemical_potential, target_mass,
                   external_field=None):
        """minimization.hpp:182-278 (``external_field`` as grand_potential)."""
        return self._run(weights, initial_density, 1, chemical_potential, target_mass=target_mass,
                         external_field=external_field)

    def _run_batch(self, weights: Weights, rhos, mode, mus, masses=None):
        torch = _torch()
        e = weights.engine
        B, N = e.batch, e.N
        if isinstance(rhos, np.ndarray) or not hasattr(rhos, "data_ptr"):
            d = torch.tensor(np.asarray(rhos, dtype=np.float64).reshape(B, N), device="cuda")
            host = True
        else:
            d = rhos.reshape(B, N).to(torch.float64).contiguous().clone()
            host = False
        mu = np.ascontiguousarray(np.broadcast_to(np.asarray(mus, dtype=np.float64), (B,)))
        mass = None if masses is None else np.ascontiguousarray(
            np.broadcast_to(np.asarray(masses, dtype=np.float64), (B,)))
        cfg = self._config(mode, 0.0)
        res = (_lib.CMinimizerResult * B)()
        ref = self.refine.engine.handle if self.refine is not None else None
        _lib.check(_lib.lib().cdft_minimize_batch(
            e.handle, ctypes.byref(cfg), mu.ctypes.data_as(_lib.c_double_p),
            None if mass is None else mass.ctypes.data_as(_lib.c_double_p), d.data_ptr(), ref, self.refine_switch,
            res, _stream()))
        torch.cuda.synchronize()
        out = d.cpu().numpy() if host else d
        return [MinimizationResult([out[b]], r.free_energy, r.grand_potential, r.rms_force, r.iterations,
                                   bool(r.converged)) for b, r in enumerate(res)], [bool(r.uphill_error) for r in res]

    def grand_potential_batch(self, model: Model, weights: Weights, initial_densities, chemical_potentials):
        """``grand_potential`` for every problem of a batched engine (make_weights(..., batch=B)):
        initial_densities (B, N), chemical_potentials (B,).  Returns B results."""
        res, uphill = self._run_batch(weights, initial_densities, 0, chemical_potentials)
        if any(uphill):
            raise RuntimeError(f"fire::step: exceeded max uphill steps (problems {np.flatnonzero(uphill).tolist()})")
        return res

    def minimize_group(self, members, mode="grand_potential"):
        """Minimise the problems of several batched engines together -- an
        uneven sweep with one engine per grid size.  ``members``: a list of
        ``(weights, initial_densities (B, N), chemical_potentials (B,),
        target_masses (B,) or None, refine_weights or None)``.  One FIRE step
        of every running member is one graph launch; each problem stops at
        its own convergence.  Returns one list of B results per member."""
        torch = _torch()
        if mode not in ("grand_potential", "fixed_mass"):
            raise ValueError("minimize_group: mode is grand_potential or fixed_mass")
        keep, cm = [], (_lib.CGroupMember * len(members))()
        outs = []
        for m, mem in enumerate(members):
            w, rhos, mus, masses = mem[:4]
            ref = mem[4] if len(mem) > 4 else None
            e = w.engine
            B, N = e.batch, e.N
            if isinstance(rhos, np.ndarray) or not hasattr(rhos, "data_ptr"):
                d = torch.tensor(np.asarray(rhos, dtype=np.float64).reshape(B, N), device="cuda")
                host = True
            else:
                d = rhos.reshape(B, N).to(torch.float64).contiguous().clone()
                host = False
            mu = np.ascontiguousarray(np.broadcast_to(np.asarray(mus, dtype=np.float64), (B,)))
            mass = None if masses is None else np.ascontiguousarray(
                np.broadcast_to(np.asarray(masses, dtype=np.float64), (B,)))
            res = (_lib.CMinimizerResult * B)()
            keep += [d, mu, mass, res]
            cm[m].engine = e.handle
            cm[m].refine = ref.engine.handle if ref is not None else None
            cm[m].refine_switch = self.refine_switch
            cm[m].mu = mu.ctypes.data_as(_lib.c_double_p)
            cm[m].target_mass = None if mass is None else mass.ctypes.data_as(_lib.c_double_p)
            cm[m].rho = d.data_ptr()
            cm[m].results = ctypes.cast(res, ctypes.POINTER(_lib.CMinimizerResult))
            outs.append((d, host, res))
        cfg = self._config(0 if mode == "grand_potential" else 1, 0.0)
        _lib.check(_lib.lib().cdft_minimize_group(len(members), cm, ctypes.byref(cfg), _stream()))
        torch.cuda.synchronize()
        results = []
        for d, host, res in outs:
            out = d.cpu().numpy() if host else d
            results.append([MinimizationResult([out[b]], r.free_energy, r.grand_potential, r.rms_force,
                                               r.iterations, bool(r.converged)) for b, r in enumerate(res)])
            if any(r.uphill_error for r in res):
                bad = [b for b, r in enumerate(res) if r.uphill_error]
                raise RuntimeError(f"fire::step: exceeded max uphill steps (member problems {bad})")
        return results

    def fixed_mass_batch(self, model: Model, weights: Weights, initial_densities, chemical_potentials,
                         target_masses):
        """``fixed_mass`` for every problem of a batched engine; target_masses (B,)."""
        res, uphill = self._run_batch(weights, initial_densities, 1, chemical_potentials, target_masses)
        if any(uphill):
            raise RuntimeError(f"fire::step: exceeded max uphill steps (problems {np.flatnonzero(uphill).tolist()})")
        return res


# ---------------------------------------------------------------- Picard


@dataclass
class FixedMassConstraint:
    """fixed_mass_constraint (minimization.hpp:159-180): after every update
    the excess over the background is rescaled to the target mass."""

    target_masses: list
    backgrounds: list
    cell_volume: float
    min_density: float = 1e-30


def fixed_mass_constraint(target_masses, backgrounds, cell_volume, min_density=1e-30):
    """minimization.hpp:159-180."""
    return FixedMassConstraint(list(np.atleast_1d(np.asarray(target_masses, dtype=np.float64))), list(backgrounds),
                               float(cell_volume), float(min_density))


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
    """picard.hpp:31-42 on the device: rho <- max(rho exp(-mixing force / dV),
    min_density) until the force RMS or the change of Omega falls below the
    tolerance.  log_interval is kept for the interface and prints nothing;
    check_interval is how many iterations run between host checks."""

    mixing: float = 0.01
    min_density: float = 1e-30
    tolerance: float = 1e-6
    max_iterations: int = 5000
    log_interval: int = 500
    check_interval: int = 25

    def _c(self):
        return _lib.CPicardConfig(self.mixing, self.min_density, self.tolerance, 1e-30, self.max_iterations,
                                  self.check_interval)

    def _solve(self, weights: Weights, rho, mus, constraint):
        torch = _torch()
        e = weights.engine
        B, N = e.batch, e.N
        if e.S != 1:
            raise ValueError("Picard: single-species engines")
        if isinstance(rho, np.ndarray) or not hasattr(rho, "data_ptr"):
            d = torch.tensor(np.asarray(rho, dtype=np.float64).reshape(B, N), device="cuda")
            host = True
        else:
            d = rho.reshape(B, N).to(torch.float64).contiguous().clone()
            host = False
        mu = np.ascontiguousarray(np.broadcast_to(np.asarray(mus, dtype=np.float64), (B,)))
        mass = None
        bg = None
        cfg = self._c()
        if constraint is not None:
            if abs(constraint.cell_volume - e.grid.cell_volume) > 1e-12 * e.grid.cell_volume:
                raise ValueError("fixed_mass_constraint: cell_volume differs from the grid's")
            mass = np.ascontiguousarray(np.broadcast_to(np.asarray(constraint.target_masses, dtype=np.float64)
                                                        .reshape(-1)[:B], (B,)))
            if constraint.backgrounds is not None and len(constraint.backgrounds):
                b = np.asarray([np.asarray(x, dtype=np.float64).reshape(-1) for x in constraint.backgrounds])
                bg = torch.tensor(np.broadcast_to(b.reshape(-1, N), (B, N)).copy(), device="cuda")
            cfg.constraint_min_density = constraint.min_density
        res = (_lib.CPicardResult * B)()
        _lib.check(_lib.lib().cdft_picard(
            e.handle, ctypes.byref(cfg), mu.ctypes.data_as(_lib.c_double_p),
            None if mass is None else mass.ctypes.data_as(_lib.c_double_p),
            None if bg is None else bg.data_ptr(), d.data_ptr(), res, _stream()))
        torch.cuda.synchronize()
        out = d.cpu().numpy() if host else d
        return [PicardResult([out[b]], r.grand_potential, r.residual, r.iterations, bool(r.converged))
                for b, r in enumerate(res)]

    def solve(self, densities, weights: Weights, chemical_potential=0.0, constraint: FixedMassConstraint = None):
        """picard.hpp:63-124 for one state (engine batch 1)."""
        if weights.engine.batch != 1:
            raise ValueError("Picard.solve: an engine with batch 1 (solve_batch for more)")
        rho = densities[0] if isinstance(densities, (list, tuple)) else densities
        return self._solve(weights, rho, [chemical_potential], constraint)[0]

    def solve_batch(self, densities, weights: Weights, chemical_potentials, constraint: FixedMassConstraint = None):
        """``solve`` for every problem of a batched engine: densities (B, N),
        chemical_potentials (B,); a constraint's target_masses (B,) and
        backgrounds (B, N) or one background for all."""
        return self._solve(weights, densities, chemical_potentials, constraint)


# ---------------------------------------------------------------- DDFT


@dataclass
class StepConfig:
    """dynamics.hpp:26-33."""

    dt: float = 1e-4
    diffusion_coefficient: float = 1.0
    min_density: float = 1e-18
    dt_max: float = 1.0
    fp_tolerance: float = 1e-4
    fp_max_iterations: int = 100

    def c(self):
        return _lib.CDDFTConfig(self.dt, self.diffusion_coefficient, self.min_density, self.dt_max,
                                self.fp_tolerance, self.fp_max_iterations)


def _set_ddft_refine(weights: Weights, refine, refine_iterations):
    _lib.check(_lib.lib().cdft_ddft_set_refine(weights.engine.handle,
                                               refine.engine.handle if refine is not None else None,
                                               int(refine_iterations) if refine is not None else 0))


def integrating_factor_step(density, weights: Weights, config: StepConfig, chemical_potential=0.0, refine=None,
                            refine_iterations=1):
    """dynamics.hpp:333-401: returns (density, energy, dt_used); config.dt is
    divided by 10 on restarts, as in the reference.  ``refine``: FP64 Weights
    of the same model that run ``refine_iterations`` (>= 0) fixed-point
    iterations after the step has converged with ``weights`` and give its
    final energy (mixed-precision defect correction)."""
    torch = _torch()
    d, host = _dev(density)
    if not host:
        d = d.clone()
    c = config.c()
    e = ctypes.c_double()
    it = ctypes.c_int()
    _set_ddft_refine(weights, refine, refine_iterations)
    try:
        _lib.check(_lib.lib().cdft_ddft_step(weights.engine.handle, ctypes.byref(c), chemical_potential,
                                             d.data_ptr(), ctypes.byref(e), ctypes.byref(it), _stream()))
    finally:
        _set_ddft_refine(weights, None, 0)
    torch.cuda.synchronize()
    config.dt = c.dt
    return (d.cpu().numpy() if host else d), e.value, c.dt


def ddft_last_step(weights: Weights) -> dict:
    """Facts of the last integrating-factor step of these weights' engine:
    fixed-point iterations, restarts, status (1 converged, 2 gave up), whether
    the loop ran on the device (a conditional graph node), and the deviation
    of the last FP64 refinement iteration."""
    info = (ctypes.c_int * 4)()
    dev = ctypes.c_double()
    _lib.check(_lib.lib().cdft_ddft_last_step(weights.engine.handle, info, ctypes.byref(dev)))
    return {"fp_iterations": info[0], "restarts": info[1], "status": info[2], "device_loop": bool(info[3]),
            "refine_deviation": dev.value}


def _ddft_single(fn, density, weights: Weights, config: StepConfig, chemical_potential, with_iterations):
    torch = _torch()
    d, host = _dev(density)
    if not host:
        d = d.clone()
    c = config.c()
    e = ctypes.c_double()
    args = [weights.engine.handle, ctypes.byref(c), chemical_potential, d.data_ptr(), ctypes.byref(e)]
    if with_iterations:
        args.append(ctypes.byref(ctypes.c_int()))
    _lib.check(fn(*args, _stream()))
    torch.cuda.synchronize()
    return (d.cpu().numpy() if host else d), e.value, config.dt


def split_operator_step(density, weights: Weights, config: StepConfig, chemical_potential=0.0):
    """dynamics.hpp:410-465 (Strang splitting: half diffusion, explicit
    excess step, half diffusion); returns (density, energy, dt_used)."""
    return _ddft_single(_lib.lib().cdft_ddft_split_step, density, weights, config, chemical_potential, False)


def crank_nicholson_step(density, weights: Weights, config: StepConfig, chemical_potential=0.0):
    """dynamics.hpp:472-538 (Crank-Nicolson fixed point); returns
    (density, energy, dt_used)."""
    return _ddft_single(_lib.lib().cdft_ddft_cn_step, density, weights, config, chemical_potential, True)


@dataclass
class ReservoirBoundary:
    """reservoir_boundary (dynamics.hpp:551-557): the cells where mask is
    true are reset to reservoir_density after every DDFT step."""

    mask: np.ndarray
    reservoir_density: float


def reservoir_boundary(mask, reservoir_density):
    """dynamics.hpp:551-557."""
    return ReservoirBoundary(np.asarray(mask).reshape(-1).astype(bool), float(reservoir_density))


@dataclass
class Snapshot:
    """dynamics.hpp:45-50."""

    step: int
    time: float
    energy: float
    densities: list


@dataclass
class Simulation:
    """dynamics.hpp:564-693 (integrating-factor DDFT with adaptive dt).

    The steps, the snapshots (copied to pinned host memory while the next
    steps run), the reservoir boundary and the stop test run through one
    call of the device driver.  ``times`` / ``energies`` of the result hold
    the entries the reference records (step 0, every log_interval-th step
    and the last one); ``all_times`` / ``all_energies`` hold every step.
    ``stop_condition(step, time, energy) -> bool`` ends the run early.

    ``anchor`` (FP64 Weights of the same model) with ``anchor_interval`` k > 0
    runs a mixed-precision engine in segments of k steps, each with the
    engine's split anchored at the state the segment starts from (one FP64
    evaluation per segment, cdft_engine_set_anchor): the FP32 round-off then
    scales with how far the density moved within the segment instead of its
    own swing (solids).  The adaptive dt carries over the segments; the
    anchor is cleared after the run.  Snapshots are then taken between
    segments: snapshot_interval must be a multiple of anchor_interval.
    """

    step: StepConfig = field(default_factory=StepConfig)
    n_steps: int = 1000
    snapshot_interval: int = 100
    log_interval: int = 50
    energy_offset: float = 0.0
    boundary: ReservoirBoundary = None
    stop_condition: object = None
    # FP64 defect correction of a mixed-precision run (see integrating_factor_step)
    refine: object = None
    refine_iterations: int = 1
    # anchored split of a mixed-precision run, re-anchored every anchor_interval steps
    anchor: object = None
    anchor_interval: int = 0

    def run(self, densities, weights: Weights, chemical_potential=0.0):
        torch = _torch()
        d, host = _dev(densities[0] if isinstance(densities, (list, tuple)) else densities)
        if not host:
            d = d.clone()
        n = d.numel()
        dv = weights.engine.grid.cell_volume
        c = self.step.c()
        times = np.zeros(self.n_steps + 1)
        energies = np.zeros(self.n_steps + 1)
        cap = 0
        if self.snapshot_interval > 0:
            cap = 1 + self.n_steps // self.snapshot_interval
        snaps = torch.empty((max(cap, 1), n), dtype=torch.float64).pin_memory() if cap else None
        snap_steps = (ctypes.c_int * max(cap, 1))()
        count = ctypes.c_int()
        done = ctypes.c_int()
        mask_dev = None
        res_density = 0.0
        if self.boundary is not None:
            m = np.asarray(self.boundary.mask).reshape(-1)
            if m.size != n:
                raise ValueError("reservoir mask: one entry per grid point")
            mask_dev = torch.tensor(m.astype(np.uint8), device="cuda")
            res_density = self.boundary.reservoir_density
        err = []
        offset = [0, 0.0]  # steps and time before the current segment

        def _stop(step, time, energy, _user):
            try:
                return 1 if self.stop_condition(step + offset[0], time + offset[1], energy) else 0
            except Exception as exc:  # surfaced after the run
                err.append(exc)
                return 1

        cb = _lib.STOP_FN(_stop) if self.stop_condition is not None else _lib.STOP_FN()
        if mask_dev is not None:
            d.masked_fill_(mask_dev.bool(), res_density)  # the driver applies it too; the initial mass needs it
        mass_initial = float(torch.sum(d).item()) * dv
        anchored = self.anchor is not None and self.anchor_interval > 0
        if anchored and self.snapshot_interval > 0 and self.snapshot_interval % self.anchor_interval:
            raise ValueError("anchored DDFT: snapshot_interval must be a multiple of anchor_interval")
        seg_len = self.anchor_interval if anchored else self.n_steps
        snapshots = []
        steps = 0

        def take(step, x):  # a snapshot between anchored segments
            rho_k = x.cpu().numpy().copy() if host else x.clone()
            snapshots.append(Snapshot(step, float(times[step]), float(energies[step]), [rho_k]))

        initial = d.clone() if anchored and self.snapshot_interval > 0 else None

        _set_ddft_refine(weights, self.refine, self.refine_iterations)
        try:
            while True:
                k = min(seg_len, self.n_steps - steps)
                if anchored:
                    weights.engine.set_anchor(self.anchor.engine, d)
                ts = np.zeros(k + 1)
                es = np.zeros(k + 1)
                scap = 1 + k // self.snapshot_interval if self.snapshot_interval > 0 and not anchored else 0
                _lib.check(_lib.lib().cdft_ddft_simulate(
                    weights.engine.handle, ctypes.byref(c), chemical_potential, k, d.data_ptr(),
                    ts.ctypes.data_as(_lib.c_double_p), es.ctypes.data_as(_lib.c_double_p),
                    self.snapshot_interval if scap else 0,
                    ctypes.cast(snaps.data_ptr(), _lib.c_double_p) if snaps is not None else None,
                    snap_steps, scap, ctypes.byref(count), mask_dev.data_ptr() if mask_dev is not None else None,
                    res_density, cb, None, ctypes.byref(done), _stream()))
                torch.cuda.synchronize()
                got = done.value
                first = steps == 0
                times[steps:steps + got + 1] = ts[:got + 1] + offset[1]
                if first:
                    energies[:got + 1] = es[:got + 1]
                else:  # step 0 of a segment repeats the previous segment's last
                    energies[steps + 1:steps + got + 1] = es[1:got + 1]
                for q in range(count.value if scap else 0):
                    st = snap_steps[q]
                    rho_k = snaps[q].numpy().copy() if host else snaps[q].to(d.device)
                    snapshots.append(Snapshot(st, float(times[st]), float(energies[st]), [rho_k]))
                if initial is not None and first:
                    take(0, initial)
                steps += got
                if anchored and self.snapshot_interval > 0 and got and steps % self.snapshot_interval == 0:
                    take(steps, d)
                offset[0], offset[1] = steps, float(times[steps])
                if got < k or steps >= self.n_steps or err:
                    break
        finally:
            _set_ddft_refine(weights, None, 0)
            if anchored:
                weights.engine.clear_anchor()
        if err:
            raise err[0]
        idx = [0]
        if self.log_interval > 0:
            idx += [s for s in range(1, steps + 1) if s % self.log_interval == 0 or s == self.n_steps]
        out = d.cpu().numpy() if host else d
        return {"densities": [out], "times": [float(times[i]) for i in idx],
                "energies": [float(energies[i]) for i in idx], "snapshots": snapshots,
                "mass_initial": mass_initial, "mass_final": float(torch.sum(d).item()) * dv, "dt": c.dt,
                "steps": steps, "all_times": times[:steps + 1], "all_energies": energies[:steps + 1]}


# ---------------------------------------------------------- saddle point


def hessian_times_vector(weights: Weights, rho, v, chemical_potential=0.0, exact=True, eps=1e-6,
                         fixed_boundary=False, force_at_rho=None):
    """H v of Omega at rho: exact (forward-over-reverse) or the reference's
    forward difference (saddle_point.hpp:30-39)."""
    torch = _torch()
    r, host = _dev(rho)
    vv, _ = _dev(v)
    hv = torch.empty_like(r)
    b = 1 if fixed_boundary else 0
    L = _lib.lib()
    if exact:
        _lib.check(L.cdft_hvp(weights.engine.handle, r.data_ptr(), vv.data_ptr(), chemical_potential, b,
                              hv.data_ptr(), _stream()))
    else:
        if force_at_rho is None:
            f0 = torch.empty_like(r)
            sc = torch.empty(10, dtype=torch.float64, device=r.device)
            weights.engine.total_device(r.data_ptr(), None, [chemical_potential], f0.data_ptr(), sc.data_ptr(),
                                        _stream())
            if fixed_boundary:
                mask = torch.tensor(weights_mask(weights), device=r.device, dtype=torch.bool)
                f0[mask] = 0.0
        else:
            f0, _ = _dev(force_at_rho)
        _lib.check(L.cdft_hvp_fd(weights.engine.handle, r.data_ptr(), f0.data_ptr(), vv.data_ptr(),
                                 chemical_potential, eps, b, hv.data_ptr(), _stream()))
    torch.cuda.synchronize()
    return hv.cpu().numpy() if host else hv


def weights_mask(weights: Weights):
    g = weights.engine.grid
    return g.boundary_mask().astype(bool)


@dataclass
class EigenvalueResult:
    """saddle_point.hpp:151-156."""

    eigenvector: object
    eigenvalue: float
    iterations: int
    converged: bool


@dataclass
class EigenvalueSolver:
    """saddle_point.hpp:158-169 (``exact_hvp`` replaces the FD product).

    ``method="lanczos"`` replaces the reference's 3-vector Rayleigh-Ritz
    iteration by block Lanczos on exact products of the same operator (the
    fixed-boundary Hessian, restricted to the interior): ``block`` directions
    per batched product, ``max_basis`` blocks before a restart, the host
    checking every ``check_interval`` products.  ``solve(..., hvp_weights=w)``
    takes the products from ``w.engine`` (same model, batch = ``block``; e.g.
    an FP64 engine under a mixed-precision one)."""

    tolerance: float = 1e-4
    max_iterations: int = 300
    hessian_eps: float = 1e-6
    exact_hvp: bool = False
    seed: int = 42
    method: str = "rayleigh_ritz"
    block: int = 1
    max_basis: int = 32
    check_interval: int = 4

    def c(self):
        if self.method not in ("rayleigh_ritz", "lanczos"):
            raise ValueError(f"unknown eigen method {self.method!r}")
        m = _lib.EIGEN_LANCZOS if self.method == "lanczos" else _lib.EIGEN_RAYLEIGH_RITZ
        return _lib.CEigenConfig(self.tolerance, self.max_iterations, self.hessian_eps, 1 if self.exact_hvp else 0,
                                 self.seed, m, self.block, self.max_basis, self.check_interval)

    def solve(self, weights: Weights, rho, chemical_potential=0.0, initial_guess=None, hvp_weights=None):
        torch = _torch()
        r, host = _dev(rho)
        if initial_guess is not None:
            vec, _ = _dev(initial_guess)
            vec = vec.clone()
        else:
            vec = torch.empty_like(r)
        ev = ctypes.c_double()
        it = ctypes.c_int()
        cv = ctypes.c_int()
        c = self.c()
        _lib.check(_lib.lib().cdft_eigen_solve_ex(weights.engine.handle,
                                                  hvp_weights.engine.handle if hvp_weights is not None else None,
                                                  ctypes.byref(c), r.data_ptr(), chemical_potential, vec.data_ptr(),
                                                  1 if initial_guess is not None else 0, ctypes.byref(ev),
                                                  ctypes.byref(it), ctypes.byref(cv), _stream()))
        torch.cuda.synchronize()
        return EigenvalueResult(vec.cpu().numpy() if host else vec, ev.value, it.value, bool(cv.value))


@dataclass
class SaddleResult:
    """saddle_point.hpp:313-320."""

    density: object
    eigenvector: object
    grand_potential: float
    eigenvalue: float
    outer_iterations: int
    converged: bool
    eigen_iterations: int = 0  # products of the eigen solves, summed over the outer iterations
    fire_steps: int = 0        # projected FIRE steps, summed over the outer iterations


@dataclass
class Search:
    """saddle_point.hpp:324-353 (same defaults)."""

    fire: Fire = field(default_factory=lambda: Fire(dt=1e-3, dt_max=1.0, alpha_start=0.01, f_alpha=1.0,
                                                    force_tolerance=1e-4, max_steps=100000))
    eigenvalue: EigenvalueSolver = field(default_factory=lambda: EigenvalueSolver(1e-4, 300, 1e-6))
    param: Unbounded = field(default_factory=lambda: Unbounded(1e-18))
    omega_tolerance: float = 1e-5
    tolerance_start: float = 1e-3
    tolerance_factor: float = 10.0
    max_outer_iterations: int = 20
    eigenvalue_clear_count: int = 2

    # FP64 defect correction of a mixed-precision search: the FP64 `refine`
    # weights take over each projected FIRE run once its rms force is below
    # refine_switch times the run's tolerance
    refine: object = None
    refine_switch: float = 10.0
    # product engine of a Lanczos eigen solve (batch = eigenvalue.block)
    hvp_weights: object = None

    def find(self, model: Model, weights: Weights, initial_density, chemical_potential, target_mass):
        torch = _torch()
        r, host = _dev(initial_density)
        r = r.clone()
        ev = torch.empty_like(r)
        cfg = _lib.CSaddleConfig(self.fire.c(), self.eigenvalue.c(), self.param.rho_min, self.omega_tolerance,
                                 self.tolerance_start, self.tolerance_factor, self.max_outer_iterations,
                                 self.eigenvalue_clear_count)
        out = (ctypes.c_double * 2)()
        counts = (ctypes.c_int * 3)()
        cv = ctypes.c_int()
        _lib.check(_lib.lib().cdft_saddle_find_ex(
            weights.engine.handle, self.refine.engine.handle if self.refine is not None else None,
            self.hvp_weights.engine.handle if self.hvp_weights is not None else None, self.refine_switch,
            ctypes.byref(cfg), r.data_ptr(), chemical_potential, target_mass, ev.data_ptr(), out, counts,
            ctypes.byref(cv), _stream()))
        torch.cuda.synchronize()
        conv = (lambda t: t.cpu().numpy()) if host else (lambda t: t)
        return SaddleResult(conv(r), conv(ev), out[0], out[1], counts[0], bool(cv.value), counts[1], counts[2])
