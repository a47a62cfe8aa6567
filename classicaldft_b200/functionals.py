"""Host-side mirror of the reference's functional API, backed by the GPU engine.

Names, argument meaning and error behaviour follow the reference
(include/dft/grid.hpp, types.hpp, physics/{potentials,interactions,model}.hpp,
functionals/{functionals,functional,types}.hpp); every evaluation runs
through the C ABI of libcdft_b200.so on the current CUDA device.
"""
from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass, field

import numpy as np

from . import _lib

# ----------------------------------------------------------------- grid


@dataclass(frozen=True)
class Grid:
    """grid.hpp:26-83: periodic uniform grid, z-fastest flat index."""

    dx: float
    box_size: tuple
    shape: tuple

    @property
    def cell_volume(self) -> float:
        return self.dx * self.dx * self.dx

    @property
    def total_points(self) -> int:
        return int(self.shape[0] * self.shape[1] * self.shape[2])

    def flat_index(self, ix, iy, iz):
        return iz + self.shape[2] * (iy + self.shape[1] * ix)

    def boundary_mask(self) -> np.ndarray:
        """grid.hpp:67-82."""
        nx, ny, nz = self.shape
        m = np.zeros(self.shape, dtype=np.uint8)
        m[[0, nx - 1], :, :] = 1
        m[:, [0, ny - 1], :] = 1
        m[:, :, [0, nz - 1]] = 1
        return m.reshape(-1)


def make_grid(dx: float, box) -> Grid:
    """grid.hpp:87-108: raises ValueError (std::invalid_argument) on bad input."""
    if dx <= 0.0:
        raise ValueError(f"make_grid: dx must be positive, got {dx}")
    shape = []
    for b in box:
        if b <= 0.0:
            raise ValueError(f"make_grid: box dimension must be positive, got {b}")
        n = b / dx
        ni = int(round(n))
        if abs(n - ni) > 1e-10:
            raise ValueError(f"make_grid: box dimension {b} is not commensurate with dx={dx}")
        shape.append(ni)
    return Grid(dx=float(dx), box_size=tuple(float(b) for b in box), shape=tuple(shape))


# ------------------------------------------------------------ potentials

WEEKS_CHANDLER_ANDERSEN = "WeeksChandlerAndersen"
BARKER_HENDERSON = "BarkerHenderson"
_SPLIT = {WEEKS_CHANDLER_ANDERSEN: _lib.SPLIT_WCA, BARKER_HENDERSON: _lib.SPLIT_BH}
# pointwise kernel variants of the TMA path (CDFT_POINTWISE_VARIANTS)
POINTWISE_VARIANTS = 6


@dataclass
class Potential:
    """potentials.hpp:248-307: LennardJones / TenWoldeFrenkel / WRDF."""

    type: int
    sigma: float
    epsilon: float
    r_cutoff: float
    alpha: float = 50.0

    def _c(self):
        return _lib.CPotential(self.type, self.sigma, self.epsilon, self.r_cutoff, self.alpha)

    def info(self):
        out = (ctypes.c_double * 4)()
        _lib.check(_lib.lib().cdft_potential_info(ctypes.byref(self._c()), out))
        return {"epsilon_shift": out[0], "r_min": out[1], "v_min": out[2], "r_zero": out[3]}

    def attractive(self, r, split=WEEKS_CHANDLER_ANDERSEN):
        r = np.ascontiguousarray(np.atleast_1d(r), dtype=np.float64)
        out = np.empty_like(r)
        _lib.check(_lib.lib().cdft_potential_attractive(
            ctypes.byref(self._c()), _SPLIT[split], r.ctypes.data_as(_lib.c_double_p), r.size,
            out.ctypes.data_as(_lib.c_double_p)))
        return out

    def hard_sphere_diameter(self, kT, split=WEEKS_CHANDLER_ANDERSEN) -> float:
        d = ctypes.c_double()
        _lib.check(_lib.lib().cdft_hard_sphere_diameter(ctypes.byref(self._c()), kT, _SPLIT[split], ctypes.byref(d)))
        return d.value

    def vdw_integral(self, kT, split=WEEKS_CHANDLER_ANDERSEN) -> float:
        d = ctypes.c_double()
        _lib.check(_lib.lib().cdft_vdw_integral(ctypes.byref(self._c()), kT, _SPLIT[split], ctypes.byref(d)))
        return d.value


def make_lennard_jones(sigma, epsilon, r_cutoff=-1.0) -> Potential:
    """potentials.hpp:311-325."""
    return Potential(_lib.POT_LJ, sigma, epsilon, r_cutoff)


def make_ten_wolde_frenkel(sigma, epsilon, r_cutoff=-1.0, alpha=50.0) -> Potential:
    """potentials.hpp:327-346."""
    return Potential(_lib.POT_TWF, sigma, epsilon, r_cutoff, alpha)


def make_wang_ramirez_dobnikar_frenkel(sigma, epsilon, r_cutoff=3.0) -> Potential:
    """potentials.hpp:348-368."""
    return Potential(_lib.POT_WRDF, sigma, epsilon, r_cutoff)


# -------------------------------------------------------- model / species


@dataclass
class Species:
    """types.hpp:25-28."""

    name: str
    hard_sphere_diameter: float


@dataclass
class Interaction:
    """interactions.hpp:23-30."""

    species_i: int
    species_j: int
    potential: Potential
    split: str = WEEKS_CHANDLER_ANDERSEN
    weight_scheme: str = "InterpolationQuadraticF"


@dataclass
class Model:
    """physics/model.hpp:15-20."""

    grid: Grid
    species: list
    interactions: list = field(default_factory=list)
    temperature: float = 1.0


@dataclass(frozen=True)
class FMTModel:
    """fmt/models.hpp:363-419: Rosenfeld, RSLT, WhiteBearI, WhiteBearII, esFMT(A, B)."""

    name: str
    A: float = 1.0
    B: float = 0.0

    def __post_init__(self):
        if self.name not in _lib.MODEL_IDS:
            raise ValueError(f"Unknown FMT model: {self.name}")

    @property
    def needs_tensor(self) -> bool:
        return self.name in ("WhiteBearI", "WhiteBearII", "esFMT")

    @staticmethod
    def from_name(name: str) -> "FMTModel":
        return FMTModel(name)


def Rosenfeld():
    return FMTModel("Rosenfeld")


def RSLT():
    return FMTModel("RSLT")


def WhiteBearI():
    return FMTModel("WhiteBearI")


def WhiteBearII():
    return FMTModel("WhiteBearII")


def EsFMT(A=1.0, B=0.0):
    return FMTModel("esFMT", A, B)


def interaction_weight(inter: Interaction, grid: Grid, kT: float):
    """mean_field.hpp:146-196 up to the FFT: (real-space weight * dV/N, a_vdw)."""
    out = np.empty(grid.total_points, dtype=np.float64)
    a = ctypes.c_double()
    _lib.check(_lib.lib().cdft_interaction_weight(
        _lib.c_long3(*grid.shape), grid.dx, ctypes.byref(inter.potential._c()), _SPLIT[inter.split],
        _lib.WEIGHT_SCHEMES[inter.weight_scheme], kT, out.ctypes.data_as(_lib.c_double_p), ctypes.byref(a)))
    return out, a.value


# ------------------------------------------------------------------ engine


class Engine:
    """An evaluation engine on the current CUDA device (owns a cdft_engine).

    ``batch`` > 1 builds a batched engine: every call evaluates ``batch``
    problems of this model at once (arrays carry a leading batch axis).
    ``weights_on``: "device" builds the mean-field cell weights on the GPU
    (cdft_create_model); "host" runs the set-up loop of mean_field.hpp:146-196
    on the CPU (cdft_interaction_weight) and uploads the result.
    """

    def __init__(self, fmt_model: FMTModel, model: Model, precision: int = _lib.FP64, batch: int = 1,
                 weights_on: str = "device"):
        L = _lib.lib()
        g = model.grid
        diam = np.array([sp.hard_sphere_diameter for sp in model.species], dtype=np.float64)
        h = ctypes.c_void_p()
        M = len(model.interactions)
        if weights_on == "device":
            inters = (_lib.CModelInteraction * max(1, M))()
            for m, it in enumerate(model.interactions):
                inters[m] = _lib.CModelInteraction(it.species_i, it.species_j, it.potential._c(), _SPLIT[it.split],
                                                   _lib.WEIGHT_SCHEMES[it.weight_scheme])
            _lib.check(L.cdft_create_model(ctypes.byref(h), _lib.c_long3(*g.shape), g.dx, len(model.species),
                                           diam.ctypes.data_as(_lib.c_double_p), _lib.MODEL_IDS[fmt_model.name],
                                           fmt_model.A, fmt_model.B, M, inters, model.temperature, precision,
                                           int(batch)))
            a = ctypes.c_double()
            self.a_vdw = []
            for m in range(M):
                _lib.check(L.cdft_engine_a_vdw(h, m, ctypes.byref(a)))
                self.a_vdw.append(a.value)
        elif weights_on == "host":
            keep = []
            inters = (_lib.CInteraction * max(1, M))()
            self.a_vdw = []
            for m, it in enumerate(model.interactions):
                w, a = interaction_weight(it, g, model.temperature)
                keep.append(w)
                inters[m] = _lib.CInteraction(it.species_i, it.species_j, w.ctypes.data_as(_lib.c_double_p), a)
                self.a_vdw.append(a)
            _lib.check(L.cdft_create_batch(ctypes.byref(h), _lib.c_long3(*g.shape), g.dx, len(model.species),
                                           diam.ctypes.data_as(_lib.c_double_p), _lib.MODEL_IDS[fmt_model.name],
                                           fmt_model.A, fmt_model.B, M, inters, precision, int(batch)))
        else:
            raise ValueError('weights_on: "device" or "host"')
        self.weights_on = weights_on
        self.handle = h
        self.grid = g
        self.S = len(model.species)
        self.N = g.total_points
        self.precision = precision
        b = ctypes.c_int()
        _lib.check(L.cdft_engine_batch(h, ctypes.byref(b)))
        self.batch = b.value
        self.info = self._query_info()

    def _query_info(self):
        info = (ctypes.c_longlong * 8)()
        _lib.check(_lib.lib().cdft_engine_info(self.handle, info))
        return {"N": info[0], "Nk": info[1], "S": info[2], "channels": info[3], "deriv_channels": info[4],
                "precision": info[5], "kernels_per_eval": info[6], "scratch_bytes": info[7]}

    def close(self):
        if getattr(self, "handle", None):
            _lib.lib().cdft_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _mu(self, mu):
        """beta*mu as a contiguous (S,) or (B, S) array; B values for one species broadcast per problem."""
        lead = (self.S,) if self.batch == 1 else (self.batch, self.S)
        m = np.asarray(mu, dtype=np.float64)
        if self.batch > 1 and self.S == 1 and m.ndim == 1 and m.size == self.batch:
            m = m[:, None]
        return np.ascontiguousarray(np.broadcast_to(m, lead))

    def total_host(self, rho: np.ndarray, mu, vext=None, want_force=True):
        """cdft_total on host arrays: rho (S, N) -> (scalars[10], force (S, N) or None).

        A batched engine takes rho (B, S, N) and mu (B, S) (or broadcastable)
        and returns scalars (B, 10) and force (B, S, N).
        """
        lead = (self.S,) if self.batch == 1 else (self.batch, self.S)
        rho = np.ascontiguousarray(rho, dtype=np.float64).reshape(*lead, self.N)
        mu = self._mu(mu)
        v = None if vext is None else np.ascontiguousarray(vext, dtype=np.float64).reshape(*lead, self.N)
        force = np.empty((*lead, self.N)) if want_force else None
        sc = np.empty(_lib.SCALAR_COUNT if self.batch == 1 else (self.batch, _lib.SCALAR_COUNT))
        _lib.check(_lib.lib().cdft_total(self.handle, rho.ctypes.data, None if v is None else v.ctypes.data,
                                         mu.ctypes.data_as(_lib.c_double_p),
                                         None if force is None else force.ctypes.data,
                                         sc.ctypes.data_as(_lib.c_double_p)))
        return sc, force

    def total_stream_ptrs(self, rho_ptrs, mu, force_ptrs=None, vext_ptrs=None):
        """cdft_total_stream on host addresses (one per state; page-locked
        memory lets the copies overlap the evaluations).  ``mu``: (count, S)
        or (count, B, S) values.  Returns the scalars, (count, 10) or
        (count, B, 10)."""
        count = len(rho_ptrs)
        lead = (self.S,) if self.batch == 1 else (self.batch, self.S)
        m = np.ascontiguousarray(np.broadcast_to(np.asarray(mu, dtype=np.float64), (count, *lead)))
        arr = ctypes.c_void_p * max(count, 1)
        rp = arr(*rho_ptrs)
        fp = None if force_ptrs is None else arr(*force_ptrs)
        vp = None if vext_ptrs is None else arr(*vext_ptrs)
        sc = np.empty((count, _lib.SCALAR_COUNT) if self.batch == 1 else (count, self.batch, _lib.SCALAR_COUNT))
        _lib.check(_lib.lib().cdft_total_stream(self.handle, count, rp, vp, m.ctypes.data_as(_lib.c_double_p), fp,
                                                sc.ctypes.data_as(_lib.c_double_p)))
        return sc

    def total_stream(self, rhos, mus, vexts=None, want_force=True):
        """cdft_total_stream on a list of host states, each shaped as for
        total_host.  Returns (scalars per state, forces per state or None)."""
        lead = (self.S,) if self.batch == 1 else (self.batch, self.S)
        rs = [np.ascontiguousarray(r, dtype=np.float64).reshape(*lead, self.N) for r in rhos]
        vs = None
        if vexts is not None:
            vs = [None if v is None else np.ascontiguousarray(v, dtype=np.float64).reshape(*lead, self.N)
                  for v in vexts]
        fs = [np.empty((*lead, self.N)) for _ in rs] if want_force else None
        mu = np.stack([self._mu(m) for m in mus]) if len(rs) else np.zeros((0, *lead))
        sc = self.total_stream_ptrs([r.ctypes.data for r in rs], mu,
                                    None if fs is None else [f.ctypes.data for f in fs],
                                    None if vs is None else [None if v is None else v.ctypes.data for v in vs])
        return sc, fs

    STAGES = ("split", "r2c_rho", "k_forward", "c2r_channels", "pointwise", "r2c_derivatives", "k_backward",
              "c2r_force", "epilogue", "reduce")
    STAGES_FUSED = ("-0", "plane_fwd_rho", "col_fwd", "plane_inv_channels", "pointwise",
                    "plane_fwd_derivatives", "col_bwd", "plane_inv_epilogue", "-8", "-9")

    @property
    def transforms(self) -> str:
        """"fused" (hand-written plane/column FFT kernels) or "cufft"."""
        t, a = ctypes.c_int(), ctypes.c_int()
        _lib.check(_lib.lib().cdft_engine_transforms(self.handle, ctypes.byref(t), ctypes.byref(a)))
        return "fused" if t.value == _lib.TRANSFORMS_FUSED else "cufft"

    @property
    def fused_available(self) -> bool:
        t, a = ctypes.c_int(), ctypes.c_int()
        _lib.check(_lib.lib().cdft_engine_transforms(self.handle, ctypes.byref(t), ctypes.byref(a)))
        return bool(a.value)

    def set_transforms(self, which: str):
        """Select "fused" (where available) or "cufft"; ValueError if fused is unavailable."""
        if which not in ("fused", "cufft"):
            raise ValueError("transforms: 'fused' or 'cufft'")
        _lib.check(_lib.lib().cdft_engine_set_transforms(
            self.handle, _lib.TRANSFORMS_FUSED if which == "fused" else _lib.TRANSFORMS_CUFFT))
        self.info = self._query_info()

    def set_plane_chunks(self, chunks: int):
        """Run the fused path's middle stages (inverse plane pass, pointwise,
        derivative plane pass) as `chunks` groups of x planes on forked
        streams (1: back to back).  Forces are unchanged; the scalars only
        by summation order.  ValueError without the fused path or for a
        count outside 1..8 or not dividing nx."""
        _lib.check(_lib.lib().cdft_engine_set_plane_chunks(self.handle, int(chunks)))
        self.info = self._query_info()

    def autotune(self, rho_ptr: int, vext_ptr: int = 0, mu=None, stream: int = 0, reps: int = 5):
        """Time every plane-chunk count of the fused path on a device state
        (rho_ptr / vext_ptr: device addresses as for total_device) and keep
        the fastest, also for engines of the same shape created later.
        Returns (chunks, {count: ms per evaluation})."""
        chunks = ctypes.c_int()
        ms = (ctypes.c_double * 8)()
        mu_arr = None
        if mu is not None:
            mu_arr = (ctypes.c_double * (self.batch * self.S))(*[float(m) for m in mu])
        _lib.check(_lib.lib().cdft_engine_autotune(self.handle, ctypes.c_void_p(rho_ptr),
                                                   ctypes.c_void_p(vext_ptr or None), mu_arr,
                                                   ctypes.c_void_p(stream or None), int(reps),
                                                   ctypes.byref(chunks), ms))
        self.info = self._query_info()
        return chunks.value, {k + 1: ms[k] for k in range(8) if ms[k] > 0.0}

    def autotune_ex(self, rho_ptr: int, vext_ptr: int = 0, mu=None, stream: int = 0, reps: int = 5):
        """Time every (plane-chunk count, pointwise variant, column tile,
        pointwise spread, middle plane width) combination the engine has and
        keep the fastest.  Returns ((chunks, variant, tile, spread),
        {(tile, variant, count, spread): ms}), each entry the faster of the
        two plane widths (``plane_width`` gives the one kept)."""
        choice = (ctypes.c_int * 4)()
        ms = (ctypes.c_double * (2 * POINTWISE_VARIANTS * 8 * 4))()
        mu_arr = None
        if mu is not None:
            mu_arr = (ctypes.c_double * (self.batch * self.S))(*[float(m) for m in mu])
        _lib.check(_lib.lib().cdft_engine_autotune_ex(self.handle, ctypes.c_void_p(rho_ptr),
                                                      ctypes.c_void_p(vext_ptr or None), mu_arr,
                                                      ctypes.c_void_p(stream or None), int(reps), choice, ms))
        self.info = self._query_info()
        idx = {(16 << t, v, k + 1, 1 << d): ((t * POINTWISE_VARIANTS + v) * 8 + k) * 4 + d
               for t in range(2) for v in range(POINTWISE_VARIANTS) for k in range(8) for d in range(4)}
        return (choice[0], choice[1], choice[2], choice[3]), {key: ms[i] for key, i in idx.items() if ms[i] > 0.0}

    def set_anchor(self, fp64_engine: "Engine", rho_anchor, stream: int = 0):
        """Anchored split (cdft_engine_set_anchor): ``rho_anchor`` a device
        tensor (B*S*N doubles) or a host array; ``fp64_engine`` an FP64 engine
        of the same model and batch."""
        torch = None
        if hasattr(rho_anchor, "data_ptr"):
            ptr = rho_anchor.data_ptr()
            keep = rho_anchor
        else:
            import torch
            keep = torch.tensor(np.ascontiguousarray(rho_anchor, dtype=np.float64).reshape(-1), device="cuda")
            ptr = keep.data_ptr()
        _lib.check(_lib.lib().cdft_engine_set_anchor(self.handle, fp64_engine.handle, ptr, stream))
        del keep, torch

    def clear_anchor(self):
        _lib.check(_lib.lib().cdft_engine_clear_anchor(self.handle))

    @property
    def anchored(self) -> bool:
        a = ctypes.c_int()
        _lib.check(_lib.lib().cdft_engine_anchored(self.handle, ctypes.byref(a)))
        return bool(a.value)

    @property
    def dependent_launch(self) -> bool:
        """Programmatic dependent launch between the fused path's passes."""
        w = ctypes.c_int()
        _lib.check(_lib.lib().cdft_engine_set_dependent_launch(self.handle, -1, ctypes.byref(w)))
        return bool(w.value)

    def set_dependent_launch(self, on: bool):
        _lib.check(_lib.lib().cdft_engine_set_dependent_launch(self.handle, 1 if on else 0, None))

    @property
    def pointwise_spread(self) -> int:
        """Divisor of the pointwise grid per plane chunk (0: the chunk count)."""
        d = ctypes.c_int()
        _lib.check(_lib.lib().cdft_engine_pointwise_spread(self.handle, ctypes.byref(d)))
        return d.value

    def set_pointwise_spread(self, spread: int):
        _lib.check(_lib.lib().cdft_engine_set_pointwise_spread(self.handle, int(spread)))

    @property
    def column_tile(self) -> int:
        """Columns per tile of the fused column passes (0 without the fused path)."""
        t = ctypes.c_int()
        _lib.check(_lib.lib().cdft_engine_column_tile(self.handle, ctypes.byref(t)))
        return t.value

    def set_column_tile(self, tile: int):
        _lib.check(_lib.lib().cdft_engine_set_column_tile(self.handle, int(tile)))

    @property
    def plane_width(self) -> int:
        """Threads per CTA of the fused path's middle plane passes: 0 the base width, 1 twice it
        (-1 without the fused path)."""
        w = ctypes.c_int()
        _lib.check(_lib.lib().cdft_engine_plane_width(self.handle, ctypes.byref(w)))
        return w.value

    def set_plane_width(self, wide: int):
        _lib.check(_lib.lib().cdft_engine_set_plane_width(self.handle, int(wide)))

    @property
    def pointwise(self) -> int:
        """Pointwise kernel variant: 0 generic; one species: 1 / 2 (5 / 6 CTAs per SM), 3 the branch-free
        FP64 path, 4 / 5 the same with two points per thread (3 / 4 CTAs per SM)."""
        v, a = ctypes.c_int(), ctypes.c_int()
        _lib.check(_lib.lib().cdft_engine_pointwise(self.handle, ctypes.byref(v), ctypes.byref(a)))
        return v.value

    @property
    def pointwise_variants(self) -> list:
        v, a = ctypes.c_int(), ctypes.c_int()
        _lib.check(_lib.lib().cdft_engine_pointwise(self.handle, ctypes.byref(v), ctypes.byref(a)))
        return list(range(POINTWISE_VARIANTS)) if a.value else [0]

    def set_pointwise(self, variant: int):
        _lib.check(_lib.lib().cdft_engine_set_pointwise(self.handle, int(variant)))

    def stage_timing(self, on: bool = True):
        """Record CUDA events between the evaluation stages (synchronises each evaluation)."""
        _lib.check(_lib.lib().cdft_engine_stage_timing(self.handle, 1 if on else 0))

    def stage_times(self):
        """({stage: accumulated ms}, evaluations) since the last call."""
        ms = (ctypes.c_double * len(self.STAGES))()
        n = ctypes.c_longlong()
        _lib.check(_lib.lib().cdft_engine_stage_times(self.handle, ms, ctypes.byref(n)))
        names = self.STAGES_FUSED if self.transforms == "fused" else self.STAGES
        return dict(zip(names, list(ms))), n.value

    def total_device(self, rho_ptr: int, vext_ptr, mu, force_ptr: int, scalars_ptr: int, stream: int = 0):
        """cdft_total_device on device pointers (ints, e.g. torch.Tensor.data_ptr())."""
        mu = self._mu(mu)
        _lib.check(_lib.lib().cdft_total_device(self.handle, rho_ptr, vext_ptr or None,
                                                mu.ctypes.data_as(_lib.c_double_p), force_ptr, scalars_ptr,
                                                stream or None))


@dataclass
class Weights:
    """functionals.hpp:19-23 with the grid weights resident on the GPU."""

    fmt_model: FMTModel
    engine: Engine

    @property
    def a_vdw(self):
        return list(self.engine.a_vdw)


def make_weights(fmt_model: FMTModel, model: Model, precision: int = _lib.FP64, batch: int = 1,
                 weights_on: str = "device") -> Weights:
    """functionals.hpp:27-33 (``batch`` > 1: a batched engine, see ``total_batch``;
    ``weights_on``: where the mean-field cell weights are made, see ``Engine``)."""
    return Weights(fmt_model, Engine(fmt_model, model, precision, batch, weights_on))


@dataclass
class Result:
    """functionals/types.hpp:18-23 (plus the per-term parts and N_s)."""

    free_energy: float
    grand_potential: float
    forces: list
    parts: dict = field(default_factory=dict)


def total(model: Model, rhos, weights: Weights, mus=None, vexts=None) -> Result:
    """functionals.hpp:64-95: F = F_id + F_ext + F_hs + F_mf, Omega = F - sum mu N.

    ``rhos`` is one profile per species (or an (S, N) array), ``mus`` the
    beta*mu per species (default 0), ``vexts`` optional external fields.
    """
    S = len(model.species)
    N = model.grid.total_points
    rho = np.stack([np.asarray(r, dtype=np.float64).reshape(-1) for r in rhos]) if not isinstance(rhos, np.ndarray) \
        else np.asarray(rhos, dtype=np.float64).reshape(S, N)
    if rho.shape != (S, N):
        raise ValueError(f"total: expected {S} profiles of {N} points")
    mus = np.zeros(S) if mus is None else np.asarray(mus, dtype=np.float64)
    v = None
    if vexts is not None and any(x is not None for x in vexts):
        v = np.stack([np.zeros(N) if x is None else np.asarray(x, dtype=np.float64).reshape(-1) for x in vexts])
    sc, force = weights.engine.total_host(rho, mus, v)
    parts = {"ideal": sc[2], "external": sc[3], "hard_sphere": sc[4], "mean_field": sc[5],
             "N": [sc[6 + s] for s in range(S)]}
    return Result(free_energy=float(sc[0]), grand_potential=float(sc[1]), forces=[force[s] for s in range(S)],
                  parts=parts)


def total_stream(model: Model, states, weights: Weights, mus=None, vexts=None) -> list:
    """``total`` for a sequence of states (each one profile per species or an
    (S, N) array) through cdft_total_stream: the copies of one state overlap
    the evaluation of the next.  ``mus``: one beta*mu set per state (default
    0); ``vexts``: None or one list of fields (or None) per state.  Returns
    one Result per state, equal to ``total`` on each."""
    S = len(model.species)
    N = model.grid.total_points
    rhos = [np.stack([np.asarray(r, dtype=np.float64).reshape(-1) for r in st]) if not isinstance(st, np.ndarray)
            else np.asarray(st, dtype=np.float64).reshape(S, N) for st in states]
    mus = [np.zeros(S)] * len(rhos) if mus is None else [np.asarray(m, dtype=np.float64) for m in mus]
    vs = None
    if vexts is not None:
        vs = [None if v is None or all(x is None for x in v) else
              np.stack([np.zeros(N) if x is None else np.asarray(x, dtype=np.float64).reshape(-1) for x in v])
              for v in vexts]
    sc, forces = weights.engine.total_stream(rhos, mus, vs)
    out = []
    for i in range(len(rhos)):
        parts = {"ideal": sc[i, 2], "external": sc[i, 3], "hard_sphere": sc[i, 4], "mean_field": sc[i, 5],
                 "N": [sc[i, 6 + s] for s in range(S)]}
        out.append(Result(free_energy=float(sc[i, 0]), grand_potential=float(sc[i, 1]),
                          forces=[forces[i][s] for s in range(S)], parts=parts))
    return out


def total_batch(model: Model, rhos, weights: Weights, mus=None, vexts=None) -> list:
    """``total`` for every problem of a batched engine in one call.

    ``rhos``: (B, S, N) (or (B, N) for one species); ``mus``: (B, S) or
    broadcastable; ``vexts``: None or like ``rhos``.  Returns B Results.
    """
    e = weights.engine
    S, N, B = len(model.species), model.grid.total_points, e.batch
    rho = np.asarray(rhos, dtype=np.float64).reshape(B, S, N)
    mus = np.zeros((B, S)) if mus is None else np.asarray(mus, dtype=np.float64)
    if mus.ndim == 1 and S == 1 and mus.shape[0] == B:
        mus = mus[:, None]  # one beta*mu per problem
    v = None if vexts is None else np.asarray(vexts, dtype=np.float64).reshape(B, S, N)
    sc, force = e.total_host(rho, np.broadcast_to(mus, (B, S)), v)
    out = []
    for b in range(B):
        parts = {"ideal": sc[b, 2], "external": sc[b, 3], "hard_sphere": sc[b, 4], "mean_field": sc[b, 5],
                 "N": [sc[b, 6 + s] for s in range(S)]}
        out.append(Result(free_energy=float(sc[b, 0]), grand_potential=float(sc[b, 1]),
                          forces=[force[b, s] for s in range(S)], parts=parts))
    return out


class Functional:
    """functional.hpp:22-107: model + GPU weights with the evaluate / callback facade."""

    def __init__(self, fmt_model: FMTModel, model: Model, precision: int = _lib.FP64):
        self.model = model
        self.weights = make_weights(fmt_model, model, precision)

    def evaluate(self, rho, chemical_potential=0.0) -> Result:
        """functional.hpp:33-36 (single profile; V_ext is zero as in init::from_profile)."""
        S = len(self.model.species)
        rhos = [np.asarray(rho, dtype=np.float64).reshape(-1)]
        rhos += [np.zeros(self.model.grid.total_points) for _ in range(1, S)]
        return total(self.model, rhos, self.weights, [chemical_potential] + [0.0] * (S - 1))

    def grand_potential(self, rho, chemical_potential) -> float:
        return self.evaluate(rho, chemical_potential).grand_potential

    def bulk(self):
        """functional.hpp:48-50: the uniform fluid with the grid a_vdw."""
        from .bulk import make_bulk_thermodynamics
        return make_bulk_thermodynamics(self.model.species, self.weights)

    def grand_potential_callback(self, chemical_potential):
        """functional.hpp:62-73."""
        def fn(densities):
            r = total(self.model, densities, self.weights, [chemical_potential] * len(densities))
            return r.grand_potential, r.forces
        return fn
