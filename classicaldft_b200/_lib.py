"""ctypes binding of the engine's C ABI (include/cdft_b200.h).

The shared library is built in-tree (``python -m classicaldft_b200.build``)
and loaded from this package's directory.  There is no fallback: if the
library is missing, importing the host API raises.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcdft_b200.so")

CDFT_OK = 0
CDFT_ERR_INVALID = -1
CDFT_ERR_RUNTIME = -2
CDFT_ERR_CUDA = -3
CDFT_ERR_CUFFT = -4
SCALAR_COUNT = 10

MODEL_IDS = {"Rosenfeld": 0, "RSLT": 1, "WhiteBearI": 2, "WhiteBearII": 3, "esFMT": 4}
FP64 = 0
MIXED = 1
TRANSFORMS_CUFFT, TRANSFORMS_FUSED = 0, 1
POT_LJ, POT_TWF, POT_WRDF = 0, 1, 2
SPLIT_WCA, SPLIT_BH = 0, 1
WEIGHT_SCHEMES = {"InterpolationZero": 0, "InterpolationLinearE": 1, "InterpolationLinearF": 2,
                  "InterpolationQuadraticF": 3, "GaussE": 4, "GaussF": 5}

c_double_p = ctypes.POINTER(ctypes.c_double)
c_long3 = ctypes.c_long * 3


class CPotential(ctypes.Structure):
    _fields_ = [("type", ctypes.c_int), ("sigma", ctypes.c_double), ("epsilon", ctypes.c_double),
                ("r_cutoff", ctypes.c_double), ("alpha", ctypes.c_double)]


class CInteraction(ctypes.Structure):
    _fields_ = [("species_i", ctypes.c_int), ("species_j", ctypes.c_int), ("weight_real", c_double_p),
                ("a_vdw", ctypes.c_double)]


class CModelInteraction(ctypes.Structure):
    _fields_ = [("species_i", ctypes.c_int), ("species_j", ctypes.c_int), ("potential", CPotential),
                ("split", ctypes.c_int), ("scheme", ctypes.c_int)]


class CFireParams(ctypes.Structure):
    _fields_ = [("dt", ctypes.c_double), ("dt_max", ctypes.c_double), ("dt_min", ctypes.c_double),
                ("alpha_start", ctypes.c_double), ("f_inc", ctypes.c_double), ("f_dec", ctypes.c_double),
                ("f_alpha", ctypes.c_double), ("n_delay", ctypes.c_int), ("max_uphill", ctypes.c_int),
                ("force_tolerance", ctypes.c_double), ("max_steps", ctypes.c_int)]


class CMinimizerConfig(ctypes.Structure):
    _fields_ = [("fire", CFireParams), ("mode", ctypes.c_int), ("parametrization", ctypes.c_int),
                ("rho_min", ctypes.c_double), ("rho_max", ctypes.c_double), ("homogeneous_boundary", ctypes.c_int),
                ("chemical_potential", ctypes.c_double), ("target_mass", ctypes.c_double),
                ("boundary_mass", ctypes.c_double), ("use_monitor", ctypes.c_int), ("check_interval", ctypes.c_int),
                ("external_field", ctypes.c_void_p)]


class CMinimizerResult(ctypes.Structure):
    _fields_ = [("free_energy", ctypes.c_double), ("grand_potential", ctypes.c_double),
                ("rms_force", ctypes.c_double), ("iterations", ctypes.c_int), ("converged", ctypes.c_int),
                ("uphill_error", ctypes.c_int)]


class CDDFTConfig(ctypes.Structure):
    _fields_ = [("dt", ctypes.c_double), ("diffusion_coefficient", ctypes.c_double),
                ("min_density", ctypes.c_double), ("dt_max", ctypes.c_double), ("fp_tolerance", ctypes.c_double),
                ("fp_max_iterations", ctypes.c_int)]


class CPicardConfig(ctypes.Structure):
    _fields_ = [("mixing", ctypes.c_double), ("min_density", ctypes.c_double), ("tolerance", ctypes.c_double),
                ("constraint_min_density", ctypes.c_double), ("max_iterations", ctypes.c_int),
                ("check_interval", ctypes.c_int)]


class CPicardResult(ctypes.Structure):
    _fields_ = [("grand_potential", ctypes.c_double), ("residual", ctypes.c_double),
                ("iterations", ctypes.c_int), ("converged", ctypes.c_int)]


STOP_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_void_p)


EIGEN_RAYLEIGH_RITZ = 0
EIGEN_LANCZOS = 1


class CGroupMember(ctypes.Structure):
    _fields_ = [("engine", ctypes.c_void_p), ("refine", ctypes.c_void_p), ("refine_switch", ctypes.c_double),
                ("mu", ctypes.POINTER(ctypes.c_double)), ("target_mass", ctypes.POINTER(ctypes.c_double)),
                ("rho", ctypes.c_void_p), ("results", ctypes.POINTER(CMinimizerResult))]


class CEigenConfig(ctypes.Structure):
    _fields_ = [("tolerance", ctypes.c_double), ("max_iterations", ctypes.c_int), ("hessian_eps", ctypes.c_double),
                ("exact_hvp", ctypes.c_int), ("seed", ctypes.c_ulonglong), ("method", ctypes.c_int),
                ("block", ctypes.c_int), ("max_basis", ctypes.c_int), ("check_interval", ctypes.c_int)]


class CBulkInteraction(ctypes.Structure):
    _fields_ = [("species_i", ctypes.c_int), ("species_j", ctypes.c_int), ("a_vdw", ctypes.c_double)]


class CBulkModel(ctypes.Structure):
    _fields_ = [("n_species", ctypes.c_int), ("diameters", ctypes.c_double * 4), ("fmt_model", ctypes.c_int),
                ("esfmt_A", ctypes.c_double), ("esfmt_B", ctypes.c_double), ("n_interactions", ctypes.c_int),
                ("interactions", CBulkInteraction * 8)]


class CSaddleConfig(ctypes.Structure):
    _fields_ = [("fire", CFireParams), ("eigen", CEigenConfig), ("rho_min", ctypes.c_double),
                ("omega_tolerance", ctypes.c_double), ("tolerance_start", ctypes.c_double),
                ("tolerance_factor", ctypes.c_double), ("max_outer_iterations", ctypes.c_int),
                ("eigenvalue_clear_count", ctypes.c_int)]


class EngineError(RuntimeError):
    """A failed C-ABI call; ``code`` is the CDFT_ERR_* status."""

    def __init__(self, code: int, msg: str):
        super().__init__(msg)
        self.code = code


_lib = None


def lib():
    """Load libcdft_b200.so once; raise if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"classicaldft_b200: CUDA library not built ({LIB_PATH} missing); "
                          "run `python -m classicaldft_b200.build`")
    L = ctypes.CDLL(LIB_PATH)
    L.cdft_last_error.restype = ctypes.c_char_p
    L.cdft_version.restype = ctypes.c_char_p
    vp = ctypes.c_void_p
    sigs = {
        "cdft_potential_info": [ctypes.POINTER(CPotential), c_double_p],
        "cdft_potential_attractive": [ctypes.POINTER(CPotential), ctypes.c_int, c_double_p, ctypes.c_long, c_double_p],
        "cdft_hard_sphere_diameter": [ctypes.POINTER(CPotential), ctypes.c_double, ctypes.c_int, c_double_p],
        "cdft_vdw_integral": [ctypes.POINTER(CPotential), ctypes.c_double, ctypes.c_int, c_double_p],
        "cdft_interaction_weight": [c_long3, ctypes.c_double, ctypes.POINTER(CPotential), ctypes.c_int, ctypes.c_int,
                                    ctypes.c_double, c_double_p, c_double_p],
        "cdft_create": [ctypes.POINTER(vp), c_long3, ctypes.c_double, ctypes.c_int, c_double_p, ctypes.c_int,
                        ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.POINTER(CInteraction), ctypes.c_int],
        "cdft_create_batch": [ctypes.POINTER(vp), c_long3, ctypes.c_double, ctypes.c_int, c_double_p, ctypes.c_int,
                              ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.POINTER(CInteraction),
                              ctypes.c_int, ctypes.c_int],
        "cdft_create_model": [ctypes.POINTER(vp), c_long3, ctypes.c_double, ctypes.c_int, c_double_p, ctypes.c_int,
                              ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.POINTER(CModelInteraction),
                              ctypes.c_double, ctypes.c_int, ctypes.c_int],
        "cdft_engine_batch": [vp, ctypes.POINTER(ctypes.c_int)],
        "cdft_destroy": [vp],
        "cdft_engine_bulk_model": [vp, ctypes.POINTER(CBulkModel)],
        "cdft_bulk_free_energy_density": [ctypes.POINTER(CBulkModel), c_double_p, c_double_p],
        "cdft_bulk_chemical_potentials": [ctypes.POINTER(CBulkModel), c_double_p, c_double_p],
        "cdft_bulk_pressure": [ctypes.POINTER(CBulkModel), c_double_p, c_double_p],
        "cdft_bulk_density_from_mu": [ctypes.POINTER(CBulkModel), ctypes.c_int, c_double_p, c_double_p, ctypes.c_int,
                                      ctypes.c_double, c_double_p, ctypes.POINTER(ctypes.c_int)],
        "cdft_bulk_spinodal": [ctypes.POINTER(CBulkModel), ctypes.c_double, ctypes.c_double, c_double_p,
                               ctypes.POINTER(ctypes.c_int)],
        "cdft_bulk_coexistence": [ctypes.POINTER(CBulkModel), ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                  ctypes.c_double, c_double_p, ctypes.POINTER(ctypes.c_int)],
        "cdft_engine_info": [vp, ctypes.POINTER(ctypes.c_longlong)],
        "cdft_engine_a_vdw": [vp, ctypes.c_int, c_double_p],
        "cdft_total": [vp, vp, vp, c_double_p, vp, c_double_p],
        "cdft_total_stream": [vp, ctypes.c_int, ctypes.POINTER(vp), ctypes.POINTER(vp), c_double_p,
                              ctypes.POINTER(vp), c_double_p],
        "cdft_total_device": [vp, vp, vp, c_double_p, vp, vp, vp],
        "cdft_engine_status": [vp, vp],
        "cdft_engine_set_transforms": [vp, ctypes.c_int],
        "cdft_engine_set_plane_chunks": [vp, ctypes.c_int],
        "cdft_set_step_graphs": [ctypes.c_int],
        "cdft_step_graphs": [ctypes.POINTER(ctypes.c_int)],
        "cdft_engine_autotune": [vp, vp, vp, ctypes.POINTER(ctypes.c_double), vp, ctypes.c_int,
                                 ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double)],
        "cdft_engine_transforms": [vp, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)],
        "cdft_engine_stage_timing": [vp, ctypes.c_int],
        "cdft_engine_stage_times": [vp, c_double_p, ctypes.POINTER(ctypes.c_longlong)],
        "cdft_local_terms_noalloc": [vp, vp, c_double_p, ctypes.c_int, ctypes.c_longlong, ctypes.c_double, vp, vp,
                                     vp],
        "cdft_minimize": [vp, ctypes.POINTER(CMinimizerConfig), vp, vp, vp, ctypes.c_double,
                          ctypes.POINTER(CMinimizerResult), vp],
        "cdft_minimize_batch": [vp, ctypes.POINTER(CMinimizerConfig), c_double_p, c_double_p, vp, vp,
                                ctypes.c_double, ctypes.POINTER(CMinimizerResult), vp],
        "cdft_ddft_step": [vp, ctypes.POINTER(CDDFTConfig), ctypes.c_double, vp, c_double_p,
                           ctypes.POINTER(ctypes.c_int), vp],
        "cdft_ddft_run": [vp, ctypes.POINTER(CDDFTConfig), ctypes.c_double, ctypes.c_int, vp, c_double_p, c_double_p,
                          vp],
        "cdft_ddft_split_step": [vp, ctypes.POINTER(CDDFTConfig), ctypes.c_double, vp, c_double_p, vp],
        "cdft_ddft_cn_step": [vp, ctypes.POINTER(CDDFTConfig), ctypes.c_double, vp, c_double_p,
                              ctypes.POINTER(ctypes.c_int), vp],
        "cdft_ddft_simulate": [vp, ctypes.POINTER(CDDFTConfig), ctypes.c_double, ctypes.c_int, vp, c_double_p,
                               c_double_p, ctypes.c_int, c_double_p, ctypes.POINTER(ctypes.c_int), ctypes.c_int,
                               ctypes.POINTER(ctypes.c_int), vp, ctypes.c_double, STOP_FN, vp,
                               ctypes.POINTER(ctypes.c_int), vp],
        "cdft_picard": [vp, ctypes.POINTER(CPicardConfig), c_double_p, c_double_p, vp, vp,
                        ctypes.POINTER(CPicardResult), vp],
        "cdft_lattice_size": [ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_long), ctypes.POINTER(ctypes.c_long)],
        "cdft_build_lattice": [ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_long), c_double_p, ctypes.c_long,
                               c_double_p],
        "cdft_lattice_export": [c_double_p, ctypes.c_long, ctypes.c_char_p, ctypes.c_int],
        "cdft_gaussian_peaks": [ctypes.POINTER(ctypes.c_long), ctypes.c_double, c_double_p, ctypes.c_long,
                                ctypes.c_double, ctypes.c_double, ctypes.c_double, vp, vp],
        "cdft_hvp": [vp, vp, vp, ctypes.c_double, ctypes.c_int, vp, vp],
        "cdft_hvp_fd": [vp, vp, vp, vp, ctypes.c_double, ctypes.c_double, ctypes.c_int, vp, vp],
        "cdft_eigen_solve": [vp, ctypes.POINTER(CEigenConfig), vp, ctypes.c_double, vp, ctypes.c_int, c_double_p,
                             ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int), vp],
        "cdft_saddle_find": [vp, ctypes.POINTER(CSaddleConfig), vp, ctypes.c_double, ctypes.c_double, vp,
                             c_double_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int), vp],
        "cdft_ddft_set_refine": [vp, vp, ctypes.c_int],
        "cdft_engine_set_pointwise": [vp, ctypes.c_int],
        "cdft_engine_pointwise": [vp, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)],
        "cdft_engine_autotune_ex": [vp, vp, vp, c_double_p, vp, ctypes.c_int, ctypes.POINTER(ctypes.c_int), c_double_p],
        "cdft_engine_set_column_tile": [vp, ctypes.c_int],
        "cdft_engine_set_pointwise_spread": [vp, ctypes.c_int],
        "cdft_engine_set_dependent_launch": [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_int)],
        "cdft_engine_set_anchor": [vp, vp, vp, vp],
        "cdft_engine_set_anchor_host": [vp, vp, vp],
        "cdft_engine_clear_anchor": [vp],
        "cdft_engine_anchored": [vp, ctypes.POINTER(ctypes.c_int)],
        "cdft_engine_pointwise_spread": [vp, ctypes.POINTER(ctypes.c_int)],
        "cdft_engine_column_tile": [vp, ctypes.POINTER(ctypes.c_int)],
        "cdft_engine_set_plane_width": [vp, ctypes.c_int],
        "cdft_engine_plane_width": [vp, ctypes.POINTER(ctypes.c_int)],
        "cdft_minimize_group": [ctypes.c_int, ctypes.POINTER(CGroupMember), ctypes.POINTER(CMinimizerConfig), vp],
        "cdft_ddft_last_step": [vp, ctypes.POINTER(ctypes.c_int), c_double_p],
        "cdft_eigen_solve_ex": [vp, vp, ctypes.POINTER(CEigenConfig), vp, ctypes.c_double, vp, ctypes.c_int,
                                c_double_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int), vp],
        "cdft_saddle_find_ex": [vp, vp, vp, ctypes.c_double, ctypes.POINTER(CSaddleConfig), vp, ctypes.c_double,
                                ctypes.c_double, vp, c_double_p, ctypes.POINTER(ctypes.c_int),
                                ctypes.POINTER(ctypes.c_int), vp],
    }
    for name, args in sigs.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = ctypes.c_int
    _lib = L
    return L


def check(status: int):
    if status != CDFT_OK:
        msg = lib().cdft_last_error().decode(errors="replace")
        if status == CDFT_ERR_INVALID:
            raise ValueError(msg)
        raise EngineError(status, msg)


def declared_symbols():
    """Names of every function declared in include/cdft_b200.h."""
    import re
    hdr = os.path.join(os.path.dirname(HERE), "include", "cdft_b200.h")
    with open(hdr) as f:
        text = f.read()
    return sorted(set(re.findall(r"CDFT_API\s+[\w\s\*]+?\b(cdft_\w+)\s*\(", text)))
