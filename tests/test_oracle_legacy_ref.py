"""The oracle against the reference's own code, compiled here.

The reference's legacy translation (legacy/classicaldft.hpp: the FMT
f-functions, Phi3 and its derivatives, the full esFMT Phi, the QF
mean-field weights and a_vdw, the Enskog thermodynamics and the
spinodal / coexistence solver) needs none of the libraries the reference's
CMake build requires, so oracle/build_ref.py compiles it with g++ behind a
C-ABI shim into oracle/_ref/liblegacy_ref.so.  These tests evaluate the
oracle and the reference's code on the same inputs -- the points of the
reference's own cross-validation tests (tests/integration/functionals/
fmt.cpp:13-139, mean_field.cpp:22-109) and more -- and require agreement
to round-off (1e-13 relative, 1e-12 for sums over the QF cell grid), tighter
than the reference's 1e-10 margins.  Skipped where neither the built library
nor the reference tree is present.
"""
import ctypes
import math
import os

import numpy as np
import pytest

from oracle import bulk as obulk
from oracle import fmt, legacy
from oracle import potentials as opot

LIB = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref",
                   "liblegacy_ref.so")
ETAS = [0.05, 0.10, 0.15, 0.20, 0.25, 0.30, 0.35, 0.40, 0.45, 0.50, 0.55, 0.60]  # fmt.cpp:13
MODEL_IDS = {"Rosenfeld": 0, "RSLT": 1, "esFMT": 2, "WhiteBearI": 3, "WhiteBearII": 4}
dp = ctypes.POINTER(ctypes.c_double)


@pytest.fixture(scope="module")
def ref():
    if not os.path.exists(LIB):
        from oracle import build_ref
        if build_ref.build() is None:
            pytest.skip("reference tree absent and the legacy library not built")
    L = ctypes.CDLL(LIB)
    L.lref_f.restype = ctypes.c_double
    L.lref_f.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double]
    L.lref_fex.restype = ctypes.c_double
    L.lref_fex.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double]
    L.lref_derived.argtypes = [dp, dp]
    L.lref_phi3.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, dp, dp]
    L.lref_phi.restype = ctypes.c_double
    L.lref_phi.argtypes = [dp, ctypes.c_double, ctypes.c_double]
    L.lref_watt2_lj.restype = ctypes.c_double
    L.lref_watt2_lj.argtypes = [ctypes.c_double] * 4
    L.lref_weight_qf.restype = ctypes.c_double
    L.lref_weight_qf.argtypes = [ctypes.c_double] * 3 + [ctypes.c_int] * 3 + [ctypes.c_double]
    L.lref_avdw_qf.restype = ctypes.c_double
    L.lref_avdw_qf.argtypes = [ctypes.c_double] * 5
    L.lref_enskog.argtypes = [ctypes.c_double, dp]
    fn = ctypes.CFUNCTYPE(ctypes.c_double, ctypes.c_double, ctypes.c_void_p)
    L.lref_spinodal.argtypes = [fn, fn, ctypes.c_void_p] + [ctypes.c_double] * 3 + [dp]
    L.lref_coexistence.argtypes = [fn, fn, ctypes.c_void_p] + [ctypes.c_double] * 3 + [dp]
    L.scalar_fn = fn
    return L


def close(a, b, rel=1e-13, abs_=1e-15):
    return abs(a - b) <= max(rel * abs(b), abs_)


def measures(eta, n2, v_mag, t_diag):
    """fmt.cpp:74-89: the oracle's measures and the reference's 19 inputs."""
    Rr = 0.5
    f = 4.0 * math.pi * Rr
    m = {"eta": eta, "n2": n2, "n1": n2 / f, "n0": n2 / (f * Rr),
         "v1": np.array([v_mag, -0.3 * v_mag, 0.1 * v_mag]),
         "v0": np.array([v_mag / f, -0.3 * v_mag / f, 0.1 * v_mag / f]),
         "T": np.array([[t_diag, 0.1, -0.05], [0.1, t_diag * 0.8, 0.02], [-0.05, 0.02, t_diag * 0.6]])}
    m["products"] = fmt.inner_products(m)
    raw = np.concatenate([[eta, m["n0"], m["n1"], n2], m["v0"], m["v1"], m["T"].ravel()]).astype(np.float64)
    return m, raw


def test_f_functions_match_the_reference(ref):
    """fmt.cpp:15-54 at its packing fractions, plus the Taylor side."""
    for name, mid in MODEL_IDS.items():
        mod = fmt.FMTModel(name)
        for eta in ETAS + [1e-3, 1e-5]:
            f1, _, f2, _, f3, _ = mod.f(eta)
            for which, mine in ((1, f1), (2, f2), (3, f3)):
                theirs = ref.lref_f(mid, which, eta)
                assert close(float(mine), theirs, rel=1e-12), (name, which, eta, float(mine), theirs)


def test_legacy_restatement_matches_the_reference(ref):
    """oracle/legacy.py restates the same code: every f, Phi3 and derivative."""
    pairs = [("Rosenfeld", legacy.rosenfeld_f), ("RSLT", legacy.rslt_f), ("WhiteBearI", legacy.whitebear1_f),
             ("WhiteBearII", legacy.whitebear2_f), ("esFMT", legacy.esfmt_f)]
    for name, lf in pairs:
        for eta in ETAS:
            mine = lf(eta)
            for which in (1, 2, 3):
                assert close(mine[which - 1], ref.lref_f(MODEL_IDS[name], which, eta), rel=1e-14), (name, eta)
    m, raw = measures(0.3, 2.5, 0.4, 0.3)
    fm = legacy.derived({"eta": 0.3, "s0": m["n0"], "s1": m["n1"], "s2": 2.5, "v1": m["v0"], "v2": m["v1"],
                         "T": m["T"]})
    out = np.zeros(20)
    ref.lref_derived(raw.ctypes.data_as(dp), out.ctypes.data_as(dp))
    assert close(fm["v2_v2"], out[1]) and close(fm["vTv"], out[2]) and close(fm["T2"], out[3])
    assert close(fm["T3"], out[4])


@pytest.mark.parametrize("point", [(0.3, 2.5, 0.4, 0.3), (0.25, 2.0, 0.3, 0.25), (0.45, 3.1, 0.7, 0.5),
                                   (0.1, 0.9, 0.05, 0.1)])
def test_phi3_and_derivatives_match_the_reference(ref, point):
    """fmt.cpp:91-139 (its two points and two more) for Rosenfeld, RSLT and
    esFMT(A, B): Phi3, dPhi3/dn2, dPhi3/dv1 and dPhi3/dT."""
    m, raw = measures(*point)
    out = np.zeros(14)
    for name, A, B in (("Rosenfeld", 1.0, 0.0), ("RSLT", 1.0, 0.0), ("esFMT", 1.0, 0.0), ("esFMT", 1.0, -1.0),
                       ("esFMT", 0.8, 0.3)):
        mod = fmt.FMTModel(name, A, B)
        ref.lref_phi3(MODEL_IDS[name], A, B, raw.ctypes.data_as(dp), out.ctypes.data_as(dp))
        assert close(float(mod.phi3(m)), out[0]), name
        assert close(float(mod.d_phi3_d_n2(m)), out[1]), name
        dv = mod.d_phi3_d_v1(m)
        for k in range(3):
            assert close(float(dv[k]), out[2 + k], abs_=1e-14), (name, k)
        if name == "esFMT":
            dT = mod.d_phi3_d_T(m)
            for j in range(3):
                for k in range(3):
                    # the reference's dPhi3/dT(j, k) is the oracle's (k, j) entry
                    assert close(float(dT[k, j]), out[5 + 3 * j + k], abs_=1e-14), (j, k)


@pytest.mark.parametrize("point", [(0.3, 2.5, 0.4, 0.3), (0.25, 2.0, 0.3, 0.25), (1e-31, 0.0, 0.0, 0.0)])
def test_full_esfmt_phi_matches_the_reference(ref, point):
    """legacy phi(): -n0 ln(1-eta) + (n1 n2 - v0.v1)/(1-eta) + Phi3/(1-eta)^2,
    zero below eta = 1e-30 as the oracle's pointwise skip."""
    m, raw = measures(*point)
    for A, B in ((1.0, 0.0), (1.0, -1.0)):
        mine = float(fmt.FMTModel("esFMT", A, B).phi(m)) if point[0] >= 1e-30 else 0.0
        assert close(mine, ref.lref_phi(raw.ctypes.data_as(dp), A, B)), (point, A, B)


def test_bulk_excess_free_energies_match_the_reference(ref):
    """The oracle's uniform-fluid excess free energy per particle of every
    model equals the reference's legacy fex(eta) (esFMT at three (A, B)); for
    Rosenfeld that is the Percus-Yevick compressibility result and for White
    Bear I/II the Carnahan-Starling one of the reference's Enskog class."""
    out = np.zeros(8)
    for rho in (0.05, 0.3, 0.6, 0.9):
        eta = math.pi * rho / 6.0
        ref.lref_enskog(rho, out.ctypes.data_as(dp))
        for name, A, B in (("Rosenfeld", 1.0, 0.0), ("RSLT", 1.0, 0.0), ("WhiteBearI", 1.0, 0.0),
                           ("WhiteBearII", 1.0, 0.0), ("esFMT", 1.0, 0.0), ("esFMT", 1.0, -1.0), ("esFMT", 0.8, 0.3)):
            fex = fmt.FMTModel(name, A, B).free_energy_density(rho, 1.0) / rho
            assert close(fex, ref.lref_fex(MODEL_IDS[name], eta, A, B), rel=1e-12), (name, A, B, rho)
        assert close(fmt.FMTModel("Rosenfeld").free_energy_density(rho, 1.0) / rho, out[0], rel=1e-12)
        for name in ("WhiteBearI", "WhiteBearII"):
            assert close(fmt.FMTModel(name).free_energy_density(rho, 1.0) / rho, out[1], rel=1e-12)


def test_qf_weights_and_a_vdw_match_the_reference(ref):
    """mean_field.cpp:22-109: the QF cell weights of the WCA-split LJ and the
    grid a_vdw, from the oracle's restatement and from the reference's code."""
    for sigma, eps, rc, dx in ((1.0, 1.0, 2.5, 0.1), (1.0, 1.0, 3.0, 0.4), (1.1, 0.8, 2.0, 0.2)):
        for r2 in (0.5, 1.0, 1.2, 2.0, 4.0, 9.5):
            assert close(legacy.watt2_lj(sigma, eps, rc, r2), ref.lref_watt2_lj(sigma, eps, rc, r2))
        for s in ((0, 0, 0), (1, 0, 0), (2, 1, 0), (3, 2, 1), (5, 4, 4)):
            assert close(legacy.generate_weight_qf(sigma, eps, rc, *s, dx),
                         ref.lref_weight_qf(sigma, eps, rc, *s, dx), abs_=1e-16), s
        for kT in (0.7, 1.0):
            mine = legacy.compute_a_vdw_qf(sigma, eps, rc, kT, dx)
            assert close(mine, ref.lref_avdw_qf(sigma, eps, rc, kT, dx), rel=1e-12), (sigma, rc, dx, kT)


def test_spinodal_and_coexistence_match_the_reference_solver(ref):
    """The reference's legacy solver (DFT_Coex) run on the oracle's equation
    of state equals the oracle's restatement of that solver, and the oracle's
    own phase search agrees with both (eos.cpp / coexistence tests)."""
    for kT in (0.7, 0.8, 0.9):
        lj = opot.make_lennard_jones(1.0, 1.0, 3.0)
        d = opot.hard_sphere_diameter(lj, kT, opot.WCA)
        eos = obulk.make_bulk_thermodynamics([d], obulk.FMTModel("WhiteBearII"), [opot.Interaction(0, 0, lj)], kT)
        P = ref.scalar_fn(lambda x, _u: float(eos.pressure([x])))
        C = ref.scalar_fn(lambda x, _u: float(eos.chemical_potential([x], 0)))
        sp = np.zeros(2)
        assert ref.lref_spinodal(P, C, None, 1.0, 0.005, 1e-8, sp.ctypes.data_as(dp)) == 0
        mine = legacy.legacy_find_spinodal(lambda x: float(eos.pressure([x])), 1.0, 0.005, 1e-8)
        assert close(mine[0], sp[0], rel=1e-12) and close(mine[1], sp[1], rel=1e-12), (kT, mine, sp)
        co = np.zeros(2)
        assert ref.lref_coexistence(P, C, None, 1.0, 0.005, 1e-8, co.ctypes.data_as(dp)) == 0
        mc = legacy.legacy_find_coex(lambda x: float(eos.pressure([x])), lambda x: float(eos.chemical_potential([x], 0)),
                                     1.0, 0.005, 1e-8)
        assert close(mc[0], co[0], rel=1e-12) and close(mc[1], co[1], rel=1e-12), (kT, mc, co)
        ps = obulk.PhaseSearch(rho_max=1.0, rho_scan_step=0.005).find_coexistence(eos)
        assert ps is not None
        assert abs(ps[0] - co[0]) <= 1e-6 * co[0] and abs(ps[1] - co[1]) <= 1e-6 * co[1], (kT, ps, co)
