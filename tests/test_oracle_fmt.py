"""Pins the oracle's FMT restatement against the reference's known-answer tests.

Each case restates one test of the reference (file:line given) with its
parameters and tolerance; the legacy cross-checks use the independent legacy
formulas (oracle/legacy.py).
"""
import math

import numpy as np
import pytest

from oracle import fmt, legacy
from oracle.functional import Model, Species, convolve, hard_sphere, make_weights
from oracle.grid import Grid, c2r, r2c

DX = 0.1
D = 1.0
R = 0.5
GRID = Grid(dx=DX, box_size=(1.6, 1.6, 1.6), shape=(16, 16, 16))
N = 16 ** 3
MODELS = ["Rosenfeld", "RSLT", "WhiteBearI", "WhiteBearII", "esFMT"]


def nd(f, x, h=1e-6):
    return (f(x + h) - f(x - h)) / (2.0 * h)


# ---- tests/unit/functionals/fmt/weights.cpp ------------------------------

def test_weight_dc_components():
    """weights.cpp:21-62: DC = volume/N, surface/N, 0, isotropic tensor."""
    ws = fmt.generate_weights(D, GRID)
    assert ws["w3"][0, 0, 0].real == pytest.approx((4.0 / 3.0) * math.pi * R ** 3 / N, abs=1e-14)
    assert ws["w2"][0, 0, 0].real == pytest.approx(4.0 * math.pi * R * R / N, abs=1e-14)
    for a in range(3):
        assert abs(ws["wv2"][a][0, 0, 0]) == pytest.approx(0.0, abs=1e-14)
    for a in range(3):
        assert ws["wT"][(a, a)][0, 0, 0].real == pytest.approx((4.0 * math.pi / 3.0) * R * R / N, abs=1e-14)
    for p in ((0, 1), (0, 2), (1, 2)):
        assert abs(ws["wT"][p][0, 0, 0]) == pytest.approx(0.0, abs=1e-14)


def test_weight_sum_rules_uniform_density():
    """weights.cpp:75-192: convolution with a uniform density."""
    rho0 = 0.8
    ws = fmt.generate_weights(D, GRID)
    rk = r2c(np.full(GRID.shape, rho0))
    eta = convolve(ws["w3"], rk, GRID.shape)
    n2 = convolve(ws["w2"], rk, GRID.shape)
    assert np.max(np.abs(eta - (math.pi / 6.0) * rho0)) < 1e-10
    assert np.max(np.abs(n2 - math.pi * rho0)) < 1e-10
    for a in range(3):
        assert np.max(np.abs(convolve(ws["wv2"][a], rk, GRID.shape))) < 1e-10
    for a in range(3):
        assert convolve(ws["wT"][(a, a)], rk, GRID.shape)[0] == pytest.approx(math.pi * rho0 / 3.0, abs=1e-10)
    for p in ((0, 1), (0, 2), (1, 2)):
        assert np.max(np.abs(convolve(ws["wT"][p], rk, GRID.shape))) < 1e-10
    m = fmt.make_uniform_measures(0.6, D)
    rk6 = r2c(np.full(GRID.shape, 0.6))
    n2_6 = convolve(ws["w2"], rk6, GRID.shape)[0]
    assert n2_6 / (4.0 * math.pi * R) == pytest.approx(float(m["n1"]), abs=1e-10)
    assert n2_6 / (4.0 * math.pi * R * R) == pytest.approx(float(m["n0"]), abs=1e-10)


def test_tensor_trace_equals_surface_weight():
    """A + 3B = w2 (trace of the tensor weight is the surface weight).

    Checked from the smallest wavevector of a 20-sigma box upward: below that
    the reference's A, B formulas lose digits to cancellation.
    """
    k = np.concatenate([[0.0], np.linspace(2.0 * math.pi / 20.0, 40.0, 2000)])
    for Rs in (0.25, 0.5, 0.77):
        w3, w2, fv, A, B = fmt.weight_kernels(k, Rs)
        assert np.max(np.abs(A + 3.0 * B - w2)) < 1e-12 * np.max(np.abs(w2))


# ---- tests/unit/functionals/fmt/models.cpp --------------------------------

def test_dilute_limits():
    """models.cpp:35-59."""
    e = 1e-10
    f1, _, f2, _, f3, _ = fmt.FMTModel("Rosenfeld").f(e)
    assert f1 == pytest.approx(math.log(1 - e), abs=1e-14)
    assert f2 == pytest.approx(1.0, abs=1e-9) and f3 == pytest.approx(1.0, abs=1e-9)
    _, _, f2, _, f3, _ = fmt.FMTModel("RSLT").f(e)
    assert f2 == pytest.approx(1.0, abs=1e-8) and f3 == pytest.approx(1.0, abs=1e-6)
    assert fmt.FMTModel("WhiteBearI").f(e)[4] == pytest.approx(1.5, abs=1e-6)
    assert fmt.FMTModel("WhiteBearII").f(e)[4] == pytest.approx(1.5, abs=1e-6)
    assert fmt.FMTModel("RSLT").f(1e-8)[4] == pytest.approx(1.0, abs=1e-6)  # models.cpp:116-120


@pytest.mark.parametrize("name", MODELS)
def test_f_derivatives_match_finite_differences(name):
    """models.cpp:63-112 (margins 1e-8 at 0.3, 1e-5 over 0.1..0.4)."""
    m = fmt.FMTModel(name)
    for eta in (0.1, 0.2, 0.3, 0.4):
        vals = m.f(eta)
        for i in (0, 2, 4):
            num = nd(lambda e: float(m.f(e)[i]), eta)
            assert float(vals[i + 1]) == pytest.approx(num, abs=1e-5)
    vals = m.f(0.3)
    for i in (0, 2, 4):
        assert float(vals[i + 1]) == pytest.approx(nd(lambda e: float(m.f(e)[i]), 0.3), abs=1e-8)


def test_taylor_branch_derivatives_are_polynomial_derivatives():
    for name in ("RSLT", "WhiteBearI", "WhiteBearII"):
        m = fmt.FMTModel(name)
        e = 5e-7
        vals = m.f(e)
        for i in (2, 4):
            assert float(vals[i + 1]) == pytest.approx(nd(lambda x: float(m.f(x)[i]), e, 1e-8), rel=1e-6)


def test_free_energy_identities():
    """models.cpp:124-142: Rosenfeld = PY compressibility, WhiteBearI = CS."""
    for rho in (0.1, 0.3, 0.5, 0.7, 0.9):
        eta = (math.pi / 6.0) * rho
        e = 1.0 - eta
        py = -math.log(e) + 1.5 * eta * (2.0 - eta) / (e * e)
        cs = eta * (4.0 - 3.0 * eta) / (e * e)
        assert fmt.FMTModel("Rosenfeld").free_energy_density(rho, 1.0) / rho == pytest.approx(py, abs=1e-10)
        assert fmt.FMTModel("WhiteBearI").free_energy_density(rho, 1.0) / rho == pytest.approx(cs, abs=1e-10)


@pytest.mark.parametrize("name", ["Rosenfeld", "WhiteBearI", "WhiteBearII", "esFMT"])
def test_chemical_potential_matches_fd(name):
    """models.cpp:146-168, 301-307."""
    m = fmt.FMTModel(name)
    mu = m.excess_chemical_potential(0.5, 1.0)
    assert mu == pytest.approx(nd(lambda r: m.free_energy_density(r, 1.0), 0.5), abs=1e-6)


def test_phi_uniform_and_tensor_derivatives():
    """models.cpp:172-202."""
    wb = fmt.FMTModel("WhiteBearI")
    m = fmt.make_uniform_measures(0.6, 1.0)
    assert float(wb.phi(m)) == pytest.approx(wb.free_energy_density(0.6, 1.0), abs=1e-14)
    m5 = fmt.make_uniform_measures(0.5, 1.0)
    dm = wb.d_phi(m5)
    for key in ("d_eta", "d_n0", "d_n1", "d_n2"):
        assert float(dm[key]) != 0.0
    assert np.sum(np.abs(wb.d_phi(m5)["d_T"])) > 0.0
    assert np.sum(np.abs(fmt.FMTModel("Rosenfeld").d_phi(m5)["d_T"])) == 0.0


def test_rslt_zero_guard():
    """models.cpp:206-213."""
    m = {"eta": 0.0, "n0": 0.0, "n1": 0.0, "n2": 1e-35, "v0": np.zeros(3), "v1": np.zeros(3),
         "T": np.zeros((3, 3))}
    m["products"] = fmt.inner_products(m)
    r = fmt.FMTModel("RSLT")
    assert float(r.phi3(m)) == 0.0 and float(r.d_phi3_d_n2(m)) == 0.0
    assert np.linalg.norm(r.d_phi3_d_v1(m)) == 0.0


def test_whitebear2_taylor_continuity():
    """models.cpp:217-238."""
    m = fmt.FMTModel("WhiteBearII")
    assert float(m.f(1e-8)[2]) == pytest.approx(1.0, abs=1e-6)
    assert float(m.f(9e-7)[2]) == pytest.approx(float(m.f(2e-6)[2]), rel=1e-4)
    assert float(m.f(1e-8)[4]) == pytest.approx(1.5, abs=1e-6)


def test_esfmt_properties():
    """models.cpp:247-299."""
    es = fmt.FMTModel("esFMT", 1.0, 0.0)
    ros = fmt.FMTModel("Rosenfeld")
    for eta in (0.1, 0.2, 0.3, 0.4):
        assert np.allclose(es.f(eta), ros.f(eta))
    m = fmt.make_uniform_measures(0.5, 1.0)
    assert float(es.phi3(m)) != 0.0 and float(es.d_phi3_d_n2(m)) != 0.0
    assert np.linalg.norm(es.d_phi3_d_v1(m)) == pytest.approx(0.0, abs=1e-14)
    assert float(es.d_phi3_d_T(m)[0, 0]) != 0.0
    es1 = fmt.FMTModel("esFMT", 1.0, 1.0)
    assert float(es.phi3(m)) != pytest.approx(float(es1.phi3(m)), abs=1e-14)
    f = es.free_energy_density(0.5, 1.0)
    assert math.isfinite(f) and f > 0.0


# ---- tests/integration/functionals/fmt.cpp (legacy cross-validation) ------

ETAS = [0.05, 0.10, 0.15, 0.20, 0.25, 0.30, 0.35, 0.40, 0.45, 0.50, 0.55, 0.60]


def test_f_functions_match_legacy():
    """fmt.cpp:13-54 (margin 1e-10)."""
    pairs = [("Rosenfeld", legacy.rosenfeld_f), ("RSLT", legacy.rslt_f), ("WhiteBearI", legacy.whitebear1_f),
             ("WhiteBearII", legacy.whitebear2_f), ("esFMT", legacy.esfmt_f)]
    for name, lf in pairs:
        m = fmt.FMTModel(name)
        for eta in ETAS:
            f1, _, f2, _, f3, _ = m.f(eta)
            l1, l2, l3 = lf(eta)
            assert float(f1) == pytest.approx(l1, abs=1e-10)
            assert float(f2) == pytest.approx(l2, abs=1e-10)
            assert float(f3) == pytest.approx(l3, abs=1e-10)


def make_test_measures(eta, n2, v_mag, t_diag):
    """fmt.cpp:74-89."""
    Rr = 0.5
    f = 4.0 * math.pi * Rr
    m = {"eta": eta, "n2": n2, "n1": n2 / f, "n0": n2 / (f * Rr),
         "v1": np.array([v_mag, -0.3 * v_mag, 0.1 * v_mag]),
         "v0": np.array([v_mag / f, -0.3 * v_mag / f, 0.1 * v_mag / f]),
         "T": np.array([[t_diag, 0.1, -0.05], [0.1, t_diag * 0.8, 0.02], [-0.05, 0.02, t_diag * 0.6]])}
    m["products"] = fmt.inner_products(m)
    fm = legacy.derived({"eta": eta, "s0": m["n0"], "s1": m["n1"], "s2": n2, "v1": m["v0"], "v2": m["v1"],
                         "T": m["T"]})
    return m, fm


def test_phi3_and_derivatives_match_legacy():
    """fmt.cpp:91-139 (margin 1e-10)."""
    m, fm = make_test_measures(0.3, 2.5, 0.4, 0.3)
    for name, lf in (("Rosenfeld", legacy.rosenfeld_phi3), ("RSLT", legacy.rslt_phi3)):
        mod = fmt.FMTModel(name)
        p, d, dv = lf(fm)
        assert float(mod.phi3(m)) == pytest.approx(p, abs=1e-10)
        assert float(mod.d_phi3_d_n2(m)) == pytest.approx(d, abs=1e-10)
        assert np.allclose(mod.d_phi3_d_v1(m), dv, atol=1e-10, rtol=0)
    m, fm = make_test_measures(0.25, 2.0, 0.3, 0.25)
    for A, B in ((1.0, 0.0), (1.0, -1.0)):
        mod = fmt.FMTModel("esFMT", A, B)
        p, d, dv, dT = legacy.esfmt_phi3(A, B, fm)
        assert float(mod.phi3(m)) == pytest.approx(p, abs=1e-10)
        assert float(mod.d_phi3_d_n2(m)) == pytest.approx(d, abs=1e-10)
        assert np.allclose(mod.d_phi3_d_v1(m), dv, atol=1e-10, rtol=0)
        assert np.allclose(mod.d_phi3_d_T(m), dT, atol=1e-10, rtol=0)
    wb = fmt.FMTModel("WhiteBearI")
    p, d, dv, dT = legacy.esfmt_phi3(1.0, -1.0, fm)
    assert float(wb.phi3(m)) == pytest.approx(p, abs=1e-10)
    assert float(wb.d_phi3_d_n2(m)) == pytest.approx(d, abs=1e-10)
    assert np.allclose(wb.d_phi3_d_T(m), dT, atol=1e-10, rtol=0)


# ---- tests/unit/functionals/hard_sphere.cpp -------------------------------

def _hs(name, rhos, diameters, A=1.0, B=0.0):
    model = Model(GRID, [Species(f"S{i}", d) for i, d in enumerate(diameters)], [], 1.0)
    w = make_weights(fmt.FMTModel(name, A, B), model)
    return hard_sphere(model, [np.full(N, r) for r in rhos], w)


@pytest.mark.parametrize("name", MODELS)
def test_hard_sphere_uniform_free_energy_matches_bulk(name):
    """hard_sphere.cpp:52-116, 263-276 (epsilon 1e-6)."""
    F, _ = _hs(name, [0.5], [D])
    expected = fmt.FMTModel(name).free_energy_density(0.5, D) * 1.6 ** 3
    assert F == pytest.approx(expected, rel=1e-6)


@pytest.mark.parametrize("name", ["Rosenfeld", "WhiteBearII"])
def test_hard_sphere_uniform_force_is_mu_ex_dv(name):
    """hard_sphere.cpp:118-163."""
    _, f = _hs(name, [0.4], [D])
    assert np.max(np.abs(f[0] - f[0].mean())) < 1e-8
    assert f[0][0] == pytest.approx(fmt.FMTModel(name).excess_chemical_potential(0.4, D) * GRID.cell_volume, rel=1e-6)


def test_hard_sphere_zero_density_and_mixture():
    """hard_sphere.cpp:167-248."""
    F, f = _hs("Rosenfeld", [0.0], [D])
    assert F == pytest.approx(0.0, abs=1e-14) and np.max(np.abs(f[0])) < 1e-14
    Fl, _ = _hs("Rosenfeld", [0.2], [D])
    Fh, _ = _hs("Rosenfeld", [0.6], [D])
    assert Fh > Fl
    F, f = _hs("Rosenfeld", [0.3, 0.2], [1.0, 0.8])
    assert F > 0.0 and len(f) == 2
    for s in range(2):
        assert np.max(np.abs(f[s] - f[s].mean())) < 1e-8
    assert abs(f[0][0] - f[1][0]) > 1e-10


def test_fft_conventions():
    """tests/unit/math/fourier.cpp:25-138 and convolution.cpp:13-89."""
    x = np.arange(64, dtype=np.float64).reshape(4, 4, 4)
    assert np.allclose(c2r(r2c(x), (4, 4, 4)) / 64.0, x, atol=1e-10)
    assert r2c(np.ones((4, 4, 4)))[0, 0, 0] == pytest.approx(64.0)
    a = np.zeros((4, 4, 4))
    a[0, 0, 0] = 1.0
    conv = c2r(r2c(a) * r2c(np.ones((4, 4, 4))), (4, 4, 4)) / 64.0
    assert np.allclose(conv, 1.0, atol=1e-10)
    conv = c2r(r2c(a) * r2c(a), (4, 4, 4)) / 64.0
    assert conv[0, 0, 0] == pytest.approx(1.0, abs=1e-12) and np.max(np.abs(conv.reshape(-1)[1:])) < 1e-12
    w = np.full((4, 4, 3), 1.0 / 64.0 + 0j)
    assert np.allclose(convolve(w, r2c(np.ones((4, 4, 4))), (4, 4, 4)), 1.0, atol=1e-10)
