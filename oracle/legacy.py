"""Second, independent formula source (oracle, test infrastructure only).

Restates the legacy translations of Lutsko's original classicalDFT that the
reference itself uses as cross-validation oracles
(legacy/classicaldft.hpp:526-793).  Measures follow the legacy naming:
s0, s1, s2, v1 (= the modern v0), v2 (= the modern v1), T.
"""
from __future__ import annotations

import math

import numpy as np

PI = math.pi


def derived(fm: dict) -> dict:
    """legacy/classicaldft.hpp:544-572 calculate_derived_quantities."""
    v1 = np.asarray(fm["v1"], dtype=np.float64)
    v2 = np.asarray(fm["v2"], dtype=np.float64)
    T = np.asarray(fm["T"], dtype=np.float64)
    out = dict(fm)
    out["v1_v2"] = float(v1 @ v2)
    out["v2_v2"] = float(v2 @ v2)
    out["vT"] = v2 @ T
    out["Tv"] = T @ v2
    out["vTv"] = float(v2 @ (T @ v2))
    TT = T @ T
    out["TT"] = TT
    out["T2"] = float(np.sum(T * T.T))
    out["T3"] = float(np.sum(T * TT.T))
    return out


def rosenfeld_f(eta):
    """legacy :576-579."""
    return math.log(1.0 - eta), 1.0 / (1.0 - eta), 1.0 / ((1.0 - eta) ** 2)


def rslt_f(x):
    """legacy :594-600."""
    if x < 1e-12:
        f3 = 1.5 + (8.0 / 3.0) * x + 3.75 * x * x + 4.8 * x * x * x
    else:
        f3 = (1.0 / (x * (1.0 - x) * (1.0 - x))) + (math.log(1.0 - x) / (x * x))
    return math.log(1.0 - x), 1.0 / (1.0 - x), f3


def whitebear1_f(x):
    """legacy :656-663."""
    return rslt_f(x)


def whitebear2_f(x):
    """legacy :667-678."""
    if x < 1e-12:
        f2 = 1.0 + x * (1.0 + x * ((10.0 / 9.0) + (7.0 / 6.0) * x))
        f3 = 1.5 + (7.0 / 3.0) * x + 3.25 * x * x + 4.2 * x * x * x
    else:
        f2 = (1.0 / 3.0) + (4.0 / 3.0) * (1.0 / (1.0 - x)) + (2.0 / (3.0 * x)) * math.log(1.0 - x)
        f3 = -((1.0 - 3.0 * x + x * x) / (x * (1.0 - x) * (1.0 - x))) - (1.0 / (x * x)) * math.log(1.0 - x)
    return math.log(1.0 - x), f2, f3


def esfmt_f(eta):
    """legacy :623-626."""
    return rosenfeld_f(eta)


def rosenfeld_phi3(fm):
    """legacy :583-591: Phi3, dPhi3/dS2, dPhi3/dV2[k]."""
    s2 = fm["s2"]
    p = (1.0 / (24.0 * PI)) * (s2 ** 3 - 3.0 * s2 * fm["v2_v2"])
    d = (1.0 / (24.0 * PI)) * (3.0 * s2 * s2 - 3.0 * fm["v2_v2"])
    dv = [(1.0 / (24.0 * PI)) * (-6.0 * s2 * fm["v2"][k]) for k in range(3)]
    return p, d, dv


def rslt_phi3(fm):
    """legacy :604-620."""
    s2 = fm["s2"]
    if s2 < 1e-20:
        return 0.0, 0.0, [0.0, 0.0, 0.0]
    psi = fm["v2_v2"] / (s2 * s2)
    p = (1.0 / (36.0 * PI)) * s2 ** 3 * (1.0 - psi) ** 3
    d = (1.0 / (12.0 * PI)) * s2 * s2 * (1.0 + psi) * (1.0 - psi) ** 2
    dv = [-(1.0 / (6.0 * PI)) * s2 * fm["v2"][k] * (1.0 - psi) ** 2 for k in range(3)]
    return p, d, dv


def esfmt_phi3(A, B, fm):
    """legacy :627-640: Phi3, dPhi3/dS2, dPhi3/dV2[k], dPhi3/dT[j][k]."""
    s2 = fm["s2"]
    p = (A / (24.0 * PI)) * (s2 ** 3 - 3.0 * s2 * fm["v2_v2"] + 3.0 * fm["vTv"] - fm["T3"]) + \
        (B / (24.0 * PI)) * (s2 ** 3 - 3.0 * s2 * fm["T2"] + 2.0 * fm["T3"])
    d = (A / (24.0 * PI)) * (3.0 * s2 * s2 - 3.0 * fm["v2_v2"]) + (B / (24.0 * PI)) * (3.0 * s2 * s2 - 3.0 * fm["T2"])
    dv = [(A / (24.0 * PI)) * (-6.0 * s2 * fm["v2"][k] + 3.0 * fm["vT"][k] + 3.0 * fm["Tv"][k]) for k in range(3)]
    dT = np.zeros((3, 3))
    for j in range(3):
        for k in range(3):
            dT[j, k] = (A / (8.0 * PI)) * (fm["v2"][j] * fm["v2"][k] - fm["TT"][k][j]) + \
                (B / (4.0 * PI)) * (-s2 * fm["T"][k][j] + fm["TT"][k][j])
    return p, d, dv, dT


def watt2_lj(sigma, eps, rcut, r2):
    """legacy :697-718: WCA attractive tail of the cut-and-shifted LJ at r^2."""
    with np.errstate(divide="ignore", invalid="ignore", over="ignore"):
        y2 = np.float64(sigma * sigma) / np.float64(r2)   # IEEE: r2 = 0 gives inf, as in C++
        y6 = y2 * y2 * y2
        vr2 = float(4.0 * eps * (y6 * y6 - y6))
    y = sigma / rcut
    y3 = y * y * y
    y6s = y3 * y3
    shift = 4.0 * eps * (y6s * y6s - y6s)
    rmin = math.pow(2.0, 1.0 / 6.0) * sigma
    y = sigma / rmin
    y3 = y * y * y
    y6s = y3 * y3
    vmin = 4.0 * eps * (y6s * y6s - y6s) - shift
    if r2 >= rcut * rcut:
        return 0.0
    if r2 < rmin * rmin:
        return vmin
    return vr2 - shift


def generate_weight_qf(sigma, eps, rcut, sx, sy, sz, dx):
    """legacy :720-737: 27-point QF cell weight."""
    vv = (1.0 / 3.0,) * 3
    pt = (-0.5, 0.0, 0.5)
    total = 0.0
    for i in range(3):
        for j in range(3):
            for k in range(3):
                r2 = ((sx + pt[i]) ** 2 + (sy + pt[j]) ** 2 + (sz + pt[k]) ** 2) * dx * dx
                total += vv[i] * vv[j] * vv[k] * watt2_lj(sigma, eps, rcut, r2)
    return total


def compute_a_vdw_qf(sigma, eps, rcut, kT, dx):
    """legacy :739-760."""
    lim = 1 + int(rcut / dx)
    total = 0.0
    g = dx ** 6
    for ix in range(-(lim + 1), lim + 2):
        for iy in range(-(lim + 1), lim + 2):
            for iz in range(-(lim + 1), lim + 2):
                a, b, c = sorted((abs(ix), abs(iy), abs(iz)), reverse=True)
                total += g * generate_weight_qf(sigma, eps, rcut, a, b, c, dx)
    return total / (dx * dx * dx) / kT


# ------------------------------------------------- legacy phase solvers
# legacy/classicaldft.hpp:799-907 (DFT_Coex.cpp of the original code): the
# spinodal by golden-section search on P(rho), mu inversion by bisection and
# the coexistence by bracketing P_v - P_l.  The reference cross-checks its
# PhaseSearch against these to 1e-6 (tests/integration/functionals/bulk/coexistence.cpp).


def legacy_find_spinodal(pressure, xmax, dx, tol=1e-8):
    x = 2 * dx
    p0 = pressure(dx)
    p = pressure(2 * dx)
    dp = p - p0
    if dp < 0:
        raise RuntimeError("Could not get started in findSpinodal")
    while dp > 0 and x < xmax - dx:
        dp = -p
        x += dx
        p = pressure(x)
        dp += p
    if x >= xmax - dx:
        raise RuntimeError("Xmax exceeded in findSpinodal (max)")
    r = (3.0 - math.sqrt(5.0)) / 2.0

    def golden(a, b, maximum):
        u = a + r * (b - a)
        v = b - r * (b - a)
        fu, fv = pressure(u), pressure(v)
        while True:
            if (fu > fv) if maximum else (fu < fv):
                b, v, fv = v, u, fu
                u = a + r * (b - a)
                fu = pressure(u)
            else:
                a, u, fu = u, v, fv
                v = b - r * (b - a)
                fv = pressure(v)
            if not (b - a > tol):
                return (a + b) / 2

    xs1 = golden(x - 2 * dx, x, True)
    x = xs1
    p = pressure(x)
    while True:
        dp = -p
        x += dx
        p = pressure(x)
        dp += p
        if not (dp < 0 and x < xmax - dx):
            break
    if x >= xmax - dx:
        raise RuntimeError("Xmax exceeded in findSpinodal (min)")
    xs2 = golden(x - 2 * dx, x, False)
    return xs1, xs2


def legacy_find_density_from_mu(chem, mu, xmin, xmax, tol=1e-8):
    mu1, mu2 = chem(xmin), chem(xmax)
    if mu1 > mu2:
        xmin, xmax, mu1, mu2 = xmax, xmin, mu2, mu1
    if mu2 < mu or mu1 > mu:
        raise RuntimeError("find_density_from_mu: target mu out of range")
    while True:
        x = (xmin + xmax) / 2
        mux = chem(x)
        if mux > mu:
            xmax, mu2 = x, mux
        else:
            xmin, mu1 = x, mux
        if not (mu2 - mu1 > tol):
            return (xmin + xmax) / 2


def legacy_find_coex(pressure, chem, xmax, dx, tol=1e-8):
    xs1, xs2 = legacy_find_spinodal(pressure, xmax, dx, tol)
    xvap = xs1
    xliq = legacy_find_density_from_mu(chem, chem(xvap), xs2, xmax - dx, tol)
    dp1 = pressure(xvap) - pressure(xliq)
    while True:
        dp2 = dp1
        xvap /= 1.1
        xliq = legacy_find_density_from_mu(chem, chem(xvap), xs2, xmax - dx, tol)
        dp1 = pressure(xvap) - pressure(xliq)
        if not (xvap > 1e-40 and ((dp1 < 0) == (dp2 < 0))):
            break
    if xvap < 1e-40:
        raise RuntimeError("findCoex bracket failed")
    y1, y2 = xvap, xvap * 1.1
    while True:
        y = (y1 + y2) / 2
        xliq = legacy_find_density_from_mu(chem, chem(y), xs2, xmax - dx, tol)
        dp = pressure(y) - pressure(xliq)
        if (dp < 0) == (dp1 < 0):
            y1, dp1 = y, dp
        else:
            y2, dp2 = y, dp
        if not (abs(y2 - y1) > xvap * tol):
            break
    rv = (y1 + y2) / 2
    return rv, legacy_find_density_from_mu(chem, chem(rv), xs2, xmax - dx, tol)
