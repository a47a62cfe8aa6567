"""FMT weights, measures and models (oracle, test infrastructure only).

Restates include/dft/functionals/fmt/{weights,measures,models}.hpp.  All
arithmetic is FP64 and vectorised over grid points / wavevectors.
"""
from __future__ import annotations

import math

import numpy as np

from .grid import Grid, wavevectors

PI = math.pi
INV_24PI = 1.0 / (24.0 * PI)
INV_8PI = 1.0 / (8.0 * PI)
INV_4PI = 1.0 / (4.0 * PI)
INV_36PI = 1.0 / (36.0 * PI)

# ---------------------------------------------------------------- weights


def weight_kernels(k: np.ndarray, R: float):
    """weights.hpp:91-137: the |k|-only factors (w3, w2, fv, A, B) of one sphere.

    w3 = 4pi (sin kR - kR cos kR)/k^3, w2 = 4pi R sin kR / k,
    wv2_a = i k_a fv, wT_ij = A k_i k_j / k^2 + B delta_ij, each with the
    k < 1e-12 limits of the reference.
    """
    small = k < 1e-12
    ks = np.where(small, 1.0, k)
    kR = ks * R
    s = np.sin(kR)
    c = np.cos(kR)
    w3 = np.where(small, (4.0 * PI / 3.0) * R * R * R, 4.0 * PI * (s - kR * c) / (ks * ks * ks))
    w2 = np.where(small, 4.0 * PI * R * R, 4.0 * PI * R * s / ks)
    fv = np.where(small, 0.0, -4.0 * PI * (R * c - s / ks) / (ks * ks))
    k2 = ks * ks
    k3 = k2 * ks
    R2 = R * R
    gp_over_k = 4.0 * PI * R * (R * c / k2 - s / k3)
    gpp = 4.0 * PI * R * (-R2 * s / ks - 2.0 * R * c / k2 + 2.0 * s / k3)
    A = np.where(small, 0.0, -(gpp - gp_over_k) / R2)
    B = np.where(small, (4.0 * PI / 3.0) * R * R, -gp_over_k / R2)
    return w3, w2, fv, A, B


TENSOR_PAIRS = ((0, 0), (0, 1), (0, 2), (1, 1), (1, 2), (2, 2))


def generate_weights(diameter: float, grid: Grid) -> dict:
    """weights.hpp:144-183: the 11 stored k-space channels of one species, x 1/N.

    Returns {"w3", "w2", "wv2": [3], "wT": {(i,j): ...}} with complex arrays on
    the half-complex grid.
    """
    R = 0.5 * diameter
    inv_n = 1.0 / float(grid.total_points)
    kx, ky, kz = wavevectors(grid)
    shp = grid.fourier_shape
    KX = np.broadcast_to(kx, shp)
    KY = np.broadcast_to(ky, shp)
    KZ = np.broadcast_to(kz, shp)
    norm2 = KX * KX + KY * KY + KZ * KZ
    k = np.sqrt(norm2)
    w3, w2, fv, A, B = weight_kernels(k, R)
    kk = (KX, KY, KZ)
    inv_k2 = np.where(k > 1e-12, 1.0 / np.where(k > 1e-12, norm2, 1.0), 0.0)
    out = {
        "w3": (w3 * inv_n).astype(np.complex128),
        "w2": (w2 * inv_n).astype(np.complex128),
        "wv2": [1j * (kk[a] * fv * inv_n) for a in range(3)],
        "wT": {},
    }
    for (i, j) in TENSOR_PAIRS:
        d = 1.0 if i == j else 0.0
        out["wT"][(i, j)] = ((A * kk[i] * kk[j] * inv_k2 + B * d) * inv_n).astype(np.complex128)
    return out


# ---------------------------------------------------------------- measures


def inner_products(m: dict) -> dict:
    """measures.hpp:34-44: v0.v1, v1.v1, tr T^2, tr T^3, v1 T v1."""
    v0, v1, T = m["v0"], m["v1"], m["T"]
    dot01 = v0[0] * v1[0] + v0[1] * v1[1] + v0[2] * v1[2]
    dot11 = v1[0] * v1[0] + v1[1] * v1[1] + v1[2] * v1[2]
    TT = np.einsum("ik...,kj...->ij...", T, T)
    T2 = np.einsum("ii...->...", TT)
    T3 = np.einsum("ik...,ki...->...", TT, T)
    qf = np.einsum("i...,ij...,j...->...", v1, T, v1)
    return {"dot_v0_v1": dot01, "dot_v1_v1": dot11, "trace_T2": T2, "trace_T3": T3,
            "quadratic_form": qf, "TT": TT}


def make_uniform_measures(density: float, diameter: float) -> dict:
    """measures.hpp:49-65: measures of a uniform fluid."""
    d = diameter
    r = 0.5 * d
    n2 = PI * density * d * d
    t = n2 / 3.0
    m = {
        "eta": np.float64((PI / 6.0) * density * d * d * d),
        "n2": np.float64(n2),
        "n1": np.float64(r * density),
        "n0": np.float64(density),
        "v0": np.zeros(3),
        "v1": np.zeros(3),
        "T": np.diag([t, t, t]).astype(np.float64),
    }
    m["products"] = inner_products(m)
    return m


# ---------------------------------------------------------------- models


class FMTModel:
    """models.hpp:115-419: one FMT model (name, f-functions, Phi3 family).

    ``name`` is one of Rosenfeld, RSLT, WhiteBearI, WhiteBearII, esFMT.
    ``f(eta)`` returns (f1, f1', f2, f2', f3, f3') elementwise; the primes are
    the closed-form derivatives of the same expressions the reference feeds
    to autodiff (models.hpp:59-61), including the eta < 1e-6 Taylor branches.
    """

    NAMES = ("Rosenfeld", "RSLT", "WhiteBearI", "WhiteBearII", "esFMT")

    def __init__(self, name: str, A: float = 1.0, B: float = 0.0):
        if name not in self.NAMES:
            raise ValueError(f"Unknown FMT model: {name}")
        self.name = name
        self.A = float(A)
        self.B = float(B)

    @property
    def needs_tensor(self) -> bool:
        return self.name in ("WhiteBearI", "WhiteBearII", "esFMT")

    # --- f-functions -------------------------------------------------------
    def f(self, eta):
        eta = np.asarray(eta, dtype=np.float64)
        with np.errstate(divide="ignore", invalid="ignore", over="ignore"):
            e = 1.0 - eta
            f1 = np.log(1.0 - eta)                      # models.hpp:157-160
            df1 = -1.0 / e
            if self.name == "WhiteBearII":               # models.hpp:280-286
                t = eta < 1e-6
                f2a = 1.0 + eta * (1.0 + eta * (10.0 / 9.0 + (7.0 / 6.0) * eta))
                df2a = 1.0 + eta * (2.0 * (10.0 / 9.0) + 3.0 * (7.0 / 6.0) * eta)
                lg = np.log(1.0 - eta)
                f2b = 1.0 / 3.0 + (4.0 / 3.0) / e + 2.0 / (3.0 * eta) * lg
                df2b = (4.0 / 3.0) / (e * e) - (2.0 / (3.0 * eta * eta)) * lg - 2.0 / (3.0 * eta * e)
                f2 = np.where(t, f2a, f2b)
                df2 = np.where(t, df2a, df2b)
            else:                                        # models.hpp:162
                f2 = 1.0 / e
                df2 = 1.0 / (e * e)
            if self.name in ("Rosenfeld", "esFMT"):      # models.hpp:164-167
                f3 = 1.0 / (e * e)
                df3 = 2.0 / (e * e * e)
            elif self.name in ("RSLT", "WhiteBearI"):    # models.hpp:198-205, 248-256
                t = eta < 1e-6
                if self.name == "RSLT":
                    f3a = 1.0 + (2.0 / 3.0) * eta + 0.5 * eta * eta
                    df3a = 2.0 / 3.0 + eta
                else:
                    f3a = 1.5 + eta * (8.0 / 3.0 + eta * (15.0 / 4.0 + (24.0 / 5.0) * eta))
                    df3a = 8.0 / 3.0 + eta * (2.0 * (15.0 / 4.0) + 3.0 * (24.0 / 5.0) * eta)
                h = eta * e * e
                lg = np.log(1.0 - eta)
                f3b = 1.0 / h + lg / (eta * eta)
                df3b = -(e * (e - 2.0 * eta)) / (h * h) - 1.0 / (e * eta * eta) - 2.0 * lg / (eta * eta * eta)
                f3 = np.where(t, f3a, f3b)
                df3 = np.where(t, df3a, df3b)
            else:                                        # WhiteBearII, models.hpp:288-295
                t = eta < 1e-6
                f3a = 1.5 + (7.0 / 3.0) * eta + 3.25 * eta * eta + 4.2 * eta * eta * eta
                df3a = 7.0 / 3.0 + 6.5 * eta + 12.6 * eta * eta
                g = 1.0 - 3.0 * eta + eta * eta
                gp = -3.0 + 2.0 * eta
                h = eta * e * e
                hp = e * (e - 2.0 * eta)
                lg = np.log(1.0 - eta)
                f3b = -(g / h) - lg / (eta * eta)
                df3b = -(gp * h - g * hp) / (h * h) + 1.0 / (e * eta * eta) + 2.0 * lg / (eta * eta * eta)
                f3 = np.where(t, f3a, f3b)
                df3 = np.where(t, df3a, df3b)
        return f1, df1, f2, df2, f3, df3

    # --- Phi3 family -------------------------------------------------------
    def phi3(self, m):
        p = m["products"]
        n2 = m["n2"]
        if self.name == "Rosenfeld":                     # models.hpp:169-172
            return INV_24PI * (n2 * n2 * n2 - 3.0 * n2 * p["dot_v1_v1"])
        if self.name == "RSLT":                          # models.hpp:207-214
            with np.errstate(divide="ignore", invalid="ignore"):
                xi = np.minimum(p["dot_v1_v1"] / (n2 * n2), 1.0)
                q = 1.0 - xi
                val = INV_36PI * n2 * n2 * n2 * q * q * q
            return np.where(n2 < 1e-30, 0.0, val)
        if self.name in ("WhiteBearI", "WhiteBearII"):   # models.hpp:22-27
            return INV_24PI * 3.0 * (n2 * p["trace_T2"] - n2 * p["dot_v1_v1"] + p["quadratic_form"] - p["trace_T3"])
        A, B = self.A, self.B                            # models.hpp:326-332
        phi_a = n2 * n2 * n2 - 3.0 * n2 * p["dot_v1_v1"] + 3.0 * p["quadratic_form"] - p["trace_T3"]
        phi_b = n2 * n2 * n2 - 3.0 * n2 * p["trace_T2"] + 2.0 * p["trace_T3"]
        return INV_24PI * (A * phi_a + B * phi_b)

    def d_phi3_d_n2(self, m):
        p = m["products"]
        n2 = m["n2"]
        if self.name == "Rosenfeld":                     # models.hpp:174-177
            return INV_8PI * (n2 * n2 - p["dot_v1_v1"])
        if self.name == "RSLT":                          # models.hpp:216-223
            with np.errstate(divide="ignore", invalid="ignore"):
                xi = np.minimum(p["dot_v1_v1"] / (n2 * n2), 1.0)
                q = 1.0 - xi
                val = INV_36PI * 3.0 * n2 * n2 * q * q * (1.0 + xi)
            return np.where(n2 < 1e-30, 0.0, val)
        if self.name in ("WhiteBearI", "WhiteBearII"):   # models.hpp:29-32
            return INV_24PI * 3.0 * (p["trace_T2"] - p["dot_v1_v1"])
        A, B = self.A, self.B                            # models.hpp:334-339
        da = 3.0 * n2 * n2 - 3.0 * p["dot_v1_v1"]
        db = 3.0 * n2 * n2 - 3.0 * p["trace_T2"]
        return INV_24PI * (A * da + B * db)

    def d_phi3_d_v1(self, m):
        n2 = m["n2"]
        v1 = m["v1"]
        if self.name == "Rosenfeld":                     # models.hpp:179-182
            return -INV_4PI * n2 * v1
        if self.name == "RSLT":                          # models.hpp:225-232
            p = m["products"]
            with np.errstate(divide="ignore", invalid="ignore"):
                xi = np.minimum(p["dot_v1_v1"] / (n2 * n2), 1.0)
                q = 1.0 - xi
                val = INV_36PI * (-6.0) * n2 * q * q * v1
            return np.where(n2 < 1e-30, 0.0, val)
        T = m["T"]
        vT = np.einsum("j...,ji...->i...", v1, T)
        Tv = np.einsum("ij...,j...->i...", T, v1)
        if self.name in ("WhiteBearI", "WhiteBearII"):   # models.hpp:34-37
            return INV_24PI * (-6.0 * n2 * v1 + 3.0 * vT + 3.0 * Tv)
        return INV_24PI * self.A * (-6.0 * n2 * v1 + 3.0 * (vT + Tv))   # models.hpp:341-346

    def d_phi3_d_T(self, m):
        """Full 3x3 (i, j) array of dPhi3/dT_ij (models.hpp:39-45, 348-357)."""
        n2 = m["n2"]
        v1 = m["v1"]
        T = m["T"]
        TT = m["products"]["TT"]
        TTji = np.swapaxes(TT, 0, 1)
        Tji = np.swapaxes(T, 0, 1)
        vv = np.einsum("i...,j...->ij...", v1, v1)
        if self.name in ("WhiteBearI", "WhiteBearII"):
            return INV_8PI * (vv + 2.0 * n2 * Tji - 3.0 * TTji)
        return INV_8PI * self.A * (vv - TTji) + (1.0 / (4.0 * PI)) * self.B * (-n2 * Tji + TTji)

    # --- Phi and derivatives ------------------------------------------------
    def phi(self, m):
        """models.hpp:49-54."""
        f1, _, f2, _, f3, _ = self.f(m["eta"])
        return -m["n0"] * f1 + (m["n1"] * m["n2"] - m["products"]["dot_v0_v1"]) * f2 + self.phi3(m) * f3

    def d_phi(self, m):
        """models.hpp:57-81: dPhi/d{eta, n0, n1, n2, v0, v1, T}."""
        f1, df1, f2, df2, f3, df3 = self.f(m["eta"])
        p3 = self.phi3(m)
        p = m["products"]
        dm = {
            "d_eta": -m["n0"] * df1 + (m["n1"] * m["n2"] - p["dot_v0_v1"]) * df2 + p3 * df3,
            "d_n0": -f1,
            "d_n1": m["n2"] * f2,
            "d_n2": m["n1"] * f2 + self.d_phi3_d_n2(m) * f3,
            "d_v0": -m["v1"] * f2,
            "d_v1": -m["v0"] * f2 + self.d_phi3_d_v1(m) * f3,
        }
        if self.needs_tensor:
            dm["d_T"] = self.d_phi3_d_T(m) * f3
        else:
            dm["d_T"] = np.zeros_like(m["T"])
        return dm

    def free_energy_density(self, density: float, diameter: float) -> float:
        """models.hpp:142-144."""
        return float(self.phi(make_uniform_measures(density, diameter)))

    def excess_chemical_potential(self, density: float, diameter: float) -> float:
        """models.hpp:84-106."""
        m = make_uniform_measures(density, diameter)
        dm = self.d_phi(m)
        d = diameter
        r = 0.5 * d
        mu = (float(dm["d_eta"]) * (PI / 6.0) * d * d * d + float(dm["d_n2"]) * PI * d * d
              + float(dm["d_n1"]) * r + float(dm["d_n0"]) * 1.0)
        if self.needs_tensor:
            dt = PI * d * d / 3.0
            for j in range(3):
                mu += float(dm["d_T"][j, j]) * dt
        return mu
