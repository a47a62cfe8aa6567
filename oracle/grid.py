"""Grid, wavevectors and FFTW-convention transforms (oracle, test infrastructure only).

Restates include/dft/grid.hpp and src/math/fourier.cpp of the reference.
Fields are NumPy arrays of shape (nx, ny, nz) in C order, i.e. the flat index
is iz + nz*(iy + ny*ix) (grid.hpp:35-37).  k-space fields have shape
(nx, ny, nz//2+1), the FFTW half-complex layout (grid.hpp:42-63).
"""
from __future__ import annotations

import os
from dataclasses import dataclass

import numpy as np
import scipy.fft as sfft

WORKERS = int(os.environ.get("CDFT_ORACLE_WORKERS", os.cpu_count() or 1))


@dataclass(frozen=True)
class Grid:
    """grid.hpp:26-83.  shape = (nx, ny, nz), dx the spacing, box the lengths."""

    dx: float
    box_size: tuple
    shape: tuple

    @property
    def cell_volume(self) -> float:
        return self.dx * self.dx * self.dx

    @property
    def total_points(self) -> int:
        return int(self.shape[0] * self.shape[1] * self.shape[2])

    @property
    def fourier_shape(self) -> tuple:
        return (self.shape[0], self.shape[1], self.shape[2] // 2 + 1)

    def flat_index(self, ix, iy, iz):
        return iz + self.shape[2] * (iy + self.shape[1] * ix)


def make_grid(dx: float, box) -> Grid:
    """grid.hpp:87-108: validated factory; box must be commensurate with dx."""
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
    return Grid(dx=dx, box_size=tuple(float(b) for b in box), shape=tuple(shape))


def wavevectors(grid: Grid):
    """grid.hpp:42-63: kx, ky, kz broadcastable over the half-complex grid.

    Index i maps to i for i <= n/2 and to i-n otherwise, so the Nyquist index
    of an even axis maps to +k (grid.hpp:53,55).  kz runs over 0..nz/2.
    """
    nx, ny, nz = grid.shape
    dx = grid.dx

    def full(n):
        i = np.arange(n)
        return (2.0 * np.pi / (n * dx)) * np.where(i <= n // 2, i, i - n).astype(np.float64)

    kx = full(nx)[:, None, None]
    ky = full(ny)[None, :, None]
    kz = ((2.0 * np.pi / (nz * dx)) * np.arange(nz // 2 + 1, dtype=np.float64))[None, None, :]
    return kx, ky, kz


def r2c(f: np.ndarray) -> np.ndarray:
    """FourierTransform::forward (fourier.cpp:97-99): unnormalised 3-D r2c."""
    return sfft.rfftn(f, axes=(0, 1, 2), workers=WORKERS)


def c2r(fk: np.ndarray, shape) -> np.ndarray:
    """FourierTransform::backward (fourier.cpp:101-103): unnormalised 3-D c2r.

    scipy's irfftn applies 1/N, FFTW does not, so the result is rescaled by N.
    Its treatment of non-Hermitian input equals ``c2r(hermitian_project(fk))``.
    """
    n = shape[0] * shape[1] * shape[2]
    return sfft.irfftn(fk, s=shape, axes=(0, 1, 2), workers=WORKERS) * float(n)


def hermitian_project(fk: np.ndarray, shape) -> np.ndarray:
    """Project a half-complex array onto the Hermitian subspace that c2r sees.

    The planes kz=0 and (for even nz) kz=nz/2 are self-conjugate under
    k -> -k; on them X'(kx,ky) = (X(kx,ky) + conj(X(-kx,-ky))) / 2.  Every
    other plane is untouched.  An FFTW/pocketfft c2r of X equals the exact
    inverse DFT of X' (the 1-D c2r over z drops Im of the kz=0 and kz=nz/2
    modes after the complex x,y transforms).
    """
    nx, ny, nz = shape
    out = np.array(fk, copy=True)
    planes = [0] + ([nz // 2] if nz % 2 == 0 else [])
    mx = (-np.arange(nx)) % nx
    my = (-np.arange(ny)) % ny
    for p in planes:
        plane = fk[:, :, p]
        mirror = plane[mx][:, my]
        out[:, :, p] = 0.5 * (plane + np.conj(mirror))
    return out


def boundary_mask(grid: Grid) -> np.ndarray:
    """grid.hpp:67-82: 1 on any face of the box, 0 in the interior (flat, uint8)."""
    nx, ny, nz = grid.shape
    m = np.zeros(grid.shape, dtype=np.uint8)
    m[0, :, :] = 1
    m[nx - 1, :, :] = 1
    m[:, 0, :] = 1
    m[:, ny - 1, :] = 1
    m[:, :, 0] = 1
    m[:, :, nz - 1] = 1
    return m.reshape(-1)


def homogeneous_boundary(forces: np.ndarray, mask: np.ndarray) -> np.ndarray:
    """grid.hpp:113-131: boundary entries replaced by their average."""
    f = np.asarray(forces, dtype=np.float64).reshape(-1)
    res = f.copy()
    sel = mask.astype(bool)
    cnt = int(sel.sum())
    if cnt > 0:
        res[sel] = f[sel].sum() / cnt
    return res


def fixed_boundary(forces: np.ndarray, mask: np.ndarray) -> np.ndarray:
    """grid.hpp:135-142: boundary entries set to zero."""
    res = np.asarray(forces, dtype=np.float64).reshape(-1).copy()
    res[mask.astype(bool)] = 0.0
    return res
