"""Crystal lattices (src/crystal.cpp, include/dft/types.hpp:51-86) and the
Gaussian-peak crystal density initialiser.

``build_lattice`` and ``Lattice.export_to`` call the library's host code;
``gaussian_peaks`` fills a density on the GPU from lattice sites.
"""
from __future__ import annotations

import ctypes
import enum
import math
from dataclasses import dataclass

import numpy as np

from . import _lib


class Structure(enum.IntEnum):
    """types.hpp:52-56."""

    BCC = 0
    FCC = 1
    HCP = 2


class Orientation(enum.IntEnum):
    """types.hpp:58-66."""

    _001 = 0
    _010 = 1
    _100 = 2
    _110 = 3
    _101 = 4
    _011 = 5
    _111 = 6


class ExportFormat(enum.IntEnum):
    """types.hpp:68-71."""

    XYZ = 0
    CSV = 1


def _shape3(shape):
    shape = [int(s) for s in shape]
    if len(shape) != 3:
        raise ValueError("Shape must have exactly 3 elements")
    return (ctypes.c_long * 3)(*shape), shape


@dataclass
class Lattice:
    """types.hpp:73-83: positions (n, 3) with unit nearest-neighbour distance."""

    structure: Structure
    orientation: Orientation
    shape: list
    dimensions: np.ndarray
    positions: np.ndarray

    def scaled_positions(self, scale):
        """crystal.cpp:247-255: by a nearest-neighbour distance (scalar) or
        onto a box (3 edges, anisotropic)."""
        if np.ndim(scale) == 0:
            return self.positions * float(scale)
        box = np.asarray(scale, dtype=np.float64).reshape(3)
        return self.positions * (box / self.dimensions)

    def export_to(self, filename, format: ExportFormat = ExportFormat.XYZ):
        """crystal.cpp:257-279."""
        pos = np.ascontiguousarray(self.positions, dtype=np.float64)
        _lib.check(_lib.lib().cdft_lattice_export(pos.ctypes.data_as(_lib.c_double_p), pos.shape[0],
                                                  str(filename).encode(), int(format)))


def build_lattice(structure: Structure, orientation: Orientation, shape=(1, 1, 1)) -> Lattice:
    """crystal.cpp:205-245."""
    L = _lib.lib()
    c_shape, shape = _shape3(shape)
    n = ctypes.c_long()
    _lib.check(L.cdft_lattice_size(int(structure), int(orientation), c_shape, ctypes.byref(n)))
    pos = np.empty((n.value, 3), dtype=np.float64)
    dims = np.empty(3, dtype=np.float64)
    _lib.check(L.cdft_build_lattice(int(structure), int(orientation), c_shape, pos.ctypes.data_as(_lib.c_double_p),
                                    n.value, dims.ctypes.data_as(_lib.c_double_p)))
    return Lattice(Structure(structure), Orientation(orientation), shape, dims, pos)


def gaussian_peaks(grid, sites, alpha, amplitude=None, background=0.0, out=None):
    """rho = background + amplitude * sum_i exp(-alpha |r - R_i|^2) on the
    grid (a float64 CUDA tensor of grid.total_points), minimum-image
    distances, peaks cut at alpha r^2 = 40.  amplitude defaults to
    (alpha / pi)^(3/2): one particle per site."""
    import torch
    sites = np.ascontiguousarray(np.asarray(sites, dtype=np.float64).reshape(-1, 3))
    if amplitude is None:
        amplitude = (alpha / math.pi) ** 1.5
    n = grid.total_points
    if out is None:
        out = torch.empty(n, dtype=torch.float64, device="cuda")
    elif not (out.is_cuda and out.dtype == torch.float64 and out.is_contiguous() and out.numel() == n):
        raise ValueError("out: a contiguous float64 CUDA tensor of grid.total_points")
    c_shape, _ = _shape3(grid.shape)
    _lib.check(_lib.lib().cdft_gaussian_peaks(c_shape, grid.dx, sites.ctypes.data_as(_lib.c_double_p),
                                              sites.shape[0], float(alpha), float(amplitude), float(background),
                                              out.data_ptr(), torch.cuda.current_stream().cuda_stream))
    return out
