"""Crystal lattices and the Gaussian-peak profile (oracle, test infrastructure only).

Restates src/crystal.cpp:14-279 (unit cells, tiling, scaling, XYZ/CSV
export) in NumPy, and the library's Gaussian-peak initialiser by a direct
sum over all sites.
"""
from __future__ import annotations

import math

import numpy as np

BCC, FCC, HCP = 0, 1, 2
O001, O010, O100, O110, O101, O011, O111 = range(7)


def _unit_cell(structure, orientation):
    """crystal.cpp:80-200: (basis positions (k, 3), cell edges (3,))."""
    fcc = [[0.0, 0.0, 0.0], [0.5, 0.5, 0.0], [0.5, 0.0, 0.5], [0.0, 0.5, 0.5]]
    bcc = [[0.0, 0.0, 0.0], [0.5, 0.5, 0.5]]
    if structure == BCC:
        a = 2.0 / math.sqrt(3.0)
        if orientation in (O001, O010, O100):
            atoms, dims = bcc, [a, a, a]
        elif orientation in (O110, O101, O011):
            atoms, dims = fcc, [a, a, a]
            two = {O110: (0, 1), O101: (0, 2), O011: (1, 2)}[orientation]
            for d in two:
                dims[d] *= math.sqrt(2.0)
        else:
            atoms = [[1 / 6, 0.5, 0.0], [0.0, 0.0, 1 / 3], [1 / 6, 0.5, 0.5], [0.0, 0.0, 5 / 6],
                     [3 / 6, 0.5, 1 / 3], [1 / 3, 0.0, 2 / 3], [3 / 6, 0.5, 5 / 6], [1 / 3, 0.0, 1 / 6],
                     [5 / 6, 0.5, 2 / 3], [2 / 3, 0.0, 0.0], [5 / 6, 0.5, 1 / 6], [2 / 3, 0.0, 0.5]]
            dims = [2.0 * math.sqrt(2.0), 2.0 * math.sqrt(2.0 / 3.0), 2.0]
    elif structure == FCC:
        if orientation in (O001, O010, O100):
            atoms, dims = fcc, [math.sqrt(2.0)] * 3
        elif orientation in (O110, O101, O011):
            atoms, dims = bcc, [1.0, 1.0, 1.0]
            dims[{O110: 2, O101: 1, O011: 0}[orientation]] *= math.sqrt(2.0)
        else:
            atoms = [[0.0, 0.0, 0.0], [0.5, 0.5, 0.0], [0.5, 1 / 6, 1 / 3], [0.0, 4 / 6, 1 / 3],
                     [0.0, 2 / 6, 2 / 3], [0.5, 5 / 6, 2 / 3]]
            dims = [1.0, math.sqrt(3.0), math.sqrt(6.0)]
    elif structure == HCP:
        if orientation not in (O001, O010, O100):
            raise ValueError("HCP only supports orientations 001, 010, 100")
        atoms = [[0.0, 0.0, 0.0], [0.5, 0.5, 0.0], [0.0, 2.0 / 6.0, 0.5], [0.5, 5.0 / 6.0, 0.5]]
        dims = [1.0, math.sqrt(3.0), math.sqrt(8.0 / 3.0)]
    else:
        raise ValueError("unknown structure")
    pos = np.array(atoms, dtype=np.float64) * np.array(dims)
    dims = list(dims)
    if structure == HCP and orientation == O010:  # crystal.cpp:47-54, 187-190
        pos = np.stack([pos[:, 0], -pos[:, 2], pos[:, 1]], axis=1)
        box = np.array([dims[0], dims[2], dims[1]])
        pos = np.fmod(pos, box)
        pos = np.where(pos < 0.0, pos + box, pos)
        dims[1], dims[2] = dims[2], dims[1]
    elif structure == HCP and orientation == O100:  # crystal.cpp:56-62, 191-194
        pos = np.stack([-pos[:, 2], pos[:, 1], pos[:, 0]], axis=1)
        box = np.array([dims[2], dims[1], dims[0]])
        pos = np.fmod(pos, box)
        pos = np.where(pos < 0.0, pos + box, pos)
        dims[0], dims[2] = dims[2], dims[0]
    return pos, np.array(dims)


def build_lattice(structure, orientation, shape=(1, 1, 1)):
    """crystal.cpp:205-245: (positions (n, 3), dimensions (3,))."""
    if len(shape) != 3:
        raise ValueError("Shape must have exactly 3 elements")
    if min(shape) <= 0:
        raise ValueError("Number of unit cells must be strictly positive in all directions")
    atoms, dims = _unit_cell(structure, orientation)
    rows = []
    for iz in range(shape[2]):
        for iy in range(shape[1]):
            for ix in range(shape[0]):
                rows.append(atoms + np.array([float(ix) * dims[0], float(iy) * dims[1], float(iz) * dims[2]]))
    return np.concatenate(rows, axis=0), dims * np.array(shape, dtype=np.float64)


def export_text(positions, fmt):
    """crystal.cpp:257-279 (C++ default stream formatting, 6 significant digits)."""
    lines = []
    if fmt == 0:
        lines.append(str(len(positions)))
        lines.append("Crystal lattice")
        lines += [f"Ar {x:g} {y:g} {z:g}" for x, y, z in positions]
    else:
        lines.append("x,y,z")
        lines += [f"{x:g},{y:g},{z:g}" for x, y, z in positions]
    return "\n".join(lines) + "\n"


def gaussian_peaks(shape, dx, sites, alpha, amplitude, background=0.0):
    """Direct sum over every site with minimum-image distances, peaks cut at alpha r^2 = 40."""
    n = np.array(shape)
    L = n * dx
    g = np.stack(np.meshgrid(*[np.arange(k) * dx for k in shape], indexing="ij"), axis=-1).reshape(-1, 3)
    out = np.full(g.shape[0], float(background))
    for s in np.asarray(sites, dtype=np.float64).reshape(-1, 3):
        d = g - s
        d -= L * np.rint(d / L)
        a = alpha * np.sum(d * d, axis=1)
        out += amplitude * np.where(a <= 40.0, np.exp(-np.minimum(a, 40.0)), 0.0)
    return out
