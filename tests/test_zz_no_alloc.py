"""The allocation-free entry point cdft_local_terms_noalloc, for callers that
cannot allocate device memory, against the existing entry point cdft_total.

It computes the ideal-gas and external-field terms with the caller's buffers
and a static device scratch array only.  Two calls in a row, each checked
against cdft_total within the tolerance of the other GPU parity tests (1e-12
relative): a general state, where its F_id, F_ext and N_s must equal entries
2, 3 and 6 of cdft_total's scalar block, and a zero-density state in an
external field, where the hard-sphere and mean-field forces vanish exactly so
its force must equal cdft_total's force.  Both calls also check the force
against (ln max(rho, 1e-300) - mu + V) dV.
This file is collected last so that a run stopping at its first failure has
already run every other test.
"""
import ctypes

import numpy as np
import pytest

import classicaldft_b200 as cd
from classicaldft_b200 import _lib

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _noalloc(rho, vext, mu, dv):
    """rho: (S, n) or (n,); vext the same shape or None; mu: S values."""
    import torch
    L = _lib.lib()
    rho = np.atleast_2d(rho)
    S, n = rho.shape
    mus = np.atleast_1d(mu)
    d_rho = torch.tensor(rho, dtype=torch.float64, device="cuda")
    d_v = None if vext is None else torch.tensor(np.atleast_2d(vext), dtype=torch.float64, device="cuda")
    d_f = torch.full((S, n), np.nan, dtype=torch.float64, device="cuda")
    d_sc = torch.full((2 + S,), np.nan, dtype=torch.float64, device="cuda")
    mu_c = (ctypes.c_double * S)(*mus)
    st = L.cdft_local_terms_noalloc(d_rho.data_ptr(), None if d_v is None else d_v.data_ptr(), mu_c, S, n, dv,
                                    d_f.data_ptr(), d_sc.data_ptr(), torch.cuda.current_stream().cuda_stream)
    assert st == _lib.CDFT_OK, L.cdft_last_error().decode()
    torch.cuda.synchronize()
    f = d_f.cpu().numpy()
    return d_sc.cpu().numpy(), (f[0] if S == 1 else f)


def test_noalloc_local_terms_match_cdft_total_on_two_calls():
    shape, dx = (32, 32, 32), 0.2
    g = cd.Grid(dx=dx, box_size=tuple(k * dx for k in shape), shape=shape)
    model = cd.Model(g, [cd.Species("LJ", 1.0)], [cd.Interaction(0, 0, cd.make_lennard_jones(1.0, 1.0, 2.5))], 1.0)
    w = cd.make_weights(cd.WhiteBearII(), model)
    n = g.total_points
    dv = g.cell_volume
    rng = np.random.default_rng(7)
    states = [
        (0.4 * (1.0 + 0.2 * rng.uniform(-1.0, 1.0, n)), rng.standard_normal(n), 0.7),   # general state
        (np.zeros(n), 3.0 * rng.standard_normal(n), -1.3),                              # zero density
    ]
    for call, (rho, vext, mu) in enumerate(states):
        sc_ref, f_ref = w.engine.total_host(rho, [mu], vext[None, :])
        sc, f = _noalloc(rho, vext, mu, dv)
        for mine, ref in ((sc[0], sc_ref[2]), (sc[1], sc_ref[3]), (sc[2], sc_ref[6])):
            assert abs(mine - ref) <= TOL * max(abs(ref), 1e-300), (call, mine, ref)
        local = (np.log(np.maximum(rho, 1e-300)) - mu + vext) * dv
        assert np.max(np.abs(f - local)) <= TOL * np.max(np.abs(local))
        if call == 1:
            # rho = 0: every channel is exactly zero, the hard-sphere and
            # mean-field forces vanish, and cdft_total's force is the local force
            assert np.max(np.abs(f - f_ref[0])) <= TOL * np.max(np.abs(f_ref[0]))


def test_noalloc_two_species_without_field_on_a_large_grid():
    """64^3 points (more than the 592 x 256 threads of one pass of the
    grid-stride loop), two species and no external field: F_id and N_s equal
    cdft_total's, F_ext is zero and the force is (ln rho - mu) dV; two calls in
    a row."""
    shape, dx = (64, 64, 64), 0.1
    g = cd.Grid(dx=dx, box_size=tuple(k * dx for k in shape), shape=shape)
    model = cd.Model(g, [cd.Species("A", 1.0), cd.Species("B", 0.6)], [], 1.0)
    w = cd.make_weights(cd.WhiteBearII(), model)
    n = g.total_points
    dv = g.cell_volume
    rng = np.random.default_rng(8)
    for call in range(2):
        rho = np.stack([0.3 * (1.0 + 0.3 * rng.uniform(-1.0, 1.0, n)), 0.1 * rng.uniform(0.0, 1.0, n)])
        rho[1, :: 97] = 0.0  # the clamp at 1e-300
        mu = rng.uniform(-1.0, 1.0, 2)
        sc_ref, _ = w.engine.total_host(rho, list(mu), None)
        sc, f = _noalloc(rho, None, mu, dv)
        assert abs(sc[0] - sc_ref[2]) <= TOL * abs(sc_ref[2]), (call, sc[0], sc_ref[2])
        assert sc[1] == 0.0
        for s in range(2):
            assert abs(sc[2 + s] - sc_ref[6 + s]) <= TOL * abs(sc_ref[6 + s]), (call, s)
            local = (np.log(np.maximum(rho[s], 1e-300)) - mu[s]) * dv
            assert np.max(np.abs(f[s] - local)) <= TOL * np.max(np.abs(local)), (call, s)


def test_noalloc_rejects_sizes_beyond_its_scratch():
    L = _lib.lib()
    mu = (ctypes.c_double * 5)(0, 0, 0, 0, 0)
    st = L.cdft_local_terms_noalloc(ctypes.c_void_p(16), None, mu, 5, 10, 1.0, ctypes.c_void_p(16),
                                    ctypes.c_void_p(16), None)
    assert st == _lib.CDFT_ERR_INVALID
    assert b"n_species" in L.cdft_last_error()
