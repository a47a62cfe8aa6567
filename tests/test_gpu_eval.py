"""GPU parity of one F[rho] + dF/drho evaluation against the FP64 oracle.

Every call goes through the C ABI (cdft_total / cdft_total_device) of
libcdft_b200.so.  Tolerances (FP64 path): |dF|/|F| <= 1e-12 and
max|d force| <= 1e-11 * max|force|, the FP64 bar of the specification; the
residual differences are FFT round-off (cuFFT vs pocketfft).
"""
import math

import numpy as np
import pytest

import classicaldft_b200 as cd
from oracle import fmt as ofmt
from tests.parity import Problem, force_err, rel_err, smooth_noise

pytestmark = pytest.mark.gpu

F_TOL = 1e-12
FORCE_TOL = 1e-11
MODELS = ["Rosenfeld", "RSLT", "WhiteBearI", "WhiteBearII", "esFMT"]
LJ = (1.0, 1.0, 2.5)


def profile(N, shape, seed, mean=0.5, amp=0.1):
    rng = np.random.default_rng(seed)
    return mean * (1.0 + amp * smooth_noise(shape, rng))


@pytest.mark.parametrize("model", MODELS)
def test_single_species_all_models(model):
    pr = Problem((16, 16, 16), 0.1, [1.0], model)
    rho = profile(pr.N, (16, 16, 16), 1)
    rng = np.random.default_rng(2)
    v = rng.standard_normal(pr.N)
    g = pr.gpu([rho], [0.7], [v])
    r = pr.ref([rho], [0.7], [v])
    assert rel_err(g.free_energy, r.free_energy) <= F_TOL
    assert rel_err(g.grand_potential, r.grand_potential) <= F_TOL
    assert rel_err(g.parts["hard_sphere"], r.parts["hard_sphere"]) <= F_TOL
    assert force_err(g.forces, r.forces) <= FORCE_TOL


@pytest.mark.parametrize("model", ["WhiteBearII", "RSLT"])
def test_mean_field_lj(model):
    pr = Problem((32, 32, 32), 0.2, [1.0], model, inters=[(0, 0) + LJ], kT=0.8)
    rho = profile(pr.N, (32, 32, 32), 3, 0.35, 0.2)
    g = pr.gpu([rho], [-2.0])
    r = pr.ref([rho], [-2.0])
    assert rel_err(g.parts["mean_field"], r.parts["mean_field"]) <= F_TOL
    assert rel_err(g.free_energy, r.free_energy) <= F_TOL
    assert force_err(g.forces, r.forces) <= FORCE_TOL
    assert pr.weights.a_vdw[0] == pytest.approx(pr.oweights.mean_field[0]["a_vdw"], rel=1e-13)


@pytest.mark.parametrize("model", ["Rosenfeld", "esFMT", "WhiteBearI"])
def test_binary_mixture_with_cross_interaction(model):
    inters = [(0, 0) + LJ, (0, 1, 1.0, 0.8, 2.5), (1, 1, 0.8, 0.5, 2.0)]
    pr = Problem((24, 20, 28), 0.2, [1.0, 0.5], model, A=1.0, B=0.0, inters=inters, kT=1.2)
    r1 = profile(pr.N, (24, 20, 28), 4, 0.3, 0.2)
    r2 = profile(pr.N, (24, 20, 28), 5, 0.2, 0.3)
    g = pr.gpu([r1, r2], [0.3, -0.4])
    r = pr.ref([r1, r2], [0.3, -0.4])
    assert rel_err(g.free_energy, r.free_energy) <= F_TOL
    assert rel_err(g.grand_potential, r.grand_potential) <= F_TOL
    assert force_err(g.forces, r.forces) <= FORCE_TOL


@pytest.mark.parametrize("shape", [(15, 17, 9), (16, 12, 10), (9, 16, 15), (8, 8, 2)])
def test_odd_and_ragged_grids(shape):
    pr = Problem(shape, 0.15, [1.0], "WhiteBearII", inters=[(0, 0, 0.5, 1.0, 0.9)])
    rho = profile(pr.N, shape, 6, 0.4, 0.2)
    g = pr.gpu([rho], [0.1])
    r = pr.ref([rho], [0.1])
    assert rel_err(g.free_energy, r.free_energy) <= F_TOL
    assert force_err(g.forces, r.forces) <= FORCE_TOL


@pytest.mark.parametrize("model", ["WhiteBearII", "esFMT"])
def test_nyquist_projection(model):
    """Density with weight on the Nyquist planes, where the odd vector and tensor
    weights are not Hermitian: the GPU must reproduce the c2r semantics."""
    shape = (16, 16, 16)
    pr = Problem(shape, 0.1, [1.0], model, A=1.0, B=-0.5)
    ix, iy, iz = np.meshgrid(*[np.arange(n) for n in shape], indexing="ij")
    rho = (0.4 + 0.04 * (-1.0) ** ix + 0.03 * (-1.0) ** (ix + iy) * np.cos(0.7 * iz) + 0.02 * (-1.0) ** iz
           * np.sin(2 * np.pi * iy / 16)).reshape(-1)
    g = pr.gpu([rho])
    r = pr.ref([rho])
    assert rel_err(g.free_energy, r.free_energy) <= F_TOL
    assert force_err(g.forces, r.forces) <= FORCE_TOL


def test_uniform_density_known_answers():
    """hard_sphere.cpp:52-163 on the GPU: F = phi_bulk V, force = (ln rho + mu_ex) dV."""
    pr = Problem((16, 16, 16), 0.1, [1.0], "WhiteBearII")
    rho = np.full(pr.N, 0.4)
    g = pr.gpu([rho])
    m = ofmt.FMTModel("WhiteBearII")
    vol = 1.6 ** 3
    assert g.parts["hard_sphere"] == pytest.approx(m.free_energy_density(0.4, 1.0) * vol, rel=1e-12)
    expect = (math.log(0.4) + m.excess_chemical_potential(0.4, 1.0)) * pr.grid.cell_volume
    assert np.max(np.abs(g.forces[0] - expect)) <= 1e-12 * abs(expect)


def test_zero_density_and_dilute_regions():
    pr = Problem((16, 16, 16), 0.1, [1.0], "RSLT")
    g = pr.gpu([np.zeros(pr.N)])
    r = pr.ref([np.zeros(pr.N)])
    assert g.free_energy == 0.0 and r.free_energy == 0.0
    assert force_err(g.forces, r.forces) <= FORCE_TOL
    # a cavity: eta below the 1e-30 skip threshold and the Taylor branches
    rho = profile(pr.N, (16, 16, 16), 8, 0.3, 0.2)
    rho[: pr.N // 3] = 1e-40
    rho[pr.N // 3: pr.N // 3 + 300] = 1e-7
    g = pr.gpu([rho])
    r = pr.ref([rho])
    assert rel_err(g.free_energy, r.free_energy) <= F_TOL
    assert force_err(g.forces, r.forces) <= FORCE_TOL


def test_64cubed_whitebear2_lj_matches_oracle():
    """The bench configuration family at 64^3 (WBII + cut LJ, QF weights)."""
    shape = (64, 64, 64)
    pr = Problem(shape, 0.1, [1.0], "WhiteBearII", inters=[(0, 0) + LJ], kT=1.0)
    rho = profile(pr.N, shape, 9, 0.5, 0.05)
    v = np.zeros(pr.N)
    v.reshape(shape)[:5] = 50.0
    g = pr.gpu([rho], [1.0], [v])
    r = pr.ref([rho], [1.0], [v])
    assert rel_err(g.free_energy, r.free_energy) <= F_TOL
    assert force_err(g.forces, r.forces) <= FORCE_TOL


def test_device_api_matches_host_api():
    import torch
    pr = Problem((32, 32, 32), 0.2, [1.0], "WhiteBearII", inters=[(0, 0) + LJ], kT=0.8)
    rho = profile(pr.N, (32, 32, 32), 10, 0.35, 0.1)
    host = pr.gpu([rho], [-1.0])
    d_rho = torch.tensor(rho, dtype=torch.float64, device="cuda")
    d_f = torch.empty_like(d_rho)
    d_sc = torch.empty(10, dtype=torch.float64, device="cuda")
    pr.weights.engine.total_device(d_rho.data_ptr(), None, [-1.0], d_f.data_ptr(), d_sc.data_ptr(),
                                   torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert float(d_sc[0]) == host.free_energy
    assert np.array_equal(d_f.cpu().numpy(), host.forces[0])


def test_repeat_evaluations_are_deterministic():
    pr = Problem((24, 24, 24), 0.1, [1.0], "esFMT")
    rho = profile(pr.N, (24, 24, 24), 11, 0.5, 0.1)
    a = pr.gpu([rho])
    b = pr.gpu([rho])
    assert a.free_energy == b.free_energy
    assert np.array_equal(a.forces[0], b.forces[0])


def test_bad_input_raises():
    pr = Problem((8, 8, 8), 0.2, [1.0], "Rosenfeld")
    with pytest.raises(ValueError):
        cd.total(pr.model, [np.zeros(10)], pr.weights)
    with pytest.raises(ValueError):
        cd.make_weights(cd.WhiteBearII(), cd.Model(pr.grid, [cd.Species("a", -1.0)], [], 1.0))


def test_tma_and_plain_pointwise_paths_agree():
    """The TMA-staged pointwise kernel (16-byte aligned inputs, N % 4 == 0) and the
    register-prefetch kernel (any alignment) give the same result."""
    import torch
    pr = Problem((32, 32, 32), 0.2, [1.0], "WhiteBearII", inters=[(0, 0) + LJ], kT=0.8)
    rho = profile(pr.N, (32, 32, 32), 12, 0.35, 0.1)
    buf = torch.zeros(pr.N + 1, dtype=torch.float64, device="cuda")
    buf[1:] = torch.tensor(rho, dtype=torch.float64)
    aligned = torch.tensor(rho, dtype=torch.float64, device="cuda")
    out = []
    for src in (aligned, buf[1:]):   # buf[1:] is 8-byte aligned only
        f = torch.empty(pr.N, dtype=torch.float64, device="cuda")
        sc = torch.empty(10, dtype=torch.float64, device="cuda")
        pr.weights.engine.total_device(src.data_ptr(), None, [0.3], f.data_ptr(), sc.data_ptr(), 0)
        torch.cuda.synchronize()
        out.append((sc.cpu().numpy(), f.cpu().numpy()))
    (s1, f1), (s2, f2) = out
    assert abs(s1[0] - s2[0]) <= 1e-13 * abs(s1[0])
    assert np.max(np.abs(f1 - f2)) <= 1e-13 * np.max(np.abs(f1))
    r = pr.ref([rho], [0.3])
    assert rel_err(s1[0], r.free_energy) <= F_TOL


@pytest.mark.parametrize("transforms", ["cufft", "fused"])
def test_stage_timing_hook_records_every_stage_and_changes_nothing(transforms):
    pr = Problem((32, 32, 32), 0.2, [1.0], "WhiteBearII", inters=[(0, 0) + LJ], kT=0.8, precision=cd.MIXED)
    rho = profile(pr.N, (32, 32, 32), 13, 0.35, 0.1)
    e = pr.weights.engine
    e.set_transforms(transforms)
    plain = pr.gpu([rho], [0.2])
    e.stage_timing(True)
    e.stage_times()
    timed = [pr.gpu([rho], [0.2]) for _ in range(70)]  # more than the 64-set event ring
    ms, n = e.stage_times()
    e.stage_timing(False)
    assert n == 70
    names = cd.Engine.STAGES if transforms == "cufft" else cd.Engine.STAGES_FUSED
    assert set(ms) == set(names)
    assert all(v >= 0.0 for v in ms.values())
    assert all(ms[k] > 0.0 for k in names[:8] if not k.startswith("-"))  # "-n": an empty slot
    for t in timed:
        assert t.free_energy == plain.free_energy
        assert np.array_equal(t.forces[0], plain.forces[0])
    assert e.stage_times()[1] == 0
