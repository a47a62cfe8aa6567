"""The fused transform path (hand-written plane / column FFT kernels with the
k-space stages in the column pass) against the FP64 oracle and against the
cuFFT path of the same engine.

Tolerances are those of the mixed-precision specification (both paths run
their transforms in FP32): near-uniform states |dF|/|F| <= 1e-9 and forces
1e-6 of their max; 10%-noise states |dF|/|F| <= 1e-6 and forces 1e-4.  On
top, the fused path's error may exceed the cuFFT path's by at most a factor
of 10 (same arithmetic precision; radix-4 stages and the R2C post-processing
round more often than cuFFT's kernels) unless it is below 5% of the
tolerance.
"""
import numpy as np
import pytest

import classicaldft_b200 as cd
from tests.parity import Problem, force_err, rel_err, smooth_noise

pytestmark = pytest.mark.gpu
LJ = (1.0, 1.0, 2.5)


def both_paths(pr, rhos, mus, vexts=None):
    e = pr.weights.engine
    assert e.transforms == "fused"
    fused = pr.gpu(rhos, mus, vexts)
    e.set_transforms("cufft")
    cufft = pr.gpu(rhos, mus, vexts)
    e.set_transforms("fused")
    return fused, cufft


def test_path_selection():
    g32 = Problem((32, 32, 32), 0.2, [1.0], "WhiteBearII", precision=cd.MIXED)
    assert g32.weights.engine.fused_available and g32.weights.engine.transforms == "fused"
    g64 = Problem((16, 16, 16), 0.2, [1.0], "WhiteBearII", precision=cd.FP64)
    assert not g64.weights.engine.fused_available and g64.weights.engine.transforms == "cufft"
    odd = Problem((24, 24, 24), 0.2, [1.0], "WhiteBearII", precision=cd.MIXED)  # no specialisation
    assert not odd.weights.engine.fused_available and odd.weights.engine.transforms == "cufft"
    with pytest.raises(ValueError):
        odd.weights.engine.set_transforms("fused")
    # rho planes, column pass, (channel planes, pointwise, derivative planes)
    # per chunk of x planes (four chunks from nx = 64), column pass, force planes
    assert g32.weights.engine.info["kernels_per_eval"] == 7
    g64m = Problem((64, 64, 64), 0.1, [1.0], "WhiteBearII", precision=cd.MIXED)
    assert g64m.weights.engine.info["kernels_per_eval"] == 16


CASES = [
    ((32, 32, 32), 0.2, [1.0], "WhiteBearII", [(0, 0) + LJ]),
    ((64, 64, 64), 0.1, [1.0], "RSLT", []),
    ((16, 32, 64), 0.2, [1.0], "WhiteBearI", [(0, 0) + LJ]),
    ((64, 16, 16), 0.2, [1.0], "Rosenfeld", [(0, 0) + LJ]),
    ((32, 16, 32), 0.2, [1.0, 0.6], "esFMT", [(0, 0) + LJ, (0, 1, 1.0, 0.8, 2.5), (1, 1, 0.8, 0.5, 2.0)]),
    ((16, 16, 32), 0.2, [1.0, 0.7], "Rosenfeld", [(0, 1, 1.0, 0.8, 2.5)]),
    ((48, 48, 48), 0.1, [1.0], "WhiteBearII", [(0, 0) + LJ]),
    ((96, 48, 96), 0.1, [1.0], "esFMT", [(0, 0) + LJ]),
    ((48, 96, 16), 0.2, [1.0, 0.6], "WhiteBearI", [(0, 1, 1.0, 0.8, 2.5)]),
    # the 128-point specialisations of every plane and column kernel
    ((128, 128, 128), 0.125, [1.0], "WhiteBearII", [(0, 0) + LJ]),
    ((128, 32, 64), 0.1, [1.0], "WhiteBearII", [(0, 0) + LJ]),
    ((32, 128, 16), 0.1, [1.0], "esFMT", [(0, 0) + LJ]),
    ((64, 64, 128), 0.1, [1.0, 0.6], "WhiteBearII", [(0, 0) + LJ, (0, 1, 1.0, 0.8, 2.5)]),
]


@pytest.mark.parametrize("shape,dx,diam,model,inters", CASES)
def test_fused_matches_oracle_and_cufft_path(shape, dx, diam, model, inters):
    pr = Problem(shape, dx, diam, model, A=1.0, B=0.1, inters=inters, kT=0.9, precision=cd.MIXED)
    rng = np.random.default_rng(sum(shape))
    S = len(diam)
    for amp, f_tol, force_tol in ((0.01, 1e-9, 1e-6), (0.1, 1e-6, 1e-4)):
        rhos = [0.3 / S * (1.0 + amp * smooth_noise(shape, rng)) for _ in range(S)]
        vexts = [0.2 * smooth_noise(shape, rng) for _ in range(S)]
        mus = list(rng.uniform(-1.0, 1.0, S))
        fused, cufft = both_paths(pr, rhos, mus, vexts)
        ref = pr.ref(rhos, mus, vexts)
        ef = rel_err(fused.free_energy, ref.free_energy)
        ec = rel_err(cufft.free_energy, ref.free_energy)
        assert ef <= f_tol
        assert rel_err(fused.grand_potential, ref.grand_potential) <= f_tol
        pf, pc = force_err(fused.forces, ref.forces), force_err(cufft.forces, ref.forces)
        assert pf <= force_tol
        assert pf <= max(10.0 * pc, 0.05 * force_tol)
        assert ef <= max(10.0 * ec, 0.05 * f_tol)


def test_fused_batch_and_unaligned_buffers():
    import torch
    shape = (32, 32, 32)
    pr = Problem(shape, 0.2, [1.0], "WhiteBearII", inters=[(0, 0) + LJ], kT=0.8, precision=cd.MIXED)
    rng = np.random.default_rng(11)
    B = 3
    rho = np.stack([0.35 * (1.0 + 0.05 * smooth_noise(shape, rng)) for _ in range(B)])
    mus = [0.1, -0.4, 0.9]
    wb = cd.make_weights(pr.fmt, pr.model, cd.MIXED, batch=B)
    assert wb.engine.transforms == "fused"
    res = cd.total_batch(pr.model, rho, wb, mus)
    for b in range(B):
        one = pr.gpu([rho[b]], [mus[b]])
        assert rel_err(res[b].free_energy, one.free_energy) <= 1e-13
        assert force_err(res[b].forces, one.forces) <= 1e-12
    # rho, vext and force only 8-byte aligned on the device API
    N = pr.N
    e = pr.weights.engine
    v = 0.3 * smooth_noise(shape, rng)
    buf = torch.zeros(3 * N + 3, dtype=torch.float64, device="cuda")
    buf[1:N + 1] = torch.tensor(rho[0])
    buf[N + 2:2 * N + 2] = torch.tensor(v)
    sc = torch.empty(10, dtype=torch.float64, device="cuda")
    e.total_device(buf[1:].data_ptr(), buf[N + 2:].data_ptr(), [mus[0]], buf[2 * N + 3:].data_ptr(), sc.data_ptr(),
                   0)
    torch.cuda.synchronize()
    ref = pr.gpu([rho[0]], [mus[0]], [v])
    assert rel_err(float(sc[0]), ref.free_energy) <= 1e-13
    # misaligned rho / vext take the register-prefetch pointwise kernel
    # instead of the TMA ring: the same FP64 formulas, but the compiler may
    # contract them into FMAs differently, and a last-bit difference in a
    # derivative can flip the FP32 rounding of its deviation from the mean
    # (one FP32 ulp of a 5% deviation: ~3e-9 of the force scale)
    assert force_err([buf[2 * N + 3:].cpu().numpy()], ref.forces) <= 1e-8


def test_plane_chunks():
    """The middle stages in 1, 2, 4 or 8 chunks of x planes on forked
    streams: forces bitwise equal (each point is computed the same way),
    scalars up to summation order; invalid counts are rejected."""
    shape = (64, 32, 32)
    pr = Problem(shape, 0.1, [1.0], "WhiteBearII", inters=[(0, 0) + LJ], kT=0.8, precision=cd.MIXED)
    rng = np.random.default_rng(5)
    rho = 0.35 * (1.0 + 0.05 * smooth_noise(shape, rng))
    e = pr.weights.engine
    assert e.info["kernels_per_eval"] == 16
    ref = pr.gpu([rho], [0.2])
    for k in (1, 2, 8, 4):
        e.set_plane_chunks(k)
        assert e.info["kernels_per_eval"] == 4 + 3 * k
        r = pr.gpu([rho], [0.2])
        assert np.array_equal(r.forces[0], ref.forces[0]), k
        assert rel_err(r.free_energy, ref.free_energy) <= 1e-13
    for bad in (0, 3, 16):
        with pytest.raises(ValueError):
            e.set_plane_chunks(bad)
    cu = Problem((24, 24, 24), 0.2, [1.0], "WhiteBearII", precision=cd.MIXED)
    with pytest.raises(ValueError):
        cu.weights.engine.set_plane_chunks(2)



def test_autotune():
    """The autotuner times every plane-chunk count on a device state, keeps
    the fastest (forces unchanged), and later engines of the same shape start
    from its choice."""
    import torch
    shape = (64, 32, 32)
    pr = Problem(shape, 0.1, [1.0], "WhiteBearII", inters=[(0, 0) + LJ], kT=0.8, precision=cd.MIXED)
    rng = np.random.default_rng(6)
    rho = 0.35 * (1.0 + 0.05 * smooth_noise(shape, rng))
    e = pr.weights.engine
    before = pr.gpu([rho], [0.2])
    rd = torch.tensor(rho.ravel(), device="cuda")
    k, ms = e.autotune(rd.data_ptr(), mu=[0.2], reps=3)
    assert sorted(ms) == [1, 2, 4, 8] and all(v > 0.0 for v in ms.values())
    assert k == min(ms, key=ms.get)
    assert e.info["kernels_per_eval"] == 4 + 3 * k
    after = pr.gpu([rho], [0.2])
    assert np.array_equal(after.forces[0], before.forces[0])
    assert rel_err(after.free_energy, before.free_energy) <= 1e-13
    again = cd.make_weights(pr.fmt, pr.model, cd.MIXED)
    assert again.engine.info["kernels_per_eval"] == 4 + 3 * k
    # an engine without the fused path keeps one chunk; with one species it
    # still times its pointwise variants (the table holds the one count)
    cu = Problem((24, 24, 24), 0.2, [1.0], "WhiteBearII", precision=cd.MIXED)
    r24 = torch.full((24 ** 3,), 0.3, dtype=torch.float64, device="cuda")
    k24, ms24 = cu.weights.engine.autotune(r24.data_ptr())
    assert k24 == 1 and sorted(ms24) == [1]
    assert cu.weights.engine.column_tile == 0
    # two species without the fused path: nothing to tune
    cu2 = Problem((24, 24, 24), 0.2, [1.0, 0.6], "WhiteBearII", precision=cd.MIXED)
    r2 = torch.full((2 * 24 ** 3,), 0.2, dtype=torch.float64, device="cuda")
    k2, ms2 = cu2.weights.engine.autotune(r2.data_ptr())
    assert k2 == 1 and ms2 == {}


def test_column_tile_widths_and_autotune_table():
    """Two species: the column passes in tiles of 16 or 32 columns give the
    same forces bitwise (each column is transformed alone); the autotuner's
    table covers both widths and every chunk count and its choice is kept."""
    import torch
    shape = (64, 32, 32)
    inters = [(0, 0) + LJ, (0, 1, 1.0, 0.8, 2.5)]
    pr = Problem(shape, 0.1, [1.0, 0.6], "WhiteBearII", inters=inters, kT=0.9, precision=cd.MIXED)
    rng = np.random.default_rng(8)
    rhos = [0.3 * (1.0 + 0.05 * smooth_noise(shape, rng)), 0.1 * (1.0 + 0.05 * smooth_noise(shape, rng))]
    e = pr.weights.engine
    assert e.column_tile == 32
    base = pr.gpu(rhos, [0.2, -0.1])
    e.set_column_tile(16)
    assert e.column_tile == 16
    r16 = pr.gpu(rhos, [0.2, -0.1])
    for s in range(2):
        assert np.array_equal(r16.forces[s], base.forces[s]), s
    assert rel_err(r16.free_energy, base.free_energy) <= 1e-13
    for bad in (0, 8, 64):
        with pytest.raises(ValueError):
            e.set_column_tile(bad)
    rd = torch.tensor(np.concatenate([r.ravel() for r in rhos]), device="cuda")
    (k, v, tq, sp), ms = e.autotune_ex(rd.data_ptr(), mu=[0.2, -0.1], reps=2)
    assert v == 0 and tq in (16, 32)
    assert sorted(ms) == sorted((t, 0, c, d) for t in (16, 32) for c in (1, 2, 4, 8) for d in (1, 2, 4, 8) if d <= c)
    assert (tq, v, k, sp) == min(ms, key=ms.get)
    assert e.pointwise_spread == sp
    assert e.column_tile == tq and e.info["kernels_per_eval"] == 4 + 3 * k
    after = pr.gpu(rhos, [0.2, -0.1])
    for s in range(2):
        assert np.array_equal(after.forces[s], base.forces[s]), s


@pytest.mark.parametrize("shape,diams", [((64, 32, 32), [1.0, 0.6]), ((128, 32, 64), [1.0]),
                                         ((32, 128, 128), [1.0]), ((48, 96, 48), [1.0])])
def test_middle_plane_widths(shape, diams):
    """The middle plane passes at the base width and at twice the threads
    per plane CTA compute every sample the same way: forces and F bitwise
    equal.  The autotuner keeps one of the two; an engine without the fused
    path has none."""
    import torch
    S = len(diams)
    inters = [(0, 0) + LJ] + ([(0, 1, 1.0, 0.8, 2.5)] if S > 1 else [])
    pr = Problem(shape, 0.1, diams, "WhiteBearII", inters=inters, kT=0.9, precision=cd.MIXED)
    rng = np.random.default_rng(10)
    rhos = [0.3 / (s + 1) * (1.0 + 0.05 * smooth_noise(shape, rng)) for s in range(S)]
    mu = [0.2, -0.1][:S]
    e = pr.weights.engine
    e.set_plane_width(0)
    assert e.plane_width == 0
    base = pr.gpu(rhos, mu)
    e.set_plane_width(1)
    assert e.plane_width == 1
    wide = pr.gpu(rhos, mu)
    for s in range(S):
        assert np.array_equal(wide.forces[s], base.forces[s]), s
    assert wide.free_energy == base.free_energy
    assert rel_err(base.free_energy, pr.ref(rhos, mu).free_energy) <= 1e-9
    with pytest.raises(ValueError):
        e.set_plane_width(2)
    rd = torch.tensor(np.concatenate([r.ravel() for r in rhos]), device="cuda")
    e.autotune_ex(rd.data_ptr(), mu=mu, reps=1)
    assert e.plane_width in (0, 1)
    cu = Problem((24, 24, 24), 0.2, [1.0], "WhiteBearII", precision=cd.MIXED)
    assert cu.weights.engine.plane_width == -1
    with pytest.raises(ValueError):
        cu.weights.engine.set_plane_width(1)


def test_pointwise_spread():
    """Each plane chunk's pointwise launch may take 1/8 .. all of the
    pointwise grid: forces bitwise equal (each point is computed the same
    way), F up to the summation order of the block partials."""
    shape = (64, 32, 32)
    pr = Problem(shape, 0.1, [1.0], "WhiteBearII", inters=[(0, 0) + LJ], kT=0.8, precision=cd.MIXED)
    rng = np.random.default_rng(9)
    rho = 0.35 * (1.0 + 0.05 * smooth_noise(shape, rng))
    e = pr.weights.engine
    e.set_plane_chunks(8)
    e.set_pointwise_spread(0)  # (an earlier autotune of this shape may have set another)
    assert e.pointwise_spread == 0
    ref = pr.gpu([rho], [0.2])
    for v in e.pointwise_variants:
        e.set_pointwise(v)
        base = pr.gpu([rho], [0.2])
        for d in (1, 2, 4, 8, 0):
            e.set_pointwise_spread(d)
            assert e.pointwise_spread == d
            r = pr.gpu([rho], [0.2])
            assert np.array_equal(r.forces[0], base.forces[0]), (v, d)
            assert rel_err(r.free_energy, ref.free_energy) <= 1e-13
    for bad in (-1, 3, 16):
        with pytest.raises(ValueError):
            e.set_pointwise_spread(bad)
