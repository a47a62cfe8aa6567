"""Every one-species pointwise kernel variant (cdft_engine_set_pointwise 1 ..
5) for every FMT model, against the oracle (hard_sphere.hpp:174-224,
models.hpp:153-359) on a 32^3 fused engine with one cut-LJ interaction.

The state mixes a liquid slab (rho ~ 0.6) with near vacuum (rho ~ 1e-9,
eta < 1e-6): warps of the liquid take the branch-free path of variants
3 - 5, warps of the vacuum the Taylor branches of f1 - f3, and warps through
a vacuum bubble in the liquid hold both kinds of point (such a warp runs the
exact path throughout).
Bars: against the oracle F and Omega to 1e-7 and forces to 1e-6 of their
largest value (the mean split's FP32 round-off scales with the density swing
inside a plane, here liquid against vacuum: |dF|/|F| ~ 3e-9 for every
variant, the generic kernel included); against the generic kernel (variant
0), which isolates the variants' own arithmetic, forces to 1e-8 and F to
1e-13 (the variants differ only in FP64 rounding)."""
import numpy as np
import pytest

import classicaldft_b200 as cd
from tests.parity import Problem, force_err, rel_err, smooth_noise

pytestmark = pytest.mark.gpu
LJ = (1.0, 1.0, 2.5)


def _slab_state(shape, rng):
    """Liquid for y in [ny/4, 3ny/4) (sharp tanh edges) around a vacuum
    bubble of radius 7 cells, near vacuum elsewhere.  A warp covers 32
    consecutive z of one (x, y) row: rows outside the slab are vacuum, rows
    inside it liquid, and rows through the bubble part liquid, part vacuum
    (eta, the density smeared over a sphere of 2.5 cells, below 1e-6 deep in
    the vacuum and the bubble)."""
    nx, ny, nz = shape
    x, y, z = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    liquid = 0.6 * (1.0 + 0.05 * smooth_noise(shape, rng).reshape(shape))
    vacuum = 1e-9 * (1.0 + 0.05 * smooth_noise(shape, rng).reshape(shape))
    w = 0.5
    slab = 0.5 * (np.tanh((y - ny / 4) / w) - np.tanh((y - 3 * ny / 4) / w))
    r = np.sqrt((x - nx / 2) ** 2 + (y - ny / 2) ** 2 + (z - nz / 2) ** 2)
    s = slab * 0.5 * (1.0 + np.tanh((r - 7.0) / w))
    return (vacuum + s * (liquid - vacuum)).ravel()


@pytest.mark.parametrize("model", ["Rosenfeld", "RSLT", "WhiteBearI", "WhiteBearII", "esFMT"])
def test_every_pointwise_variant_every_model(model):
    shape = (32, 32, 32)
    pr = Problem(shape, 0.2, [1.0], model, A=1.0, B=0.1, inters=[(0, 0) + LJ], kT=0.9, precision=cd.MIXED)
    e = pr.weights.engine
    assert e.transforms == "fused"
    assert e.pointwise_variants == list(range(cd.functionals.POINTWISE_VARIANTS))
    rng = np.random.default_rng(31)
    rho = _slab_state(shape, rng)
    mu = [0.4]
    ref = pr.ref([rho], mu)
    base = None
    for v in e.pointwise_variants:
        e.set_pointwise(v)
        got = pr.gpu([rho], mu)
        print(f"{model} variant {v}: |dF/F| {rel_err(got.free_energy, ref.free_energy):.2e}, "
              f"force {force_err(got.forces, ref.forces):.2e}")
        assert rel_err(got.free_energy, ref.free_energy) <= 1e-7, (model, v)
        assert rel_err(got.grand_potential, ref.grand_potential) <= 1e-7, (model, v)
        assert force_err(got.forces, ref.forces) <= 1e-6, (model, v)
        if base is None:
            base = got
        else:
            assert force_err(got.forces, base.forces) <= 1e-8, (model, v)
            assert rel_err(got.free_energy, base.free_energy) <= 1e-13, (model, v)
    e.set_pointwise(1)
