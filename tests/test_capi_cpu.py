"""CPU-side checks of the C ABI: the library loads, exports every declared
symbol, and its host set-up physics matches the oracle.  No GPU needed."""
import ctypes
import math

import numpy as np
import pytest

import classicaldft_b200 as cd
from classicaldft_b200 import _lib
from oracle import potentials as op
from oracle.functional import Model as OModel
from oracle.functional import Species as OSpecies
from oracle.grid import Grid as OGrid


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    names = _lib.declared_symbols()
    assert len(names) >= 13
    for n in names:
        assert hasattr(L, n), n
    assert b"sm_100a" in L.cdft_version()


def test_potential_factories_match_oracle():
    for (sig, eps, rc) in ((1.0, 1.0, 2.5), (1.0, 1.0, 3.0), (0.5, 1.0, 0.75), (1.0, 2.0, -1.0)):
        ours = cd.make_lennard_jones(sig, eps, rc).info()
        ref = op.make_lennard_jones(sig, eps, rc)
        for k in ("epsilon_shift", "r_min", "v_min", "r_zero"):
            assert ours[k] == pytest.approx(getattr(ref, k), rel=1e-15, abs=1e-15)
    t = cd.make_ten_wolde_frenkel(1.0, 1.0, 2.0, 50.0).info()
    tr = op.make_ten_wolde_frenkel(1.0, 1.0, 2.0, 50.0)
    assert t["r_min"] == pytest.approx(tr.r_min) and t["v_min"] == pytest.approx(tr.v_min)
    w = cd.make_wang_ramirez_dobnikar_frenkel(1.0, 1.0, 3.0).info()
    wr = op.make_wang_ramirez_dobnikar_frenkel(1.0, 1.0, 3.0)
    assert w["r_min"] == pytest.approx(wr.r_min) and w["v_min"] == pytest.approx(wr.v_min)


def test_attractive_tail_matches_oracle():
    r = np.linspace(0.05, 3.2, 400)
    for split, osplit in ((cd.WEEKS_CHANDLER_ANDERSEN, op.WCA), (cd.BARKER_HENDERSON, op.BH)):
        ours = cd.make_lennard_jones(1.0, 1.0, 2.5).attractive(r, split)
        ref = op.make_lennard_jones(1.0, 1.0, 2.5).attractive(r, osplit)
        assert np.allclose(ours, ref, rtol=1e-15, atol=1e-15)


def test_hard_sphere_diameter_and_vdw_integral_match_quadpack():
    for kT in (0.7, 0.8, 1.0, 1.5):
        for split, osplit in ((cd.WEEKS_CHANDLER_ANDERSEN, op.WCA), (cd.BARKER_HENDERSON, op.BH)):
            p = cd.make_lennard_jones(1.0, 1.0, 2.5)
            q = op.make_lennard_jones(1.0, 1.0, 2.5)
            assert p.hard_sphere_diameter(kT, split) == pytest.approx(op.hard_sphere_diameter(q, kT, osplit),
                                                                      rel=1e-9)
            assert p.vdw_integral(kT, split) == pytest.approx(op.vdw_integral(q, kT, osplit), rel=1e-9)


@pytest.mark.parametrize("scheme", ["InterpolationZero", "InterpolationLinearF", "InterpolationQuadraticF", "GaussE"])
def test_interaction_weight_matches_oracle(scheme):
    g = cd.make_grid(0.2, (3.2, 3.6, 4.0))
    inter = cd.Interaction(0, 0, cd.make_lennard_jones(1.0, 1.0, 2.5), cd.WEEKS_CHANDLER_ANDERSEN, scheme)
    w, a = cd.interaction_weight(inter, g, 0.8)
    og = OGrid(dx=0.2, box_size=(3.2, 3.6, 4.0), shape=g.shape)
    oi = op.Interaction(0, 0, op.make_lennard_jones(1.0, 1.0, 2.5), op.WCA, scheme)
    wr, ar = op.interaction_weight_real(oi, og, 0.8)
    assert a == pytest.approx(ar, rel=1e-13)
    assert np.max(np.abs(w - wr.reshape(-1))) <= 1e-15 * np.max(np.abs(wr))


def test_invalid_arguments_raise_value_error():
    with pytest.raises(ValueError):
        cd.make_grid(0.0, (1.0, 1.0, 1.0))
    with pytest.raises(ValueError):
        cd.make_grid(0.3, (1.0, 1.0, 1.0))
    with pytest.raises(ValueError):
        cd.FMTModel("Unknown")
    with pytest.raises(ValueError):
        cd.make_lennard_jones(1.0, 1.0, 2.5).hard_sphere_diameter(-1.0)


def test_engine_creation_fails_loudly_without_a_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    g = cd.make_grid(0.1, (1.6, 1.6, 1.6))
    model = cd.Model(g, [cd.Species("A", 1.0)], [], 1.0)
    with pytest.raises(cd.EngineError) as exc:
        cd.make_weights(cd.WhiteBearII(), model)
    assert exc.value.code in (_lib.CDFT_ERR_CUDA, _lib.CDFT_ERR_RUNTIME)


def test_batched_engine_size_is_validated_before_any_device_call():
    import ctypes
    L = _lib.lib()
    d = (ctypes.c_double * 1)(1.0)
    for bad in (0, 65):
        h = ctypes.c_void_p()
        st = L.cdft_create_batch(ctypes.byref(h), _lib.c_long3(8, 8, 8), 0.1, 1, d, 3, 1.0, 0.0, 0, None, 0, bad)
        assert st == _lib.CDFT_ERR_INVALID
        assert b"batch" in L.cdft_last_error()
        assert not h.value
