"""Crystal lattices (library host code through the C ABI) against the
reference's unit tests (tests/unit/types.cpp:161-300) and the oracle's
restatement of src/crystal.cpp (bit-exact positions and dimensions, equal
export files)."""
import numpy as np
import pytest

from classicaldft_b200 import crystal as cc
from oracle import crystal as oc

S, O, F = cc.Structure, cc.Orientation, cc.ExportFormat
VALID = [(s, o) for s in S for o in O if not (s == S.HCP and o >= O._110)]
PER_CELL = {(S.BCC, 0): 2, (S.BCC, 1): 4, (S.BCC, 2): 12, (S.FCC, 0): 4, (S.FCC, 1): 2, (S.FCC, 2): 6,
            (S.HCP, 0): 4}


def family(o):
    return 0 if o <= O._100 else (1 if o <= O._011 else 2)


def min_distance(p):
    d = np.sqrt(np.sum((p[:, None, :] - p[None, :, :]) ** 2, axis=-1))
    return float(np.min(d[np.triu_indices(len(p), 1)]))


@pytest.mark.parametrize("s,o", VALID)
def test_lattice_matches_oracle_bit_exact(s, o):
    lat = cc.build_lattice(s, o, (2, 3, 2))
    po, do = oc.build_lattice(int(s), int(o), (2, 3, 2))
    assert lat.positions.shape == (PER_CELL[(s, family(o))] * 12, 3)
    assert np.array_equal(lat.positions, po)
    assert np.array_equal(lat.dimensions, do)
    assert lat.shape == [2, 3, 2]
    # every structure and orientation has unit nearest-neighbour distance
    assert min_distance(lat.positions) == pytest.approx(1.0, abs=1e-10)
    # all sites inside the box
    assert np.all(lat.positions >= -1e-12) and np.all(lat.positions < lat.dimensions + 1e-12)


def test_reference_unit_cases():
    """types.cpp:163-300."""
    b = cc.build_lattice(S.BCC, O._001)
    assert b.positions.shape == (2, 3) and b.shape == [1, 1, 1]
    assert cc.build_lattice(S.FCC, O._001).positions.shape[0] == 4
    assert cc.build_lattice(S.HCP, O._001).positions.shape[0] == 4
    assert cc.build_lattice(S.BCC, O._001, (2, 2, 2)).positions.shape[0] == 16
    assert min_distance(cc.build_lattice(S.BCC, O._001, (3, 3, 3)).positions) == pytest.approx(1.0, abs=1e-10)
    assert min_distance(cc.build_lattice(S.FCC, O._001, (3, 3, 3)).positions) == pytest.approx(1.0, abs=1e-10)
    one = cc.build_lattice(S.BCC, O._001, (1, 1, 1))
    big = cc.build_lattice(S.BCC, O._001, (2, 3, 4))
    assert np.allclose(big.dimensions, one.dimensions * np.array([2, 3, 4]), rtol=1e-15)
    with pytest.raises(ValueError):
        cc.build_lattice(S.BCC, O._001, (1, 1))
    with pytest.raises(ValueError, match="strictly positive"):
        cc.build_lattice(S.BCC, O._001, (0, 1, 1))
    for o in (O._110, O._111):
        with pytest.raises(ValueError, match="HCP"):
            cc.build_lattice(S.HCP, o)
    sc = b.scaled_positions(2.5)
    assert sc[0, 0] == b.positions[0, 0] * 2.5 and sc[1, 2] == b.positions[1, 2] * 2.5
    f = cc.build_lattice(S.FCC, O._001, (2, 2, 2))
    box = f.scaled_positions([10.0, 20.0, 30.0])
    assert box[:, 0].max() < 10.0 + 1e-10 and box[:, 1].max() < 20.0 + 1e-10 and box[:, 2].max() < 30.0 + 1e-10
    for o in (O._010, O._100):
        assert cc.build_lattice(S.BCC, o).positions.shape[0] == 2
    for o in (O._110, O._101, O._011):
        assert cc.build_lattice(S.BCC, o).positions.shape[0] == 4
    assert cc.build_lattice(S.BCC, O._111).positions.shape[0] == 12


@pytest.mark.parametrize("fmt", [F.XYZ, F.CSV])
@pytest.mark.parametrize("s,o", [(S.BCC, O._001), (S.FCC, O._111), (S.HCP, O._010), (S.HCP, O._100)])
def test_export_matches_oracle(tmp_path, fmt, s, o):
    lat = cc.build_lattice(s, o, (2, 2, 1))
    path = tmp_path / f"lat.{fmt.name.lower()}"
    lat.export_to(path, fmt)
    text = path.read_text()
    assert text == oc.export_text(lat.positions, int(fmt))
    first = text.splitlines()[0]
    if fmt == F.XYZ:
        assert int(first) == lat.positions.shape[0]
    else:
        assert first == "x,y,z"


def test_export_to_unwritable_path_raises(tmp_path):
    lat = cc.build_lattice(S.BCC, O._001)
    from classicaldft_b200._lib import EngineError
    with pytest.raises(EngineError, match="Cannot open"):
        lat.export_to(tmp_path / "missing" / "dir" / "x.xyz")
