"""Host stages of the product (BCC load, potential-link search, Discretize)
against the oracle, bit for bit: the discretized polylines and the potential
pairs that feed the kernels must be identical (src/discretize.cpp:103-281,
src/potential_link_search.cpp:88-165). No GPU needed."""
import numpy as np
import pytest

from conftest import FIXTURES, golden_bcc
from fastlinkingnumbers_b200 import FlnError, Model, workloads
from oracle import pyoracle


def _compare(model, orc):
    off, xyz, pairs, rounds = model.Prepare(True)
    orc.prepare(True)
    ooff, oxyz = orc.polylines()
    assert rounds == orc.rounds
    assert np.array_equal(off, ooff)
    assert np.array_equal(xyz, oxyz)  # bitwise: same boxes, same refinement
    assert np.array_equal(pairs, orc.pairs())


@pytest.mark.parametrize("name", FIXTURES)
def test_prepare_matches_oracle(name, golden_dir):
    path = golden_bcc(name, golden_dir)
    _compare(Model().ImportFromFile(path), pyoracle.Oracle().load_bcc(path))


@pytest.mark.parametrize("seg_type", [0, 1, 2, 3])
def test_prepare_spline_kinds(seg_type):
    # Ring-chain control points read as B-spline, Catmull-Rom, Bezier (the
    # reference's sliding 4-point windows, curve.cpp:167-182) and polyline.
    off, xyz = workloads.ring_chain(seed=7, n_rings=12, as_bezier=True)
    counts = -np.diff(off).astype(np.int32)
    m = Model().SetCurves(seg_type, counts, xyz)
    o = pyoracle.Oracle().set_curves(seg_type, counts, xyz)
    _compare(m, o)


def test_prepare_chain_mail_small():
    off, xyz = workloads.chain_mail(rows=8, cols=8)
    counts = -np.diff(off).astype(np.int32)
    _compare(Model().SetCurves(3, counts, xyz), pyoracle.Oracle().set_curves(3, counts, xyz))


def test_no_discretize_keeps_polylines():
    off, xyz = workloads.ring_chain(seed=3, n_rings=6)
    m = Model().SetCurves(3, -np.diff(off).astype(np.int32), xyz)
    poff, pxyz, pairs, rounds = m.Prepare(False)
    assert rounds == 0 and np.array_equal(poff, off) and np.array_equal(pxyz, xyz)
    assert [tuple(p) for p in pairs] == [(i, i + 1) for i in range(5)]


def test_touching_curves_fail_like_reference():
    # Two rings sharing the vertex (1, 0, 0): the pieces at the contact keep
    # overlapping until they are smaller than eps * avg coordinate or 55
    # rounds pass; both implementations refuse (discretize.cpp:219-229, :248-253).
    t = 2 * np.pi * np.arange(16) / 16
    a = np.stack([np.cos(t), np.sin(t), 0 * t], axis=1)
    b = np.stack([2 + np.cos(t + np.pi), 0 * t, np.sin(t + np.pi)], axis=1)
    xyz = np.concatenate([a, b]).astype(np.float32).astype(np.float64)
    counts = np.array([-16, -16], dtype=np.int32)
    with pytest.raises(FlnError) as e:
        Model().SetCurves(3, counts, xyz).Prepare(True)
    assert e.value.status in (7, 8)
    with pytest.raises(pyoracle.OracleError):
        pyoracle.Oracle().set_curves(3, counts, xyz).prepare(True)


def test_open_curve_in_pair_is_an_error():
    off, xyz = workloads.ring_chain(seed=1, n_rings=2)
    counts = np.array([len(xyz) // 2, -(len(xyz) // 2)], dtype=np.int32)  # first curve open
    m = Model().SetCurves(3, counts, xyz)
    with pytest.raises(FlnError) as e:
        m.Prepare(True)
    assert e.value.status == 9  # FLN_ERR_UNLOOPED


def test_bcc_roundtrip_and_errors(tmp_path):
    off, xyz = workloads.ring_chain(seed=2, n_rings=3)
    p = str(tmp_path / "r.bcc")
    workloads.write_bcc(p, (off, xyz))
    m = Model().ImportFromFile(p)
    t, counts, got = m.GetCurves()
    assert t == 3 and list(counts) == list(-np.diff(off)) and np.array_equal(got, xyz)
    q = str(tmp_path / "s.bcc")
    m.ExportToFile(q)
    assert open(p, "rb").read()[64:] == open(q, "rb").read()[64:]
    bad = tmp_path / "bad.bcc"
    bad.write_bytes(b"XYZ" + open(p, "rb").read()[3:])
    with pytest.raises(FlnError) as e:
        Model().ImportFromFile(str(bad))
    assert e.value.status == 3
    short = tmp_path / "short.bcc"
    short.write_bytes(open(p, "rb").read()[:100])
    with pytest.raises(FlnError) as e:
        Model().ImportFromFile(str(short))
    assert e.value.status in (2, 3)
    with pytest.raises(FlnError):
        Model().ImportFromFile(str(tmp_path / "missing.bcc"))
    with pytest.raises(FlnError):
        Model().ImportFromFile(str(tmp_path / "x.obj"))
