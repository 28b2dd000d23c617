"""Discretize and the potential-link searches on the GPU against the host
path, bit for bit (offsets, every vertex coordinate, the pairs and the round
count), and the same errors on the reference's failure conditions. The host
path is itself pinned to the oracle (test_host_stages.py)."""
import numpy as np
import pytest

from conftest import FIXTURES, golden_bcc
from fastlinkingnumbers_b200 import Engine, FlnError, Model, workloads

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def engine():
    return Engine(0)


def _same(make, engine):
    host = make().Prepare(True)
    dev = make().Prepare(True, engine=engine)
    off, xyz, pairs, rounds = host
    doff, dxyz, dpairs, drounds = dev
    assert drounds == rounds
    assert np.array_equal(doff, off)
    assert np.array_equal(dxyz.view(np.uint64), xyz.view(np.uint64))  # bitwise
    assert np.array_equal(dpairs, pairs)
    return host


@pytest.mark.parametrize("name", FIXTURES)
def test_golden_inputs(engine, name, golden_dir):
    path = golden_bcc(name, golden_dir)
    _same(lambda: Model().ImportFromFile(path), engine)


@pytest.mark.parametrize("seg_type", [0, 1, 2, 3])
def test_spline_kinds(engine, seg_type):
    off, xyz = workloads.ring_chain(seed=7, n_rings=12, as_bezier=True)
    counts = -np.diff(off).astype(np.int32)
    _same(lambda: Model().SetCurves(seg_type, counts, xyz), engine)


def test_chain_mail(engine):
    off, xyz = workloads.chain_mail(rows=30, cols=30)
    counts = -np.diff(off).astype(np.int32)
    _same(lambda: Model().SetCurves(3, counts, xyz), engine)


def test_chain_mail_full_sheet(engine):
    # 10,000 rings: the device join of the loop boxes runs over 40 tiles of
    # 256 curves, with ring boxes that overlap their 8 neighbours.
    off, xyz = workloads.chain_mail()
    counts = -np.diff(off).astype(np.int32)
    _, _, pairs, _ = _same(lambda: Model().SetCurves(3, counts, xyz), engine)
    assert len(pairs) > 30_000


def test_polymer(engine):
    off, xyz = workloads.polymer(seed=41, n_loops=40, n_steps=20_000, cube=300.0)
    counts = -np.diff(off).astype(np.int32)
    poff, _, pairs, rounds = _same(lambda: Model().SetCurves(3, counts, xyz), engine)
    assert rounds > 5 and poff[-1] > off[-1] and len(pairs) > 100


def test_mixed_sizes(engine):
    off, xyz = workloads.mixed_batch(seed=9, n_loops=300, hi=2 ** 14)
    counts = -np.diff(off).astype(np.int32)
    _same(lambda: Model().SetCurves(3, counts, xyz), engine)


def test_open_curves_and_isolated_curves(engine):
    # An open curve without pairs keeps its end point; a far-away curve has
    # no pairs and is not refined.
    off, xyz = workloads.ring_chain(seed=4, n_rings=4)
    far = xyz[off[0]:off[1]] + 1000.0
    xyz2 = np.concatenate([xyz, far, far[:5] + 500.0])
    counts = np.concatenate([-np.diff(off), [-(off[1] - off[0]), 5]]).astype(np.int32)
    _same(lambda: Model().SetCurves(3, counts, xyz2), engine)


def test_touching_curves_fail_like_host(engine):
    t = 2 * np.pi * np.arange(16) / 16
    a = np.stack([np.cos(t), np.sin(t), 0 * t], axis=1)
    b = np.stack([2 + np.cos(t + np.pi), 0 * t, np.sin(t + np.pi)], axis=1)
    xyz = np.concatenate([a, b]).astype(np.float32).astype(np.float64)
    counts = np.array([-16, -16], dtype=np.int32)
    with pytest.raises(FlnError) as h:
        Model().SetCurves(3, counts, xyz).Prepare(True)
    with pytest.raises(FlnError) as d:
        Model().SetCurves(3, counts, xyz).Prepare(True, engine=engine)
    assert d.value.status == h.value.status


def test_open_curve_in_pair_is_an_error(engine):
    off, xyz = workloads.ring_chain(seed=1, n_rings=2)
    counts = np.array([len(xyz) // 2, -(len(xyz) // 2)], dtype=np.int32)
    with pytest.raises(FlnError) as e:
        Model().SetCurves(3, counts, xyz).Prepare(True, engine=engine)
    assert e.value.status == 9  # FLN_ERR_UNLOOPED


def test_float32_upload_of_bcc_points(engine, tmp_path):
    # A model loaded from a BCC file keeps its float32 points and the GPU
    # prepare uploads those (12 bytes per point) and widens them on the
    # device; the same curves given as doubles take the FP64 upload. Same
    # output bit for bit.
    off, xyz = workloads.polymer(seed=43, n_loops=30, n_steps=20_000, cube=260.0)
    path = str(tmp_path / "p.bcc")
    workloads.write_bcc(path, (off, xyz))
    a = Model().ImportFromFile(path).Prepare(True, engine=engine)
    b = Model().SetCurves(3, -np.diff(off).astype(np.int32), xyz).Prepare(True, engine=engine)
    assert a[3] == b[3]
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[2], b[2])
    assert np.array_equal(a[1].view(np.uint64), b[1].view(np.uint64))
