"""Pins the CPU oracle against the reference's own golden vectors: the five
regression certificates (results/reference_certificates/*.txt, test.sh) under
both --method values, the README answers, and the published mean off-integer
errors of the default Barnes–Hut run (test.sh:4,14,24,34,45)."""
import json
import os

import numpy as np
import pytest

from conftest import FIXTURES, GOLDEN, golden_bcc, golden_certificate
from oracle import pyoracle


@pytest.mark.parametrize("name", FIXTURES)
def test_oracle_barneshut_matches_golden(name, golden_dir):
    o = pyoracle.Oracle().load_bcc(golden_bcc(name, golden_dir))
    text, mean_off, _ = o.certificate(direct=False)
    assert text == golden_certificate(name)
    published = json.load(open(os.path.join(GOLDEN, "manifest.json")))["published_mean_off_integer_bh"]
    # test.sh prints 6 significant digits.
    assert mean_off == pytest.approx(published[name], rel=1e-5)


@pytest.mark.parametrize("name", ["knittubeinit", "knittubebroken", "blenderobj", "houdiniobj"])
def test_oracle_directsum_matches_golden(name, golden_dir):
    o = pyoracle.Oracle().load_bcc(golden_bcc(name, golden_dir))
    text, mean_off, _ = o.certificate(direct=True)
    assert text == golden_certificate(name)
    assert mean_off < 1e-12


def test_readme_answers():
    # README.md:71-78 (glove -> "70") and :86-94 (knittubebroken -> 5,6,-2).
    assert golden_certificate("glove") == "70\n"
    assert golden_certificate("knittubebroken") == "39\n5,6,-2\n"


@pytest.mark.parametrize("name", ["knittubebroken", "houdiniobj"])
def test_committed_pair_sums_reproduce(name, golden_dir):
    o = pyoracle.Oracle().load_bcc(golden_bcc(name, golden_dir)).prepare(True)
    ref = np.load(os.path.join(GOLDEN, "pairs", name + ".npz"))
    pairs = o.pairs()
    assert np.array_equal(pairs, ref["pairs"])
    off, _ = o.polylines()
    assert np.array_equal(np.diff(off), ref["vertex_counts"])
    method = pyoracle.DIRECT_ONE_ARCTAN if len(off) - 1 < 6 else pyoracle.DIRECT_FAST
    lk, _, _, _ = o.eval_pairs(method, pairs)
    np.testing.assert_allclose(lk, ref["lk_direct"], rtol=0, atol=1e-9)


@pytest.mark.parametrize("name", ["knittubebroken", "glove"])
def test_oracle_curve_order_barneshut(name, golden_dir):
    # The product's default Barnes-Hut, restated in FP64 in the oracle
    # (curve-order trees, small node pairs summed exactly): within the
    # Barnes-Hut target error (0.1, lnc.cpp:25) of the FP64 direct sums the
    # reference's own certificates were made from, the same integers, and
    # buckets replace far-field terms by exact segment pairs.
    o = pyoracle.Oracle().load_bcc(golden_bcc(name, golden_dir)).prepare(True)
    pairs = o.pairs()
    ref = np.load(os.path.join(GOLDEN, "pairs", name + ".npz"))
    runs = {b: o.eval_curve_bh(pairs, beta=2.0, bucket=b) for b in (1, 8)}
    for b, (lk, err, nfar, nex) in runs.items():
        assert np.array_equal(np.rint(lk), np.rint(ref["lk_direct"]))
        assert np.abs(lk - ref["lk_direct"]).max() < 0.1
        assert np.all(err >= 0)
    assert runs[8][2].sum() < runs[1][2].sum()
    assert runs[8][3].sum() > runs[1][3].sum()
    # Bucket 8 sums more of each pair exactly: on average closer to the direct sum.
    assert np.abs(runs[8][0] - ref["lk_direct"]).mean() <= np.abs(runs[1][0] - ref["lk_direct"]).mean()


@pytest.mark.parametrize("workload", ["ring_chain", "knots", "polymer"])
def test_oracle_curve_order_barneshut_on_synthetic_loops(workload):
    # The restated default Barnes-Hut on seeded synthetic loops (the ring
    # chain of the benchmark suite, torus knots, interleaved walks): the
    # integers of the oracle's FP64 direct sum for bucket 1 and 8.
    from fastlinkingnumbers_b200 import workloads as W
    if workload == "ring_chain":
        off, xyz = W.ring_chain(seed=5)
    elif workload == "knots":
        off, xyz = W.mixed_batch(seed=5, n_loops=24, hi=2000, cube=30.0)
    else:
        off, xyz = W.polymer(seed=5, n_loops=6, n_steps=3000, cube=40.0)
    o = pyoracle.Oracle().set_polylines(off, xyz)
    pairs = o.pairs()
    assert len(pairs) > 0
    lk_d, _, _, _ = o.eval_pairs(pyoracle.DIRECT_FAST, pairs)
    for b in (1, 8):
        lk, err, nfar, nex = o.eval_curve_bh(pairs, beta=2.0, bucket=b)
        assert np.array_equal(np.rint(lk), np.rint(lk_d))
        assert np.abs(lk - lk_d).max() < 0.1


@pytest.mark.parametrize("bucket", [1, 8])
def test_beta_retry_continues_from_the_first_pass(bucket, golden_dir):
    # The retry pass at beta* visits the same node pairs whether it starts
    # from the roots or from the beta0 pass's far node pairs with that pass's
    # exact terms reused: same sums (to FP64 summation order), same error
    # estimate, same far-field and exact counts.
    from fastlinkingnumbers_b200 import workloads as W
    off, xyz = W.polymer(seed=9, n_loops=6, n_steps=4000, cube=45.0)
    o = pyoracle.Oracle().set_polylines(off, xyz)
    pairs = o.pairs()
    assert len(pairs) > 5
    for beta in (2.3, 3.0, 10.0):
        lk, err, nf, nx = o.eval_curve_bh(pairs, beta=beta, bucket=bucket)
        lkc, errc, nfc, nxc = o.eval_curve_bh(pairs, beta=beta, bucket=bucket, continue_from=2.0)
        np.testing.assert_allclose(lkc, lk, rtol=0, atol=1e-10)
        np.testing.assert_allclose(errc, err, rtol=1e-10, atol=1e-15)
        assert np.array_equal(nfc, nf) and np.array_equal(nxc, nx)
