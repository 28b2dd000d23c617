"""GPU parity: the CUDA kernels through the C ABI against the CPU oracle and
the reference's golden vectors.

Tolerances (stated per test): FP64 direct sum within 1e-9 of the oracle's
FP64 DirectFast per pair; the mixed-precision direct sum within 1e-5 per
pair (FP32 terms, FP64 sums and near-singular terms); Barnes–Hut within its
own error bound of the FP64 direct sum, and within 1e-5 of the oracle's
Barnes–Hut on the same (reference kd-median) tree. Certificates: byte-equal.
"""
import os

import numpy as np
import pytest

from conftest import FIXTURES, GOLDEN, golden_bcc, golden_certificate
from fastlinkingnumbers_b200 import Engine, FlnError, LinkingNumberCertificate, Model, workloads
from fastlinkingnumbers_b200 import _native as N
from oracle import pyoracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def engine():
    return Engine(0)


def _prepared(name, golden_dir):
    m = Model().ImportFromFile(golden_bcc(name, golden_dir))
    off, xyz, pairs, _ = m.Prepare(True)
    return m, off, xyz, pairs


@pytest.mark.parametrize("name", FIXTURES)
def test_fp64_direct_matches_oracle(engine, name, golden_dir):
    _, off, xyz, pairs = _prepared(name, golden_dir)
    ref = np.load(os.path.join(GOLDEN, "pairs", name + ".npz"))
    assert np.array_equal(pairs, ref["pairs"])
    lk, _, flags = engine.linking_numbers(xyz, off, pairs, "directsum", precision=N.PREC_FP64)
    np.testing.assert_allclose(lk, ref["lk_direct"], rtol=0, atol=1e-9)
    assert not flags.any()


@pytest.mark.parametrize("name", FIXTURES)
def test_mixed_direct_matches_oracle(engine, name, golden_dir):
    _, off, xyz, pairs = _prepared(name, golden_dir)
    ref = np.load(os.path.join(GOLDEN, "pairs", name + ".npz"))
    lk, _, _ = engine.linking_numbers(xyz, off, pairs, "directsum", precision=N.PREC_MIXED)
    np.testing.assert_allclose(lk, ref["lk_direct"], rtol=0, atol=1e-5)


@pytest.mark.parametrize("name", FIXTURES)
@pytest.mark.parametrize("direct", [True, False])
def test_certificates_match_golden(engine, name, direct, golden_dir):
    m = Model().ImportFromFile(golden_bcc(name, golden_dir))
    c = LinkingNumberCertificate().ComputeFromModel(m, force_direct_sum=direct, engine=engine)
    assert c.text() == golden_certificate(name)


@pytest.mark.parametrize("name", FIXTURES)
def test_barneshut_within_error_of_direct(engine, name, golden_dir):
    _, off, xyz, pairs = _prepared(name, golden_dir)
    ref = np.load(os.path.join(GOLDEN, "pairs", name + ".npz"))
    lk, err, flags = engine.linking_numbers(xyz, off, pairs, "barneshut")
    dev = np.abs(lk - ref["lk_direct"])
    # Off-integer error of the same order as the reference's own BH run.
    assert dev.max() < 0.1
    assert np.mean(dev) < 5 * max(np.mean(np.abs(ref["lk_bh"] - ref["lk_direct"])), 1e-4)


@pytest.mark.parametrize("name", ["knittubeinit", "knittubebroken", "blenderobj"])
def test_barneshut_reference_tree_matches_oracle(engine, name, golden_dir):
    # Same kd-median trees as the reference (bh_tree=1): same node pairs,
    # so the GPU sum equals the oracle's FP64 BH up to FP32 evaluation.
    _, off, xyz, pairs = _prepared(name, golden_dir)
    o = pyoracle.Oracle().set_polylines(off, xyz)
    lk_o, err_o, _, _ = o.eval_pairs(pyoracle.BARNES_HUT, pairs, bh_parallel=True)
    lk, err, _ = engine.linking_numbers(xyz, off, pairs, "barneshut", bh_tree=1, fp64_margin=0.0,
                                        bh_escalations=0, bh_err_limit=1e30)
    np.testing.assert_allclose(lk, lk_o, rtol=0, atol=2e-5)
    np.testing.assert_allclose(err, err_o, rtol=1e-3, atol=1e-9)


def _circle(center, normal_axis, n=64, radius=1.0, phase=0.0):
    t = phase + 2 * np.pi * np.arange(n) / n
    c, s = radius * np.cos(t), radius * np.sin(t)
    z = np.zeros(n)
    pts = {2: (c, s, z), 1: (c, z, s), 0: (z, c, s)}[normal_axis]
    return np.stack(pts, axis=1) + np.asarray(center, dtype=float)


def test_known_answers(engine):
    # Hopf link: +-1; far apart: 0; orientation reversal flips the sign; (2, 2q)
    # torus link components: q.
    a = _circle([0, 0, 0], 2)
    b = _circle([1, 0, 0], 1)
    far = _circle([10, 0, 0], 1)
    for prec in (N.PREC_FP64, N.PREC_MIXED):
        h = engine.direct_pair(a, b, prec)
        assert abs(abs(h) - 1) < 1e-6
        assert abs(engine.direct_pair(a, b[::-1], prec) + h) < 1e-6
        assert abs(engine.direct_pair(a, far, prec)) < 1e-6
    for q in (1, 2, 3, 5):
        n = 400
        t = 2 * np.pi * np.arange(n) / n
        comps = []
        for shift in (0.0, np.pi):
            phi = q * t + shift
            r = 1.0 + 0.4 * np.cos(phi)
            comps.append(np.stack([r * np.cos(t), r * np.sin(t), 0.4 * np.sin(phi)], axis=1))
        # Components of the (2, 2q) torus link: phi = q theta and phi = q theta + pi.
        lk = engine.direct_pair(comps[0], comps[1], N.PREC_FP64)
        assert abs(abs(lk) - q) < 1e-6


def test_ring_chain_certificate(engine, tmp_path):
    off, xyz = workloads.ring_chain()
    m = Model().SetCurves(3, -np.diff(off).astype(np.int32), xyz)
    for direct in (True, False):
        c = LinkingNumberCertificate().ComputeFromModel(m, force_direct_sum=direct, engine=engine)
        ent = c.entries()
        assert [tuple(e[:2]) for e in ent] == [(i, i + 1) for i in range(63)]
        assert set(np.abs(ent[:, 2])) == {1}


def test_chain_mail_full_size(engine):
    # Chain-mail sheet at full size (10,000 48-gons): the mixed-precision
    # direct sum, its FP64 recompute and Barnes–Hut all give the oracle's
    # direct-sum certificate; real sums agree within the stated tolerances.
    off, xyz = workloads.chain_mail()
    m = Model().SetCurves(3, -np.diff(off).astype(np.int32), xyz)
    poff, pxyz, pairs, _ = m.Prepare(True)
    o = pyoracle.Oracle().set_polylines(poff, pxyz)
    lk_o, _, _, _ = o.eval_pairs(pyoracle.DIRECT_FAST, pairs)
    lk64, _, _ = engine.linking_numbers(pxyz, poff, pairs, "directsum", precision=N.PREC_FP64)
    np.testing.assert_allclose(lk64, lk_o, rtol=0, atol=1e-9)
    lkm, _, _ = engine.linking_numbers(pxyz, poff, pairs, "directsum", precision=N.PREC_MIXED)
    np.testing.assert_allclose(lkm, lk_o, rtol=0, atol=1e-5)
    lkb, _, _ = engine.linking_numbers(pxyz, poff, pairs, "barneshut")
    assert np.array_equal(np.round(lkb), np.round(lk_o))
    assert np.array_equal(np.round(lkm), np.round(lk_o))


def test_beta_retry_path(engine, golden_dir):
    # A small initial beta forces the reference's retry rule (lnc.cpp:165-184).
    _, off, xyz, pairs = _prepared("knittubebroken", golden_dir)
    ref = np.load(os.path.join(GOLDEN, "pairs", "knittubebroken.npz"))
    lk, err, flags = engine.linking_numbers(xyz, off, pairs, "barneshut", barnes_hut_init_beta=1.0)
    assert (flags & N.PAIR_BETA_RETRIED).any()
    assert np.array_equal(np.round(lk), np.round(ref["lk_direct"]))


def test_low_margin_pairs_are_recomputed_in_fp64(engine, golden_dir):
    # fp64_margin = 0.5 marks every pair as low-margin: all go through the
    # FP64 direct sum and must equal it.
    _, off, xyz, pairs = _prepared("knittubeinit", golden_dir)
    ref = np.load(os.path.join(GOLDEN, "pairs", "knittubeinit.npz"))
    lk, _, flags = engine.linking_numbers(xyz, off, pairs, "barneshut", fp64_margin=0.5)
    assert (flags & N.PAIR_FP64_RECOMPUTED).all()
    lk2, err2, flags2 = engine.linking_numbers(xyz, off, pairs, "barneshut", bh_err_limit=0.0,
                                               bh_escalations=1)
    # Every pair is escalated once (beta x2) and then recomputed in FP64.
    assert (flags2 & N.PAIR_BETA_ESCALATED).all() and (flags2 & N.PAIR_FP64_RECOMPUTED).all()
    np.testing.assert_allclose(lk2, ref["lk_direct"], rtol=0, atol=1e-9)
    np.testing.assert_allclose(lk, ref["lk_direct"], rtol=0, atol=1e-9)


def test_edge_cases(engine):
    a = _circle([0, 0, 0], 2, n=2)  # two-vertex loops (a segment there and back)
    b = _circle([0.5, 0, 0], 1, n=3)
    lk, _, _ = engine.linking_numbers(np.concatenate([a, b]), [0, 2, 5], [[0, 1]], "directsum")
    assert np.isfinite(lk).all()
    lk, _, _ = engine.linking_numbers(np.zeros((0, 3)), [0], np.zeros((0, 2), np.int32), "barneshut")
    assert lk.shape == (0,)
    with pytest.raises(FlnError) as e:
        engine.linking_numbers(a, [0, 2], [[0, 1]], "directsum")
    assert e.value.status == 1
    with pytest.raises(FlnError) as e:
        engine.linking_numbers(np.concatenate([a, a]), [0, 2, 4], [[0, 0]], "directsum")
    assert e.value.status == 1
    # Very different loop sizes in one launch.
    big = _circle([0, 0, 0], 2, n=5000)
    small = _circle([1, 0, 0], 1, n=16)
    xyz = np.concatenate([big, small, _circle([1, 0, 0.001], 1, n=7)])
    lk, _, _ = engine.linking_numbers(xyz, [0, 5000, 5016, 5023], [[0, 1], [0, 2], [1, 2]], "directsum",
                                      precision=N.PREC_FP64)
    assert abs(abs(lk[0]) - 1) < 1e-6 and abs(abs(lk[1]) - 1) < 1e-6


def test_device_pointer_entry(engine):
    torch = pytest.importorskip("torch")
    off, xyz = workloads.ring_chain(seed=4, n_rings=8)
    pairs = np.array([[i, i + 1] for i in range(7)], dtype=np.int32)
    d_xyz = torch.from_numpy(xyz).cuda()
    d_off = torch.from_numpy(off).cuda()
    d_pairs = torch.from_numpy(pairs).cuda()
    d_lk = torch.zeros(len(pairs), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    engine.linking_numbers_device(d_xyz.data_ptr(), d_off.data_ptr(), len(off) - 1, d_pairs.data_ptr(),
                                  len(pairs), d_lk.data_ptr(), method="directsum")
    host, _, _ = engine.linking_numbers(xyz, off, pairs, "directsum")
    np.testing.assert_allclose(d_lk.cpu().numpy(), host, rtol=0, atol=1e-12)


@pytest.mark.parametrize("name", ["knittubebroken", "glove"])
def test_traversal_schedules_agree(engine, name, golden_dir):
    # Fused rounds (default), the persistent work queue and the split-
    # evaluation rounds evaluate the same node pairs at the same beta; only
    # the grouping of the FP64 partial sums differs. The retry beta, (err /
    # 0.1)^(1/4) beta0, is computed by the host for rounds and on the device
    # for the persistent queue; one ulp of difference can flip a node pair
    # that sits on the opening boundary, so retried pairs agree within the
    # Barnes-Hut error and pairs run once agree to rounding. The persistent
    # and split schedules sum leaf pairs only (bh_bucket 1).
    _, off, xyz, pairs = _prepared(name, golden_dir)
    runs = []
    for sched in (0, 1, 2):
        lk, err, fl = engine.linking_numbers(xyz, off, pairs, "barneshut", bh_schedule=sched, bh_bucket=1)
        runs.append((lk, err, fl, engine.stats()))
    lk0, err0, fl0, s0 = runs[0]
    for lk, err, fl, s in runs[1:]:
        once = (fl == 0) & (fl0 == 0)
        assert once.mean() > 0.5
        np.testing.assert_allclose(lk[once], lk0[once], rtol=0, atol=1e-9)
        np.testing.assert_allclose(err[once], err0[once], rtol=1e-6, atol=1e-12)
        assert np.array_equal(np.rint(lk), np.rint(lk0))
        np.testing.assert_allclose(lk, lk0, rtol=0, atol=0.05)
        assert s["bh_wait_timeouts"] == 0


@pytest.mark.parametrize("name", ["knittubebroken", "glove"])
def test_buckets_keep_integers(engine, name, golden_dir):
    # Node pairs of at most bh_bucket segments a side are summed exactly
    # instead of being split further: fewer far-field terms, the same
    # integers, sums within the Barnes-Hut target error (0.1) of the FP64
    # direct sum.
    _, off, xyz, pairs = _prepared(name, golden_dir)
    ref = np.load(os.path.join(GOLDEN, "pairs", name + ".npz"))
    lk1, err1, _ = engine.linking_numbers(xyz, off, pairs, "barneshut", bh_bucket=1)
    s1 = engine.stats()
    assert np.array_equal(np.rint(lk1), np.rint(ref["lk_direct"]))
    for b in (2, 4, 8, 16):
        lk, err, _ = engine.linking_numbers(xyz, off, pairs, "barneshut", bh_bucket=b)
        s = engine.stats()
        assert np.array_equal(np.rint(lk), np.rint(ref["lk_direct"]))
        np.testing.assert_allclose(lk, ref["lk_direct"], rtol=0, atol=0.1)
        assert s["bh_far_evals"] < s1["bh_far_evals"]
        assert s["bh_leaf_evals"] > s1["bh_leaf_evals"]


@pytest.mark.parametrize("name", ["knittubebroken", "glove"])
@pytest.mark.parametrize("bucket", [1, 8])
def test_curve_order_barneshut_matches_oracle(engine, name, bucket, golden_dir):
    # The default tree and traversal against the oracle's FP64 restatement of
    # them (one pass at beta 2, no retry, no FP64 recompute): the same node
    # pairs, so the sums agree up to the FP32 far field and exact terms, and
    # the work counts agree up to node pairs on the opening boundary.
    _, off, xyz, pairs = _prepared(name, golden_dir)
    o = pyoracle.Oracle().set_polylines(off, xyz)
    lk_o, err_o, far_o, ex_o = o.eval_curve_bh(pairs, beta=2.0, bucket=bucket)
    lk, err, _ = engine.linking_numbers(xyz, off, pairs, "barneshut", bh_bucket=bucket, target_error=1e30,
                                        bh_escalations=0, fp64_margin=0.0, bh_err_limit=1e30)
    s = engine.stats()
    np.testing.assert_allclose(lk, lk_o, rtol=0, atol=2e-5)
    np.testing.assert_allclose(err, err_o, rtol=1e-3, atol=1e-9)
    assert abs(s["bh_far_evals"] - float(far_o.sum())) <= 1e-5 * float(far_o.sum()) + 2
    assert abs(s["bh_leaf_evals"] - float(ex_o.sum())) <= 1e-5 * float(ex_o.sum()) + 64


def test_buckets_ignored_on_reference_tree(engine, golden_dir):
    # The kd-median tree has no contiguous segment ranges: bh_bucket has no
    # effect there (leaf pairs only, the reference's traversal).
    _, off, xyz, pairs = _prepared("knittubebroken", golden_dir)
    a, ea, _ = engine.linking_numbers(xyz, off, pairs, "barneshut", bh_tree=1, bh_bucket=1)
    b, eb, _ = engine.linking_numbers(xyz, off, pairs, "barneshut", bh_tree=1, bh_bucket=16)
    np.testing.assert_array_equal(a, b)
    np.testing.assert_array_equal(ea, eb)


def test_buckets_on_polymer_loops(engine):
    # Long random walks, where most of the work sits near the leaves: every
    # bucket size gives the integers of the FP64 direct sum on a sample.
    off, xyz = workloads.polymer(seed=71, n_loops=24, n_steps=20_000, cube=220.0)
    m = Model().SetCurves(3, -np.diff(off).astype(np.int32), xyz)
    poff, pxyz, pairs, _ = m.Prepare(True, engine=engine)
    pick = np.random.default_rng(5).permutation(len(pairs))[:12]
    lk64, _, _ = engine.linking_numbers(pxyz, poff, pairs[pick], "directsum", precision=N.PREC_FP64)
    for b in (1, 4, 8, 16):
        lk, err, fl = engine.linking_numbers(pxyz, poff, pairs, "barneshut", bh_bucket=b)
        assert np.array_equal(np.rint(lk[pick]), np.rint(lk64))
        assert np.abs(lk[pick] - lk64).max() < 0.1


def test_bucket_argument_checked(engine, golden_dir):
    _, off, xyz, pairs = _prepared("knittubebroken", golden_dir)
    with pytest.raises(FlnError):
        engine.linking_numbers(xyz, off, pairs, "barneshut", bh_bucket=17)


def test_autotune_budget_keeps_results(engine):
    # The round budget changes only how work is handed between launches: the
    # same node pairs, grouped differently into FP64 partial sums (1e-9).
    off, xyz = workloads.polymer(seed=61, n_loops=30, n_steps=20_000, cube=250.0)
    m = Model().SetCurves(3, -np.diff(off).astype(np.int32), xyz)
    poff, pxyz, pairs, _ = m.Prepare(True, engine=engine)
    tuned, res = engine.autotune(pxyz, poff, pairs, sample_pairs=64)
    assert res["trials"] == 6 and res["sample_pairs"] == min(64, len(pairs))
    assert res["best_occupancy"] in (5, 6, 7)
    assert tuned.bh_budget in (128, 256, 512) and tuned.barnes_hut_init_beta == 2.0
    assert res["best_ms"] <= res["default_ms"]
    lk0, err0, fl0 = engine.linking_numbers(pxyz, poff, pairs, "barneshut")
    lk1, err1, fl1 = engine.linking_numbers(pxyz, poff, pairs, "barneshut", params=tuned)
    np.testing.assert_allclose(lk1, lk0, rtol=0, atol=1e-9)
    np.testing.assert_array_equal(fl1, fl0)
    tb, rb = engine.autotune(pxyz, poff, pairs, tune_beta=True, sample_pairs=64)
    assert rb["trials"] == 15 and tb.barnes_hut_init_beta in (1.5, 2.0, 2.5, 3.0)
    lk2, _, _ = engine.linking_numbers(pxyz, poff, pairs, "barneshut", params=tb)
    assert np.array_equal(np.rint(lk2), np.rint(lk0))
    # The exact-bucket size changes the node pairs, never the integers.
    tk, rk = engine.autotune(pxyz, poff, pairs, tune_bucket=True, sample_pairs=64)
    assert rk["trials"] == 11 and rk["best_bucket"] in (4, 6, 8, 10, 12, 16)
    lk3, _, _ = engine.linking_numbers(pxyz, poff, pairs, "barneshut", params=tk)
    assert np.array_equal(np.rint(lk3), np.rint(lk0))


@pytest.mark.parametrize("prec,tol", [(N.PREC_FP64, 1e-9), (N.PREC_MIXED, 1e-5)])
def test_direct_tile_shapes_and_autotune(engine, prec, tol, golden_dir):
    # Every tile shape of the direct sum gives the oracle's sums within the
    # precision's tolerance; the autotuner times them all and picks one.
    _, off, xyz, pairs = _prepared("knittubebroken", golden_dir)
    ref = np.load(os.path.join(GOLDEN, "pairs", "knittubebroken.npz"))["lk_direct"]
    for t in range(6):
        lk, _, _ = engine.linking_numbers(xyz, off, pairs, "directsum", precision=prec, direct_tile=t)
        np.testing.assert_allclose(lk, ref, rtol=0, atol=tol)
    tuned, res = engine.autotune_direct(xyz, off, pairs, precision=prec, sample_pairs=64)
    assert res["trials"] == 6 and 0 <= res["best_direct_tile"] < 6
    assert tuned.direct_tile == res["best_direct_tile"] and res["best_ms"] <= res["default_ms"]
    with pytest.raises(FlnError):
        engine.linking_numbers(xyz, off, pairs, "directsum", precision=prec, direct_tile=6)


def test_traversal_occupancy_keeps_results(engine, golden_dir):
    # The traversal kernels built for 5, 6 and 7 CTAs per SM walk the same node
    # pairs; only the grouping of the FP64 partial sums differs (1e-9).
    _, off, xyz, pairs = _prepared("knittubebroken", golden_dir)
    lk5, err5, fl5 = engine.linking_numbers(xyz, off, pairs, "barneshut", bh_occupancy=5)
    s5 = engine.stats()
    for occ in (6, 7):
        lk, err, fl = engine.linking_numbers(xyz, off, pairs, "barneshut", bh_occupancy=occ)
        s = engine.stats()
        np.testing.assert_allclose(lk, lk5, rtol=0, atol=1e-9)
        np.testing.assert_allclose(err, err5, rtol=1e-6, atol=1e-12)
        np.testing.assert_array_equal(fl, fl5)
        assert s["bh_far_evals"] == s5["bh_far_evals"] and s["bh_leaf_evals"] == s5["bh_leaf_evals"]
    with pytest.raises(FlnError):
        engine.linking_numbers(xyz, off, pairs, "barneshut", bh_occupancy=4)
