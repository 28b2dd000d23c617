"""The beta retry continued from the first pass's frontier.

linking_number_certificate.cpp:165-184 re-runs a pair whose scaled error
estimate is too large at beta* = min((err / 0.1)^(1/4) beta0, beta_limit).
A node pair opened at beta0 is opened at beta* > beta0 (far at beta* implies
far at beta0), and an exact node pair stays exact (the bucket test does not
depend on beta), so the beta* traversal is the beta0 traversal continued from
its far node pairs. The engine records those far pairs in its first pass and
continues from them (bh_retry_from_roots = 0, the default): a frontier pair
still far at beta* keeps its first-pass value (a far-field value does not
depend on beta), one that opens gives its value back and is traversed.

Checked against the oracle's restatement (curve_bh_eval_continued: the
continued pass node pair for node pair, sums within 2e-5 as the one-pass
parity test, estimates within 1e-3 relative, counts within 1e-5), and
against the engine's own retry from the roots (the same node pairs: integers
and flags equal, sums within 1e-8, the rounding of the fixed-point partial
sums of differently grouped batches).
"""
import numpy as np
import pytest

from conftest import golden_bcc
from fastlinkingnumbers_b200 import Engine, Model, workloads
from oracle import pyoracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def engine():
    return Engine(0)


def _polymer(engine, seed=71, loops=24, steps=20_000, cube=220.0):
    off, xyz = workloads.polymer(seed=seed, n_loops=loops, n_steps=steps, cube=cube)
    m = Model().SetCurves(3, -np.diff(off).astype(np.int32), xyz)
    poff, pxyz, pairs, _ = m.Prepare(True, engine=engine)
    return poff, pxyz, pairs


def _golden(name, golden_dir):
    m = Model().ImportFromFile(golden_bcc(name, golden_dir))
    poff, pxyz, pairs, _ = m.Prepare(True)
    return poff, pxyz, pairs


@pytest.mark.parametrize("case", ["knittubebroken", "glove", "polymer"])
@pytest.mark.parametrize("beta1", [2.5, 4.0])
def test_continued_retry_matches_oracle(engine, case, beta1, golden_dir):
    # Every pair with a far-field term retries at beta1 (a vanishing target
    # error makes beta* = beta_limit = beta1); no escalation, no recompute.
    poff, pxyz, pairs = _polymer(engine) if case == "polymer" else _golden(case, golden_dir)
    o = pyoracle.Oracle().set_polylines(poff, pxyz)
    lk0_o, err0_o, far0_o, ex0_o = o.eval_curve_bh(pairs, beta=2.0, bucket=8)
    lk1_o, err1_o, far1_o, ex1_o = o.eval_curve_bh(pairs, beta=beta1, bucket=8, continue_from=2.0)
    lk, err, flags = engine.linking_numbers(pxyz, poff, pairs, "barneshut", target_error=1e-300,
                                            barnes_hut_beta_limit=beta1, bh_escalations=0, fp64_margin=0.0,
                                            bh_err_limit=1e30)
    s = engine.stats()
    # A pair retries when its estimate is positive; one whose estimate rounds
    # to zero in the fixed-point sum (far pairs of ~1e-12 error) keeps its
    # first pass, so the expected values follow the engine's retry flags.
    retried = (flags & 2) != 0
    assert retried.sum() > 0 and np.all(far0_o[retried] > 0)
    assert s["bh_retry_from_roots"] == 0 and s["bh_front_records"] > 0
    np.testing.assert_allclose(lk, np.where(retried, lk1_o, lk0_o), rtol=0, atol=2e-5)
    np.testing.assert_allclose(err, np.where(retried, err1_o, err0_o), rtol=1e-3, atol=1e-9)
    # Frontier pairs still far at beta1 keep their first-pass values and are
    # not evaluated again: evaluated + kept = the oracle's far pairs.
    far_total = float(far0_o.sum() + far1_o[retried].sum())
    ex_total = float(np.where(retried, ex1_o, ex0_o).sum())
    assert abs(s["bh_far_evals"] + s["bh_far_reused"] - far_total) <= 1e-5 * far_total + 2
    assert abs(s["bh_leaf_evals"] - ex_total) <= 1e-5 * ex_total + 64
    # The frontier was used (at beta1 = 4 every frontier pair may open).
    assert s["bh_far_reused"] + s["bh_far_subtracted"] > 0


@pytest.mark.parametrize("case", ["polymer", "mixed"])
def test_continued_retry_equals_retry_from_roots(engine, case):
    if case == "polymer":
        poff, pxyz, pairs = _polymer(engine, seed=61, loops=30, cube=250.0)
    else:
        # Knots and walks of mixed sizes, packed densely enough that a pair retries.
        off, xyz = workloads.mixed_batch(seed=9, n_loops=300, hi=2 ** 14, cube=80.0)
        m = Model().SetCurves(3, -np.diff(off).astype(np.int32), xyz)
        poff, pxyz, pairs, _ = m.Prepare(True, engine=engine)
    lk_r, err_r, fl_r = engine.linking_numbers(pxyz, poff, pairs, "barneshut", bh_retry_from_roots=1)
    s_r = engine.stats()
    lk_c, err_c, fl_c = engine.linking_numbers(pxyz, poff, pairs, "barneshut")
    s_c = engine.stats()
    assert s_c["beta_retried"] == s_r["beta_retried"] > 0
    assert s_r["bh_retry_from_roots"] == s_r["beta_retried"] and s_c["bh_retry_from_roots"] == 0
    np.testing.assert_array_equal(fl_c, fl_r)
    assert np.array_equal(np.rint(lk_c), np.rint(lk_r))
    np.testing.assert_allclose(lk_c, lk_r, rtol=0, atol=1e-8)
    np.testing.assert_allclose(err_c, err_r, rtol=1e-6, atol=1e-12)
    # The continuation evaluates fewer node pairs: the first pass's exact
    # terms, its opened node pairs and its far pairs that stay far are not
    # evaluated again.
    assert s_c["bh_far_evals"] < s_r["bh_far_evals"] and s_c["bh_leaf_evals"] < s_r["bh_leaf_evals"]
    assert s_c["bh_far_reused"] > 0 and s_r["bh_far_reused"] == 0
    print(f"{case}: retried {s_c['beta_retried']} of {len(pairs)}, retry {s_c['ms_retry']:.2f} ms "
          f"(from roots {s_r['ms_retry']:.2f} ms), far {s_c['bh_far_evals']:.3g} vs {s_r['bh_far_evals']:.3g}")


@pytest.mark.parametrize("budget", [0, 16])
def test_repeated_calls_are_bit_identical(engine, budget):
    # Each batch writes its own frontier records and exact-list chunks and
    # adds its far-field sum once, so a slot's sums are the same integer sums
    # of the same partial sums in every call, whatever the warps' timing (the
    # exact list also runs beside the next traversal on a second stream). A
    # small budget spreads each loop pair over many batches.
    poff, pxyz, pairs = _polymer(engine, seed=61, loops=30, cube=250.0)
    runs = []
    for _ in range(3):
        runs.append(engine.linking_numbers(pxyz, poff, pairs, "barneshut", bh_budget=budget))
        s = engine.stats()
        assert s["beta_retried"] > 0 and s["bh_front_records"] > 0 and s["bh_retry_from_roots"] == 0
    for lk, err, fl in runs[1:]:
        assert np.array_equal(lk, runs[0][0]) and np.array_equal(err, runs[0][1])
        np.testing.assert_array_equal(fl, runs[0][2])


def test_serial_exact_list_gives_the_same_bits(engine):
    # bh_exact_serial runs each round's exact list on the context's stream
    # after its traversal instead of beside the next one: the same work, the
    # same partial sums, so the same bits.
    poff, pxyz, pairs = _polymer(engine, seed=61, loops=30, cube=250.0)
    a = engine.linking_numbers(pxyz, poff, pairs, "barneshut")
    s_a = engine.stats()
    b = engine.linking_numbers(pxyz, poff, pairs, "barneshut", bh_exact_serial=1)
    s_b = engine.stats()
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
    assert s_a["ms_traverse"] > 0 and s_b["ms_traverse"] > 0 and s_a["ms_exact"] > 0 and s_b["ms_exact"] > 0


def test_learned_criterion_with_continued_retry(engine):
    # The learned criterion scales its threshold with (beta0 / beta)^4, so a
    # pair it opens at beta0 it also opens at beta*: the continuation applies.
    # Same integers as the plain run.
    from fastlinkingnumbers_b200 import LearnedCriterion
    poff, pxyz, pairs = _polymer(engine, seed=61, loops=30, cube=250.0)
    toff, txyz, tpairs = workloads.walk_pairs(seed=13, n_pairs=4, n_steps=40_000)
    model = LearnedCriterion.train(engine, txyz, toff, tpairs, epochs=10)
    lk0, _, _ = engine.linking_numbers(pxyz, poff, pairs, "barneshut")
    engine.set_learned(model)
    try:
        lk1, _, _ = engine.linking_numbers(pxyz, poff, pairs, "barneshut")
        s = engine.stats()
    finally:
        engine.set_learned(None)
    assert np.array_equal(np.rint(lk1), np.rint(lk0))
    assert s["bh_retry_from_roots"] == 0
