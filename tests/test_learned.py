"""The learned Barnes–Hut opening criterion (no counterpart in the reference):
the training kernel's gradients against a numpy float64 restatement of the
MLP, the traversal's BF16 warp-MMA inference against the FP32 forward, and
learned Barnes–Hut on held-out polymer loops against the plain traversal and
the FP64 direct sum.

Tolerances: gradients within 2e-3 of the largest gradient entry (FP32
forward/backward, FP32 atomic sums over samples); BF16 inference within
0.03 + 0.01 |y| of the FP32 output (BF16 inputs, weights and hidden
activations, FP32 accumulation); learned Barnes–Hut certificates identical
to the FP64 direct sum's.
"""
import numpy as np
import pytest

from fastlinkingnumbers_b200 import Engine, LearnedCriterion, Model, workloads
from fastlinkingnumbers_b200 import _native as N
from mlp_ref import _features, _init, mlp_forward, mlp_loss_grad

pytestmark = pytest.mark.gpu


def _polymer(seed, loops=40, steps=20_000, cube=300.0):
    """Closed Gaussian random walks and their potentially linked pairs."""
    off, xyz = workloads.polymer(seed=seed, n_loops=loops, n_steps=steps, cube=cube)
    m = Model().SetCurves(3, -np.diff(off).astype(np.int32), xyz)
    poff, pxyz, pairs, _ = m.Prepare(True)
    return poff, pxyz, pairs


@pytest.fixture(scope="module")
def engine():
    return Engine(0)


@pytest.mark.parametrize("n,q", [(1000, 0.9), (128, 0.5), (4097, 0.75)])
def test_training_gradients_match_numpy(engine, n, q):
    rng = np.random.default_rng(n)
    p = _init(rng)
    X, T = _features(rng, n), rng.uniform(-10, -1, n).astype(np.float32)
    loss, g = engine.mlp_gradients(p, X, T, q)
    ref_loss, ref_g = mlp_loss_grad(p, X, T, q)
    assert abs(loss - ref_loss) <= 1e-4 * max(1.0, abs(ref_loss))
    tol = 2e-3 * np.abs(ref_g).max()
    np.testing.assert_allclose(g, ref_g, rtol=0, atol=tol)


def test_fp32_forward_matches_numpy(engine):
    rng = np.random.default_rng(5)
    p = _init(rng)
    X = _features(rng, 3000)
    y = engine.mlp_predict(p, X, use_mma=False)
    np.testing.assert_allclose(y, mlp_forward(p, X), rtol=1e-5, atol=1e-4)


@pytest.fixture(scope="module")
def polymer_small():
    return _polymer(41)


def test_mma_inference_matches_fp32_on_traversal_features(engine, polymer_small):
    off, xyz, pairs = polymer_small
    X, T, S, E = engine.learned_collect(xyz, off, pairs, cap=20000, s_min=1.0, sample_keep=0.5)
    # The keep rate is lowered until the sample fits the cap; most samples
    # are small enough for the exact range sum.
    assert 10000 <= len(X) <= 20000
    assert np.all(S >= 1.0 - 1e-6) and np.all(S <= 2.5 + 1e-4)
    assert np.all(np.isfinite(T)) and np.all(T >= -14.01)
    rng = np.random.default_rng(1)
    p = _init(rng)
    y32 = engine.mlp_predict(p, X, use_mma=False)
    ybf = engine.mlp_predict(p, X, use_mma=True)
    assert np.all(np.abs(ybf - y32) <= 0.03 + 0.01 * np.abs(y32))


def test_learned_barneshut_on_held_out_loops(engine):
    # Train on one seed of dense closed random walks (60 x 50k segments), apply
    # to another seed.
    off_tr, xyz_tr, pairs_tr = _polymer(51, loops=60, steps=50_000, cube=250.0)
    off, xyz, pairs = _polymer(52, loops=60, steps=50_000, cube=250.0)
    # Trained and applied on the reference's traversal (leaf pairs only,
    # bh_bucket 1): the recorded node pairs are those the criterion then sees.
    model = LearnedCriterion.train(engine, xyz_tr, off_tr, pairs_tr, params=N.default_params(bh_bucket=1))
    info = model.info()
    assert info["samples"] > 100_000 and info["val_coverage"] > 0.85, info
    lk_plain, _, _ = engine.linking_numbers(xyz, off, pairs, "barneshut", bh_bucket=1)
    s_plain = engine.stats()
    engine.set_learned(model)
    try:
        lk_l, err_l, fl_l = engine.linking_numbers(xyz, off, pairs, "barneshut", bh_bucket=1)
        s_l = engine.stats()
    finally:
        engine.set_learned(None)
    # Same integers as the plain traversal on every pair; the FP64 direct sum
    # on the 40 pairs closest to a rounding boundary and 40 random ones.
    assert np.array_equal(np.rint(lk_l), np.rint(lk_plain))
    assert np.abs(lk_l - lk_plain).max() < 0.05
    frac = np.abs(lk_l - np.rint(lk_l))
    pick = np.unique(np.concatenate([np.argsort(-frac)[:40],
                                     np.random.default_rng(3).permutation(len(pairs))[:40]]))
    lk_d, _, _ = engine.linking_numbers(xyz, off, pairs[pick], "directsum", precision=N.PREC_FP64)
    assert np.array_equal(np.rint(lk_l[pick]), np.rint(lk_d))
    # within the Barnes-Hut target error (0.1, lnc.cpp:25)
    assert np.abs(lk_l[pick] - lk_d).max() < 0.1
    # The gain: node pairs the traversal no longer evaluates (the kernel
    # time, which the inference adds to, is reported alongside). It is about
    # 1 % here with the continued retry (2-4 % when the retry re-ran from the
    # roots; training sums gradients with FP32 atomics, so the trained weights
    # vary slightly from run to run).
    work_plain = s_plain["bh_far_evals"] + s_plain["bh_leaf_evals"]
    work_l = s_l["bh_far_evals"] + s_l["bh_leaf_evals"]
    print(f"learned: {work_l:.4g} node pairs vs {work_plain:.4g} plain; main kernel "
          f"{s_l['ms_main_kernel']:.2f} ms vs {s_plain['ms_main_kernel']:.2f} ms")
    assert work_l < 0.99 * work_plain, (work_l, work_plain)
    # Turned off again: the plain traversal's exact node-pair counts.
    engine.linking_numbers(xyz, off, pairs, "barneshut", bh_bucket=1)
    s_off = engine.stats()
    assert s_off["bh_far_evals"] == s_plain["bh_far_evals"]


def test_learned_criterion_rejects_other_schedules(engine, polymer_small):
    off, xyz, pairs = polymer_small
    p = _init(np.random.default_rng(2))
    model = LearnedCriterion.from_params(p, s_min=1.0, log10_tau=-6.0)
    engine.set_learned(model)
    try:
        with pytest.raises(N.FlnError):
            engine.linking_numbers(xyz, off, pairs[:10], "barneshut", bh_schedule=1)
    finally:
        engine.set_learned(None)


def test_learned_time_on_default_path(engine):
    # The default traversal (exact buckets of 8 segments, frontier retry):
    # plain against learned, the MLP applied to every candidate and only to
    # node pairs whose smaller node holds >= 32 segments. Device time of the
    # whole stage, best of three runs each. Integers must agree; the measured
    # times and node pairs are printed (and bounded: the learned run may not
    # evaluate more node pairs than the plain one).
    off_tr, xyz_tr, pairs_tr = _polymer(53, loops=60, steps=50_000, cube=250.0)
    off, xyz, pairs = _polymer(54, loops=60, steps=50_000, cube=250.0)
    model = LearnedCriterion.train(engine, xyz_tr, off_tr, pairs_tr)

    def best_of(n=3):
        runs = []
        for _ in range(n):
            lk, _, _ = engine.linking_numbers(xyz, off, pairs, "barneshut")
            runs.append((engine.stats(), lk))
        return min(runs, key=lambda r: r[0]["ms_kernels"])

    s_p, lk_p = best_of()
    res = {}
    for min_seg in (0, 32):
        model.configure(min_candidates=4, min_node_segments=min_seg)
        engine.set_learned(model)
        try:
            res[min_seg] = best_of()
        finally:
            engine.set_learned(None)
    work_p = s_p["bh_far_evals"] + s_p["bh_exact_entries"]
    for min_seg, (s, lk) in res.items():
        assert np.array_equal(np.rint(lk), np.rint(lk_p))
        work = s["bh_far_evals"] + s["bh_exact_entries"]
        print(f"learned (min_node_segments {min_seg}): {s['ms_kernels']:.2f} ms vs plain {s_p['ms_kernels']:.2f} ms "
              f"({s['ms_kernels'] / s_p['ms_kernels']:.3f}x), node pairs {work:.5g} vs {work_p:.5g} "
              f"({work / work_p:.4f}x)")
        assert work <= work_p * 1.001
