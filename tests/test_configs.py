"""Full-size parity of the mixed-size batch workload: 5,000 loops, half (p,q)
torus knots and half closed random walks, 16 to 2^18 segments each (134M
segments; 137M and 35,717 potentially linked pairs after Discretize).

The FP64 direct sum of every pair would take hours. The certificate is
therefore checked where it can fail: every pair's real sum is finite and
either has margin >= 0.25 to the rounding boundary or was recomputed in
FP64. The FP64 direct sum runs on the 40 non-recomputed pairs with the
smallest margin and on 40 random pairs, and must give the same integers and
agree within 0.05 (Barnes-Hut error). The mixed direct sum must agree with
the FP64 direct sum on the same pairs within 1e-5.
"""
import numpy as np
import pytest

from fastlinkingnumbers_b200 import Engine, Model, workloads
from fastlinkingnumbers_b200 import _native as N

pytestmark = pytest.mark.gpu


def test_mixed_batch_full_size():
    off, xyz = workloads.mixed_batch(seed=5)
    m = Model().SetCurves(3, -np.diff(off).astype(np.int32), xyz)
    del xyz
    poff, pxyz, pairs, _ = m.Prepare(True)
    assert len(pairs) > 30_000
    n = np.diff(poff).astype(np.float64)
    work = n[pairs[:, 0]] * n[pairs[:, 1]]
    eng = Engine(0)
    try:
        lk, err, flags = eng.linking_numbers(pxyz, poff, pairs, "barneshut")
        s = eng.stats()
        assert np.all(np.isfinite(lk))
        margin = 0.5 - np.abs(lk - np.rint(lk))
        recomputed = (flags & N.PAIR_FP64_RECOMPUTED) != 0
        assert np.all((margin >= 0.25) | recomputed)
        assert np.all((err <= 0.25) | recomputed)
        assert s["bh_wait_timeouts"] == 0
        # FP64 direct sum where the certificate is most fragile, and at random.
        cand = np.flatnonzero(~recomputed & (work <= 2e10))
        low = cand[np.argsort(margin[cand])[:40]]
        rnd = np.random.default_rng(7).choice(cand, size=min(40, len(cand)), replace=False)
        pick = np.unique(np.concatenate([low, rnd]))
        lk64, _, _ = eng.linking_numbers(pxyz, poff, pairs[pick], "directsum", precision=N.PREC_FP64)
        assert np.array_equal(np.rint(lk[pick]), np.rint(lk64))
        assert np.abs(lk[pick] - lk64).max() < 0.05
        lkm, _, _ = eng.linking_numbers(pxyz, poff, pairs[pick], "directsum", precision=N.PREC_MIXED,
                                        fp64_margin=0.0)
        print(f"mixed batch: {len(pairs)} pairs, BH {s['ms_kernels']:.1f} ms, max |BH - FP64| "
              f"{np.abs(lk[pick] - lk64).max():.3g}, max |mixed - FP64| {np.abs(lkm - lk64).max():.3g}, "
              f"recomputed {int(recomputed.sum())}, retried {s['beta_retried']}")
        np.testing.assert_allclose(lkm, lk64, rtol=0, atol=1e-5)
    finally:
        eng.close()
