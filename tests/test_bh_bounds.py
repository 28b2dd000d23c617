"""The bounded failure paths of the Barnes–Hut traversal fire and are reported.

Two bounds keep every traversal finite and every wait short:

* the per-warp stacks: 224 node pairs in shared memory plus a global spill
  area (bh_spill_cap entries, at most 8192). A traversal that needs more
  abandons its pair, sets a status word, and the call returns
  FLN_ERR_STACK_OVERFLOW; the context stays usable.
* the persistent schedule's waits (bh_schedule 1): a warp waiting for work
  polls at most bh_wait_polls times, then sets a status bit and exits; the
  host then reruns the stage with budgeted rounds (fln_stats.bh_wait_timeouts).

Both are made to fire by lowering the bound through fln_params: no trap, no
unbounded wait, nothing that faults.
"""
import numpy as np
import pytest

from fastlinkingnumbers_b200 import Engine, FlnError, Model, workloads

pytestmark = pytest.mark.gpu

STACK_OVERFLOW = 11


@pytest.fixture(scope="module")
def case():
    eng = Engine(0)
    off, xyz = workloads.polymer(seed=71, n_loops=24, n_steps=20_000, cube=220.0)
    m = Model().SetCurves(3, -np.diff(off).astype(np.int32), xyz)
    poff, pxyz, pairs, _ = m.Prepare(True, engine=eng)
    lk, _, _ = eng.linking_numbers(pxyz, poff, pairs, "barneshut")
    return eng, poff, pxyz, pairs, lk


@pytest.mark.parametrize("schedule", [0, 1])
def test_spill_bound_reports_stack_overflow(case, schedule):
    eng, poff, pxyz, pairs, lk = case
    with pytest.raises(FlnError) as ex:
        eng.linking_numbers(pxyz, poff, pairs, "barneshut", bh_schedule=schedule, bh_spill_cap=1)
    assert ex.value.status == STACK_OVERFLOW
    assert "stack" in str(ex.value)
    # The context stays usable: the same call at the default bound.
    lk2, _, _ = eng.linking_numbers(pxyz, poff, pairs, "barneshut", bh_schedule=schedule)
    assert np.array_equal(np.rint(lk2), np.rint(lk))


def test_wait_bound_falls_back_to_rounds(case):
    eng, poff, pxyz, pairs, lk = case
    # Fewer pairs than warps: idle warps wait on the ring at once and give up
    # after a few polls; the stage is redone with budgeted rounds.
    assert len(pairs) < 148 * 4
    lk1, err1, fl1 = eng.linking_numbers(pxyz, poff, pairs, "barneshut", bh_schedule=1, bh_wait_polls=2)
    s = eng.stats()
    assert s["bh_wait_timeouts"] >= 1
    assert np.array_equal(np.rint(lk1), np.rint(lk))
    np.testing.assert_allclose(lk1, lk, rtol=0, atol=1e-8)
    # At the default bound the persistent schedule finishes on its own.
    lk2, _, _ = eng.linking_numbers(pxyz, poff, pairs, "barneshut", bh_schedule=1)
    assert eng.stats()["bh_wait_timeouts"] == 0
    assert np.array_equal(np.rint(lk2), np.rint(lk))


def test_bounds_checked(case):
    eng, poff, pxyz, pairs, _ = case
    with pytest.raises(FlnError):
        eng.linking_numbers(pxyz, poff, pairs, "barneshut", bh_spill_cap=-1)
    with pytest.raises(FlnError):
        eng.linking_numbers(pxyz, poff, pairs, "barneshut", bh_wait_polls=-5)
