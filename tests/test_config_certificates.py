"""Full-size certificates of the benchmark workloads, byte for byte.

tests/golden/configs/<name>.txt holds the certificate of the FP64 direct sum
over every potentially linked pair of a seeded workload (the reference's
certificate method, linking_number_certificate.cpp:241-338 rounded as at
:294-322), and <name>.npz every pair's FP64 sum, written by
tests/golden/make_config_certs.py:

  polymer       200 x 50,000-step closed walks (14.0M segments after Discretize)
  held_out_20M  1,000 x 20,000-step closed walks (31.3M segments)
  mixed_batch   5,000 torus knots and walks, 16 to 2^18 segments (139.5M)

The test regenerates each workload, checks that the prepared polylines and
pairs are the ones the fixture was made from (digest), runs the default
Barnes–Hut (mixed precision, beta retry, escalation, margin check), and
requires its certificate to equal the fixture byte for byte, every pair's
integer to equal the FP64 one, and every real sum to lie within the
Barnes–Hut target error (0.1) of the FP64 sum. On the held-out set the
learned opening criterion (trained on other seeds) must give the same
certificate.
"""
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN
from fastlinkingnumbers_b200 import Engine, Model, workloads

pytestmark = pytest.mark.gpu

CONFIGS = ["polymer", "held_out_20M", "mixed_batch"]


def _fixture(name):
    z = np.load(os.path.join(GOLDEN, "configs", name + ".npz"))
    with open(os.path.join(GOLDEN, "configs", name + ".txt")) as f:
        text = f.read()
    return text, z["lk"], json.loads(str(z["meta"]))


@pytest.fixture(scope="module")
def engine():
    return Engine(0)


@pytest.mark.parametrize("name", CONFIGS)
def test_full_size_certificate(engine, name):
    text, lk64, meta = _fixture(name)
    off, xyz, _ = workloads.named(name, meta["seed"])
    m = Model().SetCurves(3, -np.diff(off).astype(np.int32), xyz)
    del xyz
    poff, pxyz, pairs, rounds = m.Prepare(True, engine=engine)
    assert workloads.digest(poff, pxyz, pairs) == meta["digest"], "regenerated workload differs from the fixture's"
    lk, err, flags = engine.linking_numbers(pxyz, poff, pairs, "barneshut")
    s = engine.stats()
    assert workloads.certificate_text(len(poff) - 1, pairs, lk) == text
    r64 = np.sign(lk64) * np.floor(np.abs(lk64) + 0.5)
    r = np.sign(lk) * np.floor(np.abs(lk) + 0.5)
    assert np.array_equal(r, r64), f"{int(np.sum(r != r64))} pairs round differently"
    dev = np.abs(lk - lk64)
    assert dev.max() < 0.1
    print(f"{name}: {len(pairs)} pairs, {meta['nonzero_links']} links, max |BH - FP64| {dev.max():.3g} "
          f"(mean {dev.mean():.3g}), min FP64 margin {meta['min_margin']:.3f}, retried {s['beta_retried']}, "
          f"escalated {s['bh_escalated']}, FP64 recomputed {s['fp64_recomputed']}, {s['ms_kernels']:.1f} ms")
    if name == "held_out_20M":
        from fastlinkingnumbers_b200 import LearnedCriterion
        toff, txyz, tpairs = workloads.walk_pairs(seed=meta["seed"] + 1000)
        model = LearnedCriterion.train(engine, txyz, toff, tpairs)
        engine.set_learned(model)
        try:
            lkl, _, _ = engine.linking_numbers(pxyz, poff, pairs, "barneshut")
        finally:
            engine.set_learned(None)
        assert workloads.certificate_text(len(poff) - 1, pairs, lkl) == text
        assert np.abs(lkl - lk64).max() < 0.1
