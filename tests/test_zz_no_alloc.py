"""The allocation-free direct sum, fln_linking_numbers_direct_noalloc.

Callers that cannot call cudaMalloc (another framework owns the device's
memory pool, a latency-critical loop must not take allocator locks, or an
allocation failure cannot be handled there) use this entry point: it works
in the caller's device buffers plus one fixed array inside libfln.so. This
file is collected last so that a stop at its first failure has already run
every other test; it passes alone in a fresh process as well, because its
first call performs the once-per-device set-up itself.

Checked through the C ABI against fln_linking_numbers_device (the entry point
that allocates) on two calls in a row, with the tolerances of the other
parity tests: 1e-9 for FP64, 1e-5 for the mixed precision.
"""
import ctypes as C

import numpy as np
import pytest

from fastlinkingnumbers_b200 import Engine, Model, workloads
from fastlinkingnumbers_b200 import _native as N

pytestmark = pytest.mark.gpu


def _call(L, d_xyz, d_off, nloops, d_pairs, npairs, prec, d_out, stream=None):
    return L.fln_linking_numbers_direct_noalloc(
        C.c_void_p(d_xyz), C.c_void_p(d_off), nloops, C.c_void_p(d_pairs), npairs, prec,
        C.c_void_p(d_out), C.c_void_p(stream))


@pytest.mark.parametrize("prec,tol", [(N.PREC_FP64, 1e-9), (N.PREC_MIXED, 1e-5)])
def test_noalloc_matches_allocating_entry_point(prec, tol):
    torch = pytest.importorskip("torch")
    L = N.load()
    off, xyz = workloads.chain_mail(rows=12, cols=12, seed=9)
    m = Model().SetCurves(3, -np.diff(off).astype(np.int32), xyz)
    poff, pxyz, pairs, _ = m.Prepare(True)
    d_xyz = torch.from_numpy(pxyz).cuda()
    d_off = torch.from_numpy(poff).cuda()
    d_pairs = torch.from_numpy(pairs).cuda()
    n = len(pairs)
    ref = torch.zeros(n, dtype=torch.float64, device="cuda")
    eng = Engine(0)
    eng.linking_numbers_device(d_xyz.data_ptr(), d_off.data_ptr(), len(poff) - 1, d_pairs.data_ptr(), n,
                               ref.data_ptr(), method="directsum", precision=prec, fp64_margin=0.0)
    torch.cuda.synchronize()
    for _ in range(2):  # the array keeps the previous call's contents
        out = torch.full((n,), float("nan"), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        st = _call(L, d_xyz.data_ptr(), d_off.data_ptr(), len(poff) - 1, d_pairs.data_ptr(), n, prec,
                   out.data_ptr())
        assert st == 0, L.fln_last_error()
        torch.cuda.synchronize()
        np.testing.assert_allclose(out.cpu().numpy(), ref.cpu().numpy(), rtol=0, atol=tol)
    assert np.count_nonzero(np.round(ref.cpu().numpy())) > 0


def test_noalloc_mixed_near_contacts():
    """Dense knots and walks: many segment pairs lie between one and four
    segment lengths apart, where the mixed precision's FP64 rule for near
    terms (near_factor, default 4) decides the result. The allocation-free
    call must use the same factor as the allocating entry point."""
    torch = pytest.importorskip("torch")
    L = N.load()
    off, xyz = workloads.mixed_batch(seed=9, n_loops=40, hi=2 ** 12, cube=20.0)
    m = Model().SetCurves(3, -np.diff(off).astype(np.int32), xyz)
    poff, pxyz, pairs, _ = m.Prepare(True)
    d_xyz = torch.from_numpy(pxyz).cuda()
    d_off = torch.from_numpy(poff).cuda()
    d_pairs = torch.from_numpy(pairs).cuda()
    n, nl = len(pairs), len(poff) - 1
    eng = Engine(0)
    ref = {}
    near = {}
    for name, prec, factor in (("fp64", N.PREC_FP64, 4.0), ("mixed", N.PREC_MIXED, 4.0),
                               ("mixed_f1", N.PREC_MIXED, 1.0)):
        r = torch.zeros(n, dtype=torch.float64, device="cuda")
        eng.linking_numbers_device(d_xyz.data_ptr(), d_off.data_ptr(), nl, d_pairs.data_ptr(), n, r.data_ptr(),
                                   method="directsum", precision=prec, fp64_margin=0.0, near_factor=factor)
        torch.cuda.synchronize()
        ref[name] = r.cpu().numpy()
        near[name] = eng.stats()["near_fp64_terms"]
    # The band between one and four segment lengths is populated.
    assert near["mixed"] > near["mixed_f1"] > 0
    for _ in range(2):
        out = torch.full((n,), float("nan"), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        st = _call(L, d_xyz.data_ptr(), d_off.data_ptr(), nl, d_pairs.data_ptr(), n, N.PREC_MIXED,
                   out.data_ptr())
        assert st == 0, L.fln_last_error()
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        np.testing.assert_allclose(got, ref["mixed"], rtol=0, atol=1e-5)
        np.testing.assert_allclose(got, ref["fp64"], rtol=0, atol=1e-5)
    print(f"near contacts: {n} pairs, FP64 near terms {near['mixed']:.0f} (factor 4) / "
          f"{near['mixed_f1']:.0f} (factor 1), max |no-alloc - FP64| {np.abs(got - ref['fp64']).max():.3g}, "
          f"max |factor 1 - FP64| {np.abs(ref['mixed_f1'] - ref['fp64']).max():.3g}")


def test_noalloc_rejects_oversize_and_bad_input():
    torch = pytest.importorskip("torch")
    L = N.load()
    off, xyz = workloads.ring_chain(seed=2, n_rings=4)
    d_xyz = torch.from_numpy(xyz).cuda()
    d_off = torch.from_numpy(off).cuda()
    out = torch.zeros(70000, dtype=torch.float64, device="cuda")
    big = torch.zeros((70000, 2), dtype=torch.int32, device="cuda")
    st = _call(L, d_xyz.data_ptr(), d_off.data_ptr(), 4, big.data_ptr(), 70000, N.PREC_FP64, out.data_ptr())
    assert st == 1 and b"65536" in L.fln_last_error()
    bad = torch.tensor([[0, 9]], dtype=torch.int32, device="cuda")
    st = _call(L, d_xyz.data_ptr(), d_off.data_ptr(), 4, bad.data_ptr(), 1, N.PREC_FP64, out.data_ptr())
    assert st == 1 and b"out of range" in L.fln_last_error()
    # A valid call right after the rejected ones still works.
    ok = torch.tensor([[0, 1], [1, 2]], dtype=torch.int32, device="cuda")
    st = _call(L, d_xyz.data_ptr(), d_off.data_ptr(), 4, ok.data_ptr(), 2, N.PREC_FP64, out.data_ptr())
    assert st == 0
    torch.cuda.synchronize()
    assert np.allclose(np.abs(out[:2].cpu().numpy()), 1.0, atol=1e-9)
