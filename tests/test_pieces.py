"""Pinned host vertices of a Barnes–Hut call go to the device in pieces on a
copy stream (split at loop boundaries), and the tree build of each piece's
loops waits only for its own piece (capi.cpp: copy_xyz_pieces; bh.cu: the
grouped tree build). The tree records, and so every sum, must be those of the
same call on device arrays, bit for bit."""
import numpy as np
import pytest

from fastlinkingnumbers_b200 import Engine, workloads

pytestmark = pytest.mark.gpu


def test_pinned_vertices_in_pieces_match_device_arrays():
    torch = pytest.importorskip("torch")
    eng = Engine(0)
    off, xyz, pairs = workloads.walk_pairs(seed=21, n_pairs=16, n_steps=100_000)
    assert xyz.nbytes >= 64 << 20 and len(off) - 1 >= 8  # large enough to go in pieces
    h_xyz = torch.from_numpy(np.ascontiguousarray(xyz)).pin_memory().numpy()
    lk_h, err_h, fl_h = eng.linking_numbers(h_xyz, off, pairs, "barneshut")
    d_xyz = torch.from_numpy(np.ascontiguousarray(xyz)).cuda()
    d_off = torch.from_numpy(off).cuda()
    d_pairs = torch.from_numpy(pairs).cuda()
    n = len(pairs)
    d_lk = torch.zeros(n, dtype=torch.float64, device="cuda")
    d_err = torch.zeros(n, dtype=torch.float64, device="cuda")
    d_fl = torch.zeros(n, dtype=torch.int32, device="cuda")
    eng.linking_numbers_device(d_xyz.data_ptr(), d_off.data_ptr(), len(off) - 1, d_pairs.data_ptr(), n,
                               d_lk.data_ptr(), d_err.data_ptr(), d_fl.data_ptr(), method="barneshut")
    torch.cuda.synchronize()
    assert np.array_equal(lk_h, d_lk.cpu().numpy())
    assert np.array_equal(err_h, d_err.cpu().numpy())
    assert np.array_equal(fl_h, d_fl.cpu().numpy())
    # A second call reuses the copy stream and the piece events.
    lk_h2, _, _ = eng.linking_numbers(h_xyz, off, pairs, "barneshut")
    assert np.array_equal(lk_h2, lk_h)
