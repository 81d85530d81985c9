"""The allocation-free binning entry point (pbbfmm_bin_points_noalloc).

It serves callers that cannot call cudaMalloc, e.g. a process whose device
memory is already reserved by another allocator, or a deployment that fixes
its memory footprint at start-up.  Its scratch is one fixed device array in
the library, so the test checks, through the C ABI, that two calls in a row
(different sizes, so the second sees the first one's leftovers) give exactly
the leaf offsets and sort permutation of the binning inside the ordinary
matvec entry point, and that sizes beyond the array's limit are refused.
This file is collected last on purpose."""
import ctypes

import numpy as np
import pytest

import pbbfmm3d_b200 as fmm
from pbbfmm3d_b200 import _lib

pytestmark = pytest.mark.gpu

MAX_POINTS = 524288


def _reference_binning(tree, pts):
    """Leaf offsets and permutation from the existing matvec entry point."""
    n = pts.shape[0]
    out = np.zeros(n)
    fmm.H2_3D_Compute(tree, pts, pts, np.zeros(n), 1, out)
    return tree.debug_copy(2).astype(np.int64), tree.debug_copy(3).astype(np.int64)


def _noalloc(torch, pts, box, level):
    n = pts.shape[0]
    d_pts = torch.tensor(pts, device="cuda")
    d_perm = torch.full((max(n, 1),), -1, dtype=torch.int32, device="cuda")
    d_start = torch.full((8 ** level + 1,), -1, dtype=torch.int32, device="cuda")
    d_ctr = torch.zeros(3, dtype=torch.float64, device="cuda")
    rc = _lib.lib().pbbfmm_bin_points_noalloc(
        ctypes.c_void_p(d_pts.data_ptr()), n, box, level, ctypes.c_void_p(d_perm.data_ptr()),
        ctypes.c_void_p(d_start.data_ptr()), ctypes.c_void_p(d_ctr.data_ptr()), None)
    _lib.check(rc)
    torch.cuda.synchronize()
    return d_start.cpu().numpy().astype(np.int64), d_perm.cpu().numpy()[:n].astype(np.int64), \
        d_ctr.cpu().numpy()


def test_noalloc_binning_matches_matvec_binning_twice():
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(17)
    level, box = 5, 1.0
    tree = fmm.kernel_Laplacian(box, level, 3, 1e-4, 1)
    tree.buildFMMTree()
    for n in (200_000, 50_000):  # second call smaller than the first
        pts = rng.uniform(-0.5, 0.5, (n, 3))
        pts[:n // 2] *= 0.3  # uneven occupancy, many empty leaves
        ref_start, ref_perm = _reference_binning(tree, pts)
        start, perm, ctr = _noalloc(torch, pts, box, level)
        assert np.array_equal(start, ref_start)
        assert np.array_equal(perm, ref_perm)
        lo, hi = pts.min(axis=0), pts.max(axis=0)
        assert np.allclose(ctr, 0.5 * (lo + hi), rtol=0, atol=1e-15)
    tree.close()


def test_noalloc_rejects_sizes_beyond_its_array():
    rc = _lib.lib().pbbfmm_bin_points_noalloc(None, MAX_POINTS + 1, 1.0, 3, None, None, None, None)
    assert rc == _lib.ERR_ARG
    assert b"at most" in _lib.lib().pbbfmm_last_error()


def test_noalloc_largest_size():
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(3)
    level, box = 6, 1.0
    pts = rng.uniform(-0.5, 0.5, (MAX_POINTS, 3))
    start, perm, _ = _noalloc(torch, pts, box, level)
    tree = fmm.kernel_Laplacian(box, level, 3, 1e-4, 1)
    tree.buildFMMTree()
    ref_start, ref_perm = _reference_binning(tree, pts)
    assert np.array_equal(start, ref_start) and np.array_equal(perm, ref_perm)
    tree.close()
