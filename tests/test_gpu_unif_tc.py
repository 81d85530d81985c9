"""The frequency-domain M2L of the mixed uniform path on the tensor cores
(csrc/m2l_unif_tc.cu: tcgen05 kind::f16 on power-of-two scaled F16 hi / lo
splits of both operands, float32 accumulation), through the C-ABI, against
the CUDA-core float32 kernel it replaces and against the float64 path.

It runs at levels with at least 16 parents per side and for column groups of
8; other levels and column counts stay on the CUDA cores.  Tolerances: the
locals F of every level and the output within 2e-6 of the CUDA-core float32
kernel, and the output within 2e-6 of float64 (the mixed path's bound
everywhere)."""
import numpy as np
import pytest

import pbbfmm3d_b200 as fmm
from helpers import make_tree, rel

pytestmark = pytest.mark.gpu


def _clustered(rng, n, blobs=16, sigma=0.03):
    nb = int(0.9 * n)
    ctr = rng.uniform(-0.4, 0.4, (blobs, 3))
    p = ctr[rng.integers(0, blobs, nb)] + sigma * rng.standard_normal((nb, 3))
    return np.vstack([np.clip(p, -0.5, 0.5), rng.uniform(-0.5, 0.5, (n - nb, 3))])


def _run(t, p, w, C, precision, tc=True):
    t.set_precision(precision)
    t.set_tensor_cores(tc)
    out = np.zeros(p.shape[0] * C)
    fmm.H2_3D_Compute(t, p, p, w, C, out)
    return out


CASES = [
    # kernel, param, level, order, C, clustered
    ("ExpCov", 0.3, 6, 5, 8, False),     # the headline workload's shape at 1/5 of its size
    ("ExpCov", 0.3, 6, 5, 8, True),      # empty cells and empty source lines
    ("ExpCov", 0.3, 5, 4, 16, False),    # two column groups
    ("OneOverR2", 0.0, 5, 4, 8, False),  # homogeneous: one operator set
    ("Laplacian", 0.0, 5, 3, 24, True),  # three column groups, order 3
]


@pytest.mark.parametrize("case", CASES, ids=["%s_L%d_n%d_C%d%s" % (c[0], c[2], c[3], c[4],
                                                                    "_clustered" if c[5] else "")
                                             for c in CASES])
def test_unif_tensor_core_mac_matches_cuda_cores(case):
    kernel, param, level, order, C, clustered = case
    rng = np.random.default_rng(55)
    N = 200000 if level == 6 else 40000
    p = _clustered(rng, N) if clustered else rng.uniform(-0.5, 0.5, (N, 3))
    w = rng.standard_normal(N * C)
    t = make_tree(kernel, param, 1.0, level, order, 1e-6, 0)
    t.buildFMMTree()
    t.set_timing(True)
    o64 = _run(t, p, w, C, fmm.PREC_FP64)
    o_cc = _run(t, p, w, C, fmm.PREC_MIXED, tc=False)
    F_cc = {l: t.debug_copy(1, l) for l in range(2, level + 1)}
    t.reset_kernel_times()
    o_tc = _run(t, p, w, C, fmm.PREC_MIXED, tc=True)
    assert t.kernel_times()["m2l_mac"][1] > 0
    cnt = np.diff(t.debug_copy(2).astype(np.int64))
    n3 = order ** 3
    for l in range(5, level + 1):
        occ = cnt.reshape(-1, 8 ** (level - l)).sum(1) > 0
        F = t.debug_copy(1, l).reshape(-1, C * n3)[occ]
        Fr = F_cc[l].reshape(-1, C * n3)[occ]
        assert rel(F, Fr) < 2e-6, (l, rel(F, Fr))
    # both float32-accurate; the tensor pipe's float32 accumulation (about
    # 100 steps per accumulator and frequency) adds a little: measured 1.1e-6
    # against 4.4e-7 for the CUDA cores (clustered), 6.0e-7 against 1.8e-7
    e_tc, e_cc = rel(o_tc, o64), rel(o_cc, o64)
    assert rel(o_tc, o_cc) < 2e-6, rel(o_tc, o_cc)
    assert e_tc < 2e-6, (e_tc, e_cc)
    t.close()


def test_unif_tensor_core_mac_not_used_for_other_column_counts():
    """Columns not in groups of 8 stay on the CUDA cores: bit-identical to
    the tensor cores switched off."""
    rng = np.random.default_rng(56)
    N, C = 40000, 4
    p = rng.uniform(-0.5, 0.5, (N, 3))
    w = rng.standard_normal(N * C)
    t = make_tree("ExpCov", 0.3, 1.0, 5, 4, 1e-6, 0)
    t.buildFMMTree()
    a = _run(t, p, w, C, fmm.PREC_MIXED, tc=True)
    b = _run(t, p, w, C, fmm.PREC_MIXED, tc=False)
    assert np.array_equal(a, b)
    t.close()


def test_unif_tensor_core_scale_invariance():
    """The operand scales are powers of two taken from the spectra's maxima:
    weights scaled by 2^60 and 2^-60 scale the result by exactly that."""
    rng = np.random.default_rng(57)
    N, C = 40000, 8
    p = rng.uniform(-0.5, 0.5, (N, 3))
    w = rng.standard_normal(N * C)
    t = make_tree("ExpCov", 0.3, 1.0, 5, 4, 1e-6, 0)
    t.buildFMMTree()
    o = _run(t, p, w, C, fmm.PREC_MIXED)
    for s in (2.0 ** 60, 2.0 ** -60):
        assert rel(_run(t, p, w * s, C, fmm.PREC_MIXED), o * s) < 1e-12
    t.close()


def test_unif_tensor_core_columns_of_any_magnitude():
    """Each column (mod 8) has its own spectra scale: columns whose weights
    differ by 2^-40 .. 2^30 each keep float32 accuracy on their own."""
    rng = np.random.default_rng(59)
    N, C = 60000, 8
    p = rng.uniform(-0.5, 0.5, (N, 3))
    w = rng.standard_normal((C, N))
    w *= np.exp2(10.0 * (np.arange(C) - 4))[:, None]
    w = w.ravel()
    t = make_tree("ExpCov", 0.3, 1.0, 5, 4, 1e-6, 0)
    t.buildFMMTree()
    o64 = _run(t, p, w, C, fmm.PREC_FP64).reshape(C, N)
    o_tc = _run(t, p, w, C, fmm.PREC_MIXED, tc=True).reshape(C, N)
    for c in range(C):
        assert rel(o_tc[c], o64[c]) < 2e-6, (c, rel(o_tc[c], o64[c]))
    t.close()


def test_unif_tensor_core_timeout_reports_and_recovers():
    """With the pipeline waits limited to one poll the kernel stops, drains
    what it issued and reports PBBFMM_ERR_TIMEOUT; the output is untouched
    and the next compute, with the limit restored, is correct."""
    lib = fmm._lib.lib()
    rng = np.random.default_rng(58)
    N, C = 60000, 8
    p = rng.uniform(-0.5, 0.5, (N, 3))
    w = rng.standard_normal(N * C)
    t = make_tree("ExpCov", 0.3, 1.0, 5, 4, 1e-6, 0)
    t.buildFMMTree()
    ref = _run(t, p, w, C, fmm.PREC_MIXED, tc=False)
    t.set_tensor_cores(True)
    out = np.full(N * C, 3.0)
    assert lib.pbbfmm_debug_set_pipeline_wait_limit(0, 1) == fmm._lib.OK
    try:
        with pytest.raises(fmm.FMMError) as ei:
            fmm.H2_3D_Compute(t, p, p, w, C, out)
        assert ei.value.code == fmm._lib.ERR_TIMEOUT
    finally:
        assert lib.pbbfmm_debug_set_pipeline_wait_limit(0, 0) == fmm._lib.OK
    assert np.all(out == 3.0)
    assert rel(_run(t, p, w, C, fmm.PREC_MIXED), ref) < 1e-6
    t.close()
