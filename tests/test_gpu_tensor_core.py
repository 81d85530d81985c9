"""The Chebyshev M2L of the mixed path on the tensor cores (tcgen05, split
hi + lo operands with three products, float32 accumulation) in both operand
formats -- power-of-two scaled F16 (the default) and TF32 -- against the
float64 path and against the CUDA-core float32 kernel, through the C-ABI.

Tolerance: 2e-6 relative L2 against float64 -- the bound the mixed path
keeps everywhere (test_gpu_parity); the split products carry ~2^-21 relative
error each, and the TMEM accumulators are drained every offset (F16) or
every few offsets (TF32), into a running sum kept in registers (r_f <= 128),
in TMEM (r_f <= 160) or in the output."""
import numpy as np
import pytest

import oracle
import pbbfmm3d_b200 as fmm
from helpers import make_tree, rel

pytestmark = pytest.mark.gpu


def _tree(kernel, param, level, order, eps):
    t = make_tree(kernel, param, 1.0, level, order, eps, 1)
    t.buildFMMTree()
    return t


FORMATS = ("f16", "tf32")


def _run(t, p, w, ncols, precision, tc=True, fmt="f16"):
    t.set_precision(precision)
    t.set_tensor_cores(tc, fmt)
    out = np.zeros(p.shape[0] * ncols)
    fmm.H2_3D_Compute(t, p, p, w, ncols, out)
    return out


def _clustered(rng, n, blobs=16, sigma=0.03):
    """90% of the points in Gaussian blobs, 10% uniform, clipped to the cube."""
    nb = int(0.9 * n)
    ctr = rng.uniform(-0.4, 0.4, (blobs, 3))
    p = ctr[rng.integers(0, blobs, nb)] + sigma * rng.standard_normal((nb, 3))
    p = np.clip(p, -0.5, 0.5)
    return np.vstack([p, rng.uniform(-0.5, 0.5, (n - nb, 3))])


CASES = [
    # kernel, param, level, order, eps, ncols, clustered
    ("Laplacian", 0.0, 4, 5, 1e-7, 1, False),
    ("Laplacian", 0.0, 5, 6, 1e-7, 1, True),     # config-3 shape at 1/40 the size
    ("GaussSigma", 0.1, 4, 4, 1e-6, 2, False),   # one operator set per level
    ("OneOverR2", 0.0, 4, 4, 1e-5, 3, True),     # 42 targets x 3 columns per tile
    ("Laplacian", 0.0, 3, 4, 1e-5, 64, False),   # two targets per tile
    ("Laplacian", 0.0, 3, 7, 1e-9, 1, False),    # r_f near 256: two stages, N up to 256
    ("Laplacian", 0.0, 3, 6, 1e-8, 1, False),    # r_f 150: running sum in TMEM
    ("Laplacian", 0.0, 3, 7, 1e-7, 1, False),    # n^3 = 343: post-transform as two MMAs
]


@pytest.mark.parametrize("fmt", FORMATS)
@pytest.mark.parametrize("case", CASES, ids=[f"{c[0]}n{c[3]}C{c[5]}" for c in CASES])
def test_tensor_core_m2l_matches_fp64(case, fmt):
    kernel, param, level, order, eps, C, clustered = case
    rng = np.random.default_rng(31)
    N = 40000 if C < 8 else 3000
    p = _clustered(rng, N) if clustered else rng.uniform(-0.5, 0.5, (N, 3))
    w = rng.uniform(-1, 1, N * C)
    t = _tree(kernel, param, level, order, eps)
    o64 = _run(t, p, w, C, fmm.PREC_FP64)
    o_tc = _run(t, p, w, C, fmm.PREC_MIXED, tc=True, fmt=fmt)
    on_tc = t.get_operators()["rf"] <= 256
    assert t.tensor_core_m2l() == on_tc
    assert t.tensor_core_format() == (fmt if on_tc else None)
    o_cc = _run(t, p, w, C, fmm.PREC_MIXED, tc=False)
    assert rel(o_tc, o64) < 2e-6, rel(o_tc, o64)
    assert rel(o_cc, o64) < 2e-6
    assert rel(o_tc, o_cc) < 2e-6


@pytest.mark.parametrize("fmt", FORMATS)
def test_tensor_core_locals_every_level(fmt):
    """Locals F after the far field and L2L, level by level, mixed (tensor
    cores) against float64."""
    rng = np.random.default_rng(8)
    N, C, level, n = 30000, 2, 4, 5
    p = rng.uniform(-0.5, 0.5, (N, 3))
    w = rng.standard_normal(N * C)
    t = _tree("Laplacian", 0.0, level, n, 1e-7)
    _run(t, p, w, C, fmm.PREC_FP64)
    F64 = {l: t.debug_copy(1, l) for l in range(2, level + 1)}
    _run(t, p, w, C, fmm.PREC_MIXED, tc=True, fmt=fmt)
    cnt = np.diff(t.debug_copy(2).astype(np.int64))  # points per leaf
    n3 = n ** 3
    for l in range(2, level + 1):
        occ = cnt.reshape(-1, 8 ** (level - l)).sum(1) > 0  # cells with targets
        F = t.debug_copy(1, l).reshape(-1, C * n3)[occ]
        Fr = F64[l].reshape(-1, C * n3)[occ]
        assert rel(F, Fr) < 2e-6, (l, rel(F, Fr))


def test_tensor_core_accuracy_against_direct_sum():
    """Clustered Laplacian, Chebyshev n=6, eps 1e-7: the mixed result is as
    close to the float64 direct sum as the float64 FMM is."""
    rng = np.random.default_rng(77)
    N = 100000
    p = _clustered(rng, N, blobs=64, sigma=0.02)
    w = rng.uniform(-1, 1, N)
    t = _tree("Laplacian", 0.0, 5, 6, 1e-7)
    o64 = _run(t, p, w, 1, fmm.PREC_FP64)
    o_tc = _run(t, p, w, 1, fmm.PREC_MIXED)
    rows = rng.choice(N, 1024, replace=False)
    d = oracle.direct("Laplacian", [0.0], p, p, w, 1, rows=rows)
    e64, etc = rel(o64[rows], d), rel(o_tc[rows], d)
    assert etc < 1.05 * e64 + 1e-6, (etc, e64)


@pytest.mark.parametrize("fmt", FORMATS)
def test_tensor_core_scale_invariance(fmt):
    """Weights scaled by 2^60 or 2^-60 scale the mixed result by exactly that
    factor: the F16 operands carry a power-of-two scale per proxy row and per
    operator (unscaled, 2^-60 x O(1) lies below the smallest F16 subnormal
    and 2^60 above the largest F16), and every float32 step scales exactly."""
    rng = np.random.default_rng(12)
    N = 20000
    p = _clustered(rng, N)
    w = rng.uniform(-1, 1, N)
    t = _tree("Laplacian", 0.0, 4, 5, 1e-7)
    o = _run(t, p, w, 1, fmm.PREC_MIXED, fmt=fmt)
    assert t.tensor_core_format() == fmt
    for s in (2.0 ** 60, 2.0 ** -60):
        os_ = _run(t, p, w * s, 1, fmm.PREC_MIXED, fmt=fmt)
        assert rel(os_, o * s) < 1e-12, (s, rel(os_, o * s))


def test_tensor_core_kernel_times_and_switch():
    rng = np.random.default_rng(3)
    p = rng.uniform(-0.5, 0.5, (5000, 3))
    w = rng.standard_normal(5000)
    t = _tree("Laplacian", 0.0, 3, 4, 1e-5)
    t.set_timing(True)
    t.reset_kernel_times()
    _run(t, p, w, 1, fmm.PREC_MIXED, tc=True)
    kt = t.kernel_times()
    assert kt["m2l_split"][1] > 0 and kt["m2l"][1] > 0
    t.reset_kernel_times()
    _run(t, p, w, 1, fmm.PREC_MIXED, tc=False)
    kt = t.kernel_times()
    assert kt["m2l_split"][1] == 0 and kt["m2l"][1] > 0
    t.set_tensor_cores(True)
    assert t.tensor_core_m2l() and t.tensor_core_format() == "f16"
    t.set_tensor_cores(True, "tf32")
    assert t.tensor_core_format() == "tf32"
    t.set_tensor_cores(False)
    assert not t.tensor_core_m2l() and t.tensor_core_format() is None
    with pytest.raises(ValueError):
        t.set_tensor_cores(True, "bf16")
    # the C-ABI refuses unknown modes
    assert fmm._lib.lib().pbbfmm_set_tensor_cores(t._h, 7) == fmm._lib.ERR_ARG


@pytest.mark.parametrize("kernel,param", [("Laplacian", 0.0), ("GaussSigma", 0.1)])
def test_tensor_core_extreme_scales(kernel, param):
    """Weights near 2^-110 (about 8e-34): proxy rows then carry exponents near
    125 and, for the Gaussian, the coarse levels' operators near 30, so that
    e_row + e_op passes the float exponent range, and the pre/post transforms'
    column exponents pass 126.  Every unscaling is applied as exact powers of
    two, so the result scales by 2^-110 up to the float32 subnormal rounding
    of terms far below the result (measured 6e-9; a mis-scaled factor shows
    as 2e-6 or more)."""
    rng = np.random.default_rng(19)
    N = 20000
    p = _clustered(rng, N)
    w = rng.uniform(-1, 1, N)
    t = _tree(kernel, param, 4, 4, 1e-6)
    o = _run(t, p, w, 1, fmm.PREC_MIXED, fmt="f16")
    assert t.tensor_core_format() == "f16"
    s = 2.0 ** -110
    os_ = _run(t, p, w * s, 1, fmm.PREC_MIXED, fmt="f16")
    assert rel(os_, o * s) < 1e-7, rel(os_, o * s)


def test_tensor_core_timeout_reports_and_recovers():
    """The bounded-wait path.  With the M2L pipeline waits limited to one
    poll they run out; each CTA stops, waits with the full bound for the
    copies and MMAs it has already issued, frees its TMEM and sets the
    timeout flag.  The host entry returns PBBFMM_ERR_TIMEOUT and leaves the
    caller's output untouched; once the limit is restored the next compute
    is correct again."""
    lib = fmm._lib.lib()
    rng = np.random.default_rng(23)
    N = 60000
    p = _clustered(rng, N)
    w = rng.uniform(-1, 1, N)
    t = _tree("Laplacian", 0.0, 5, 5, 1e-7)
    o64 = _run(t, p, w, 1, fmm.PREC_FP64)
    t.set_precision(fmm.PREC_MIXED)
    t.set_tensor_cores(True, "f16")
    out = np.full(N, 7.0)
    assert lib.pbbfmm_debug_set_pipeline_wait_limit(0, 1) == fmm._lib.OK
    try:
        with pytest.raises(fmm.FMMError) as ei:
            fmm.H2_3D_Compute(t, p, p, w, 1, out)
        assert ei.value.code == fmm._lib.ERR_TIMEOUT
    finally:
        assert lib.pbbfmm_debug_set_pipeline_wait_limit(0, 0) == fmm._lib.OK
    assert np.all(out == 7.0)
    o = _run(t, p, w, 1, fmm.PREC_MIXED, fmt="f16")
    assert rel(o, o64) < 2e-6, rel(o, o64)
