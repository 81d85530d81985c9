"""FP64 parity at the interpolation orders and shapes the benchmark workloads
run, through the C-ABI.

Part 1 -- the order-templated passes (P2M, M2M, the pre/post transforms, M2L,
L2L, L2P + P2P) at Chebyshev orders 5, 6 and 7 and uniform order 5 with 8
columns, against the oracle phase by phase: leaf binning bit-exact, moments S
and locals F at every level and the output within 1e-12 (F 1e-11), with the
same operators fed to both.  Reference passes: include/compute.hpp:287-333
(P2M), :957-1034 (M2M), :373-396 and :464-508 (Chebyshev M2L), :337-372 and
:930-943 (uniform M2L), :799-878 (L2L), :594-737 (L2P, P2P).

Part 2 -- the reference itself, run live (oracle/_ref, one thread, so that
its upward pass is deterministic), on the shapes of the benchmark workloads
at reduced N; the GPU tree is given the operator files the reference wrote
(so the comparison isolates the matvec from SVD differences) and must match
the reference's output within 1e-12 in float64.  The mixed path is held to
the float64 path's 2e-6 bound against the same reference output.
"""
import numpy as np
import pytest

import oracle
import pbbfmm3d_b200 as fmm
from helpers import make_tree, rel
from test_gpu_parity import _meta, phase_by_phase

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _clustered(rng, n, blobs=64, sigma=0.02, half=0.5):
    """90 % of the points in Gaussian blobs (centres uniform in the middle
    80 % of the cube), 10 % uniform, clipped to the cube [-half, half]^3:
    the clustered benchmark workload's distribution, centred on 0."""
    nb = int(0.9 * n)
    ctr = rng.uniform(-0.8 * half, 0.8 * half, (blobs, 3))
    p = ctr[rng.integers(0, blobs, nb)] + sigma * rng.standard_normal((nb, 3))
    p = np.clip(p, -half, half)
    return np.vstack([p, rng.uniform(-half, half, (n - nb, 3))])


HIGH_ORDERS = [
    # meta, clustered points
    (_meta("Laplacian", 0.0, 1.0, 4, 5, 1e-7, 1, 1), False),
    (_meta("Laplacian", 0.0, 1.0, 4, 6, 1e-7, 1, 1), False),
    (_meta("Laplacian", 0.0, 1.0, 5, 6, 1e-7, 1, 1), True),
    (_meta("Laplacian", 0.0, 1.0, 4, 7, 1e-7, 1, 1), False),
    (_meta("GaussSigma", 0.1, 1.0, 4, 5, 1e-6, 1, 4), False),
    (_meta("ExpCov", 0.3, 1.0, 5, 5, 1e-5, 0, 8), False),
]


@pytest.mark.parametrize("case", HIGH_ORDERS,
                         ids=["%s%s%d_L%d_C%d%s" % (m["kernel"], "C" if m["cheb"] else "U",
                                                    m["order"], m["level"], m["ncols"],
                                                    "_clustered" if c else "")
                              for m, c in HIGH_ORDERS])
def test_gpu_matches_oracle_high_orders(case):
    meta, clustered = case
    rng = np.random.default_rng(101)
    N = 6000
    p = _clustered(rng, N) if clustered else rng.uniform(-0.5, 0.5, (N, 3))
    w = rng.standard_normal(N * meta["ncols"])
    phase_by_phase(meta, p, w)


def _gpu_with_reference_ops(meta, ops):
    t = make_tree(meta["kernel"], meta["param"], meta["box"], meta["level"], meta["order"],
                  meta["eps"], meta["cheb"])
    t.set_operators(ops["K"], ops["U"], ops["VT"], rf=ops["rf"], rs=ops["rs"])
    return t


def _reference(meta, points, weight):
    out, _, wd = oracle.run_reference(meta["kernel"], meta["param"], meta["box"], meta["level"],
                                      meta["order"], meta["eps"], meta["cheb"], points, weight,
                                      meta["ncols"], threads=1)
    _, hom = oracle.KERNELS[meta["kernel"]]
    ops = oracle.read_reference_cache(wd + "/output",
                                      oracle.kernel_type_name(meta["kernel"], meta["param"]),
                                      meta["order"], meta["cheb"], meta["level"], abs(hom) > 0.1)
    return out, ops


def _both_precisions(t, target, source, w, C, ref):
    out = np.zeros(target.shape[0] * C)
    fmm.H2_3D_Compute(t, target, source, w, C, out)
    e64 = rel(out, ref)
    t.set_precision(fmm.PREC_MIXED)
    out32 = np.zeros(target.shape[0] * C)
    fmm.H2_3D_Compute(t, target, source, w, C, out32)
    e32 = rel(out32, ref)
    t.close()
    return e64, e32


def test_reference_live_laplacian_config1_shape():
    """Laplacian 1/r, N = 20,000 uniform in the unit cube, weights U[-1, 1],
    one column, L = 4, Chebyshev n = 4, eps 1e-5: the small CPU workload at
    its exact shape."""
    rng = np.random.default_rng(2025)
    N = 20000
    p = rng.uniform(-0.5, 0.5, (N, 3))
    w = rng.uniform(-1, 1, N)
    meta = _meta("Laplacian", 0.0, 1.0, 4, 4, 1e-5, 1, 1)
    ref, ops = _reference(meta, p, w)
    e64, e32 = _both_precisions(_gpu_with_reference_ops(meta, ops), p, p, w, 1, ref)
    assert e64 < TOL, e64
    assert e32 < 2e-6, e32


def test_reference_live_clustered_laplacian_cheb6():
    """The clustered Laplacian workload's shape at 1/200 of its size: 20,000
    points, 90 % in 64 Gaussian blobs of sigma 0.02, weights U[-1, 1],
    Chebyshev n = 6, eps 1e-7, L = 5."""
    rng = np.random.default_rng(2026)
    N = 20000
    p = _clustered(rng, N)
    w = rng.uniform(-1, 1, N)
    meta = _meta("Laplacian", 0.0, 1.0, 5, 6, 1e-7, 1, 1)
    ref, ops = _reference(meta, p, w)
    e64, e32 = _both_precisions(_gpu_with_reference_ops(meta, ops), p, p, w, 1, ref)
    assert e64 < TOL, e64
    assert e32 < 2e-6, e32


def test_reference_live_gaussian_sources_differ_from_targets():
    """The differentiation workload's shape: Gaussian exp(-r^2 / (2 0.1^2)),
    10,000 targets and a separate 10,000 sources uniform in the unit cube,
    4 columns N(0, 1), Chebyshev n = 5, L = 4.  The reference bins its
    targets only, so it runs on S u T with zero weights on T (the union
    trick); two targets sit on the corners of bbox(S u T) so that both
    programs recentre on the same box."""
    rng = np.random.default_rng(2027)
    Nf, Ns, C = 10000, 10000, 4
    tg = rng.uniform(-0.5, 0.5, (Nf, 3))
    sr = rng.uniform(-0.5, 0.5, (Ns, 3))
    x = np.concatenate([tg, sr])
    tg[0], tg[1] = x.min(axis=0), x.max(axis=0)
    w = rng.standard_normal(Ns * C)
    meta = _meta("GaussSigma", 0.1, 1.0, 4, 5, 1e-6, 1, C)
    wu = np.zeros((C, Nf + Ns))
    wu[:, Nf:] = w.reshape(C, Ns)
    refu, ops = _reference(meta, np.concatenate([tg, sr]), wu.ravel())
    ref = refu.reshape(C, Nf + Ns)[:, :Nf].ravel()
    e64, e32 = _both_precisions(_gpu_with_reference_ops(meta, ops), tg, sr, w, C, ref)
    assert e64 < TOL, e64
    assert e32 < 2e-6, e32
