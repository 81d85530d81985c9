"""The CPU oracle (oracle/fmm_oracle.c) pinned against the golden vectors the
unmodified reference produced (tests/golden/make_golden.py).  CPU only."""
import numpy as np
import pytest

import oracle
from helpers import case_ops, golden_names, host_ops, load_case, oracle_ops, rel


@pytest.mark.parametrize("name", golden_names())
def test_oracle_matches_reference_golden(name):
    case = load_case(name)
    meta = case["meta"]
    ops = case_ops(case)
    exact = True
    if ops is None:
        # uniform operators have no SVD ambiguity: our precompute reproduces
        # the reference's to rounding; Chebyshev without stored operators can
        # only agree to the truncation level (degenerate singular values)
        ops = host_ops(meta["kernel"], meta["param"], meta["box"], meta["level"], meta["order"],
                       meta["eps"], meta["cheb"])
        exact = not meta["cheb"]
    out = oracle.matvec(oracle_ops(ops, meta), case["target"], case["source"], case["weight"],
                        meta["ncols"])
    err = rel(out, case["output"])
    assert err < (1e-12 if exact else 1e-4), (name, err)


def test_oracle_direct_sum_against_numpy():
    rng = np.random.default_rng(3)
    t = rng.uniform(-0.5, 0.5, (300, 3))
    s = rng.uniform(-0.5, 0.5, (400, 3))
    w = rng.standard_normal(800)
    d = t[:, None, :] - s[None, :, :]
    r = np.sqrt((d ** 2).sum(-1))
    K = np.exp(-r / 0.3)
    ref = (K @ w.reshape(2, 400).T).T.ravel()
    got = oracle.direct("ExpCov", [0.3], t, s, w, 2)
    assert rel(got, ref) < 1e-14


def test_oracle_fixture_accuracy_vs_direct_sum():
    """The reference's own 5000-point fixture: FMM error vs the FP64 direct
    sum is the reference's (2.06e-5, include/test.hpp:19-47 protocol)."""
    case = load_case("ref_fixture_lap_cheb4")
    d = oracle.direct("Laplacian", [0.0], case["target"], case["target"], case["weight"], 1)
    assert abs(rel(case["output"], d) - 2.065e-5) < 1e-7
