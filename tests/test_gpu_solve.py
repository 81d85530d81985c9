"""Kernel solve (K + lam I) x = b by GMRES with FMM matvecs, and its adjoint
backward (pbbfmm3d_b200.solve).

- The GMRES residual, recomputed with the FMM operator, meets the tolerance.
- Against the exact dense operator the residual is explained by the FMM's
  operator error on x (itself at the approximation level, 1e-4 of K|x|).
- dL/db and dL/d(points) of L = sum(x * g0) match central finite differences
  of the solve (h = 1e-6, solves to 1e-12): agreement to 1e-4 relative, the
  limit set by solver tolerance / h."""
import numpy as np
import pytest

import pbbfmm3d_b200 as fmm
from helpers import make_tree, rel

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
from pbbfmm3d_b200.solve import gmres, gmres_ir, kernel_operator, kernel_solve  # noqa: E402

ELL, LAM = 0.2, 1e-2


def _setup(N=3000, C=2, seed=5):
    rng = np.random.default_rng(seed)
    P = rng.uniform(-0.5, 0.5, (N, 3))
    b = rng.standard_normal((C, N))
    t = make_tree("ExpCov", ELL, 1.0, 4, 5, 1e-5, 0)
    t.buildFMMTree()
    return t, P, b


def _dense(P):
    d = np.sqrt(((P[:, None, :] - P[None, :, :]) ** 2).sum(-1))
    return np.exp(-d / ELL)


def test_gmres_converges():
    t, P, b = _setup()
    Pt = torch.tensor(P, device="cuda")
    bt = torch.tensor(b, device="cuda")
    x, info = gmres(kernel_operator(t, Pt, LAM), bt, tol=1e-8, restart=60, maxiter=3000)
    assert info["converged"], info
    assert np.all(info["rel_residual"] < 1e-8)
    # With the exact dense operator the residual is the FMM's operator error
    # on x (amplified by the conditioning: lam = 1e-2 makes ||x|| >> ||b||):
    # b - A x = (b - A_fmm x) + (K_fmm - K) x.
    K = _dense(P)
    xs = x.cpu().numpy()
    kx = xs @ K.T
    kx_fmm = (kernel_operator(t, Pt, 0.0)(x)).cpu().numpy()
    # the FMM's approximation level, against the cancellation-free scale K|x|
    # (x carries large components that cancel in K x: lam = 1e-2)
    assert np.linalg.norm(kx_fmm - kx) < 1e-4 * np.linalg.norm(np.abs(xs) @ K.T)
    r = b - (kx + LAM * xs)
    assert np.linalg.norm(r) <= 1.01 * np.linalg.norm(kx_fmm - kx) + 1e-7 * np.linalg.norm(b)


def test_mixed_precision_solve_converges():
    t, P, b = _setup(seed=6)
    Pt = torch.tensor(P, device="cuda")
    bt = torch.tensor(b, device="cuda")
    # plain GMRES on the mixed operator stalls above 1e-6 (rounding floor
    # near eps * ||K|x||| with ||x|| >> ||b||); float64 iterative refinement
    # reaches the float64 residual
    _, plain = gmres(kernel_operator(t, Pt, LAM, fmm.PREC_MIXED), bt, tol=1e-8, restart=60,
                     maxiter=1500)
    x, info = gmres_ir(kernel_operator(t, Pt, LAM, fmm.PREC_MIXED), kernel_operator(t, Pt, LAM),
                       bt, tol=1e-8, inner_tol=1e-3, restart=60, maxiter=3000)
    assert info["converged"], info
    r64 = bt - kernel_operator(t, Pt, LAM)(x)
    assert float(torch.linalg.norm(r64) / torch.linalg.norm(bt)) < 1e-8
    assert not plain["converged"]
    # and the differentiable entry uses it
    x2 = kernel_solve(t, Pt, bt, LAM, tol=1e-8, precision=fmm.PREC_MIXED, restart=60,
                      maxiter=3000)
    r2 = bt - kernel_operator(t, Pt, LAM)(x2)
    assert float(torch.linalg.norm(r2) / torch.linalg.norm(bt)) < 1e-8


def test_solve_gradients_match_finite_differences():
    t, P, b = _setup(N=2000, C=2, seed=7)
    rng = np.random.default_rng(8)
    g0 = rng.standard_normal(b.shape)
    G0 = torch.tensor(g0, device="cuda")
    kw = dict(tol=1e-12, restart=80, maxiter=6000)
    Pt = torch.tensor(P, device="cuda", requires_grad=True)
    bt = torch.tensor(b, device="cuda", requires_grad=True)
    x = kernel_solve(t, Pt, bt, LAM, **kw)
    (x * G0).sum().backward()
    gP, gb = Pt.grad.cpu().numpy(), bt.grad.cpu().numpy()

    def loss(Pm, bm):
        xm = kernel_solve(t, torch.tensor(Pm, device="cuda"), torch.tensor(bm, device="cuda"),
                          LAM, **kw)
        return float((xm * G0).sum().item())

    h = 1e-6
    fd, an = [], []
    for c, i in ((0, 11), (1, 500)):
        bp, bm = b.copy(), b.copy()
        bp[c, i] += h
        bm[c, i] -= h
        fd.append((loss(P, bp) - loss(P, bm)) / (2 * h))
        an.append(gb[c, i])
    # point coordinates: not a bounding-box extreme, not near a leaf boundary
    ctr = 0.5 * (P.min(0) + P.max(0))
    w = 1.0 / 16
    ext = set(np.argmin(P, 0)) | set(np.argmax(P, 0))
    picked = 0
    for i in rng.permutation(len(P)):
        if i in ext:
            continue
        d = int(rng.integers(3))
        u = (P[i, d] - (ctr[d] - 0.5)) / w
        if min(u - np.floor(u), np.ceil(u) - u) < 1e-3:
            continue
        Pp, Pm = P.copy(), P.copy()
        Pp[i, d] += h
        Pm[i, d] -= h
        fd.append((loss(Pp, b) - loss(Pm, b)) / (2 * h))
        an.append(gP[i, d])
        picked += 1
        if picked == 6:
            break
    fd, an = np.array(fd), np.array(an)
    assert rel(an, fd) < 1e-4, np.c_[an, fd]
