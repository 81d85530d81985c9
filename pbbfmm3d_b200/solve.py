"""Kernel solves with FMM matvecs on the GPU.

``gmres`` solves (K + lam I) x = b for several right-hand sides at once by
restarted GMRES: one Arnoldi process per column, every step's matvec shared
by all columns (one FMM call with nCols columns).  It restates the
reference's driver app/gmres.cpp:44-64 with app/fmm.hpp:66-86 as its
operator.  The tree stays resident across iterations; the reference
rebuilds it on every matvec.

``KernelSolve`` is a torch.autograd.Function around it.  Its backward is
the adjoint solve (K + lam I)^T mu = dL/dx, then dL/db = mu and
dL/d(points) = -(d/d points) [mu^T K x], the latter from the adjoint FMM
(pbbfmm_compute_adjoint_device: grad_target + grad_source with g = mu, w = x).
"""
from __future__ import annotations

from typing import Callable, Optional

import numpy as np
import torch

from . import PREC_FP64, H2_3D_Tree, compute_adjoint_device, compute_device


def gmres(apply: Callable[[torch.Tensor], torch.Tensor], b: torch.Tensor, tol: float = 1e-6,
          restart: int = 50, maxiter: int = 2000, x0: Optional[torch.Tensor] = None):
    """Restarted GMRES(restart) on every column of b (C, N) float64 CUDA,
    with ``apply(v) = A v`` for all columns at once.  Stops when every column
    has ||b - A x|| <= tol ||b|| or after ``maxiter`` matvecs.  Returns
    (x, info) with info = {"matvecs", "restarts", "rel_residual" (per column,
    recomputed with apply), "converged"}."""
    C, N = b.shape
    dev = b.device
    bnorm = torch.linalg.norm(b, dim=1)
    bnorm = torch.where(bnorm > 0, bnorm, torch.ones_like(bnorm))
    x = torch.zeros_like(b) if x0 is None else x0.clone()
    r = b - apply(x) if x0 is not None else b.clone()
    matvecs = 1 if x0 is not None else 0
    restarts = 0
    tiny = 1e-300
    while True:
        beta = torch.linalg.norm(r, dim=1)
        if bool((beta <= tol * bnorm).all()) or matvecs >= maxiter:
            break
        m = min(restart, maxiter - matvecs)
        V = torch.empty(m + 1, C, N, dtype=b.dtype, device=dev)
        V[0] = r / torch.clamp(beta, min=tiny)[:, None]
        H = np.zeros((C, m + 1, m))
        cs = np.zeros((C, m))
        sn = np.zeros((C, m))
        g = np.zeros((C, m + 1))
        g[:, 0] = beta.cpu().numpy()
        bn = bnorm.cpu().numpy()
        k = 0
        for j in range(m):
            w = apply(V[j])
            matvecs += 1
            # modified Gram-Schmidt, all columns at once
            hcol = torch.empty(j + 2, C, dtype=b.dtype, device=dev)
            for i in range(j + 1):
                hij = (w * V[i]).sum(dim=1)
                w -= hij[:, None] * V[i]
                hcol[i] = hij
            hcol[j + 1] = torch.linalg.norm(w, dim=1)
            V[j + 1] = w / torch.clamp(hcol[j + 1], min=tiny)[:, None]
            hc = hcol.cpu().numpy().T  # (C, j + 2)
            # Givens rotations per column
            for i in range(j):
                t = cs[:, i] * hc[:, i] + sn[:, i] * hc[:, i + 1]
                hc[:, i + 1] = -sn[:, i] * hc[:, i] + cs[:, i] * hc[:, i + 1]
                hc[:, i] = t
            den = np.hypot(hc[:, j], hc[:, j + 1])
            den = np.where(den > 0, den, 1.0)
            cs[:, j] = hc[:, j] / den
            sn[:, j] = hc[:, j + 1] / den
            hc[:, j] = cs[:, j] * hc[:, j] + sn[:, j] * hc[:, j + 1]
            hc[:, j + 1] = 0.0
            g[:, j + 1] = -sn[:, j] * g[:, j]
            g[:, j] = cs[:, j] * g[:, j]
            H[:, : j + 1, j] = hc[:, : j + 1]
            k = j + 1
            if np.all(np.abs(g[:, j + 1]) <= tol * bn):
                break
        # y = H^{-1} g per column (upper triangular k x k), x += V[:k]^T y
        Y = np.zeros((C, k))
        for c in range(C):
            Hc = H[c, :k, :k]
            y = np.zeros(k)
            for i in range(k - 1, -1, -1):
                d = Hc[i, i]
                y[i] = (g[c, i] - Hc[i, i + 1:k] @ y[i + 1:k]) / (d if d != 0 else 1.0)
            Y[c] = y
        Yt = torch.tensor(Y, dtype=b.dtype, device=dev)  # (C, k)
        x += torch.einsum("kcn,ck->cn", V[:k], Yt)
        r = b - apply(x)
        matvecs += 1
        restarts += 1
    rel = (torch.linalg.norm(b - apply(x), dim=1) / bnorm).cpu().numpy()
    return x, {"matvecs": matvecs, "restarts": restarts, "rel_residual": rel,
               "converged": bool(np.all(rel <= tol * 1.0000001))}


def gmres_ir(apply_fast: Callable[[torch.Tensor], torch.Tensor],
             apply_exact: Callable[[torch.Tensor], torch.Tensor], b: torch.Tensor,
             tol: float = 1e-6, inner_tol: float = 1e-3, restart: int = 50,
             maxiter: int = 2000, max_outer: int = 30):
    """Mixed-precision iterative refinement: residuals r = b - A x with the
    float64 operator, corrections from GMRES on the fast (mixed-precision)
    operator to ``inner_tol``.  The fast operator's rounding sets a floor
    near eps * ||K|x|||, which a plain mixed GMRES cannot go below when
    ||x|| >> ||b||; refinement reaches the float64 residual ``tol``.
    Returns (x, info) like ``gmres`` plus "outer" and "exact_matvecs"."""
    bnorm = torch.linalg.norm(b, dim=1)
    bnorm = torch.where(bnorm > 0, bnorm, torch.ones_like(bnorm))
    x = torch.zeros_like(b)
    r = b.clone()
    fast = exact = outer = 0
    while outer < max_outer and fast < maxiter:
        rel = torch.linalg.norm(r, dim=1) / bnorm
        if bool((rel <= tol).all()):
            break
        d, info = gmres(apply_fast, r, inner_tol, restart, maxiter - fast)
        fast += info["matvecs"]
        x += d
        r = b - apply_exact(x)
        exact += 1
        outer += 1
    rel = (torch.linalg.norm(r, dim=1) / bnorm).cpu().numpy()
    return x, {"matvecs": fast, "exact_matvecs": exact, "outer": outer, "rel_residual": rel,
               "converged": bool(np.all(rel <= tol * 1.0000001))}


def kernel_operator(tree: H2_3D_Tree, points: torch.Tensor, lam: float,
                    precision: int = PREC_FP64, adjoint: bool = False,
                    max_cols: Optional[int] = None):
    """v (C, N) -> (K + lam I) v, or its transpose (the adjoint FMM).  With
    ``max_cols`` the columns go through the FMM in groups of at most that
    many (the tree's spectra workspace grows with the columns of a call)."""
    pts = points.contiguous()

    def apply_block(v):
        C = v.shape[0]
        out = torch.zeros_like(v)
        if adjoint:
            compute_adjoint_device(tree, pts, pts, None, v, C, grad_weight=out,
                                   precision=precision)
        else:
            compute_device(tree, pts, pts, v, C, out, precision=precision)
        return out

    def apply(v):
        v = v.contiguous()
        C = v.shape[0]
        step = C if not max_cols else max(1, int(max_cols))
        out = torch.cat([apply_block(v[c:c + step].contiguous()) for c in range(0, C, step)])
        return out + lam * v

    return apply


def _solve(tree, points, b, lam, tol, precision, restart, maxiter, adjoint=False,
           exact_cols=None):
    """float64: GMRES; mixed: GMRES on the mixed operator inside float64
    iterative refinement (float64 matvecs in groups of ``exact_cols``
    columns when given)."""
    exact = kernel_operator(tree, points, lam, PREC_FP64, adjoint, exact_cols)
    if precision == PREC_FP64:
        return gmres(exact, b, tol, restart, maxiter)
    fast = kernel_operator(tree, points, lam, precision, adjoint)
    return gmres_ir(fast, exact, b, tol, 1e-3, restart, maxiter)


class KernelSolve(torch.autograd.Function):
    """x = (K(P, P) + lam I)^{-1} b, differentiable in b and in the points P.
    Mixed precision: GMRES on the mixed-precision FMM inside float64 iterative
    refinement, so the float64 residual meets ``tol``."""

    @staticmethod
    def forward(ctx, points, b, tree, lam, tol, precision, restart, maxiter, exact_cols=None,
                info_out=None):
        x, info = _solve(tree, points, b.contiguous(), lam, tol, precision, restart, maxiter,
                         exact_cols=exact_cols)
        ctx.save_for_backward(points, x)
        ctx.cfg = (tree, lam, tol, precision, restart, maxiter, exact_cols, info_out)
        ctx.info = info
        if info_out is not None:
            info_out["forward"] = info
        return x

    @staticmethod
    def backward(ctx, gx):
        points, x = ctx.saved_tensors
        tree, lam, tol, precision, restart, maxiter, exact_cols, info_out = ctx.cfg
        mu, ainfo = _solve(tree, points, gx.contiguous(), lam, tol, precision, restart, maxiter,
                           adjoint=True, exact_cols=exact_cols)
        if info_out is not None:
            info_out["adjoint"] = ainfo
        grad_points = None
        if ctx.needs_input_grad[0]:
            gt = torch.zeros_like(points)
            gs = torch.zeros_like(points)
            C = x.shape[0]
            compute_adjoint_device(tree, points.contiguous(), points.contiguous(), x.contiguous(),
                                   mu.contiguous(), C, grad_source=gs, grad_target=gt,
                                   precision=precision)
            grad_points = -(gt + gs)
        return grad_points, mu, None, None, None, None, None, None, None, None


def kernel_solve(tree: H2_3D_Tree, points: torch.Tensor, b: torch.Tensor, lam: float,
                 tol: float = 1e-6, precision: Optional[int] = None, restart: int = 50,
                 maxiter: int = 2000, exact_cols: Optional[int] = None,
                 info: Optional[dict] = None) -> torch.Tensor:
    """(K + lam I)^{-1} b for b (C, N); differentiable in b and points (N, 3).
    ``exact_cols`` bounds the columns of one float64 matvec (memory);
    ``info``, if given, receives the solver statistics of the forward solve
    ("forward") and, after backward, of the adjoint solve ("adjoint")."""
    prec = tree.precision if precision is None else int(precision)
    return KernelSolve.apply(points, b, tree, lam, tol, prec, restart, maxiter, exact_cols, info)
