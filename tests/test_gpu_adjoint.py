"""The adjoint FMM (pbbfmm_compute_adjoint_device) and its autograd wrapper.

- dL/d(weight) = K^T g is the exact transpose of this tree's FMM:
  <g, K w> = <K^T g, w> to 1e-11 relative in float64.  With S = T and uniform
  interpolation the FMM is self-adjoint, so K^T g equals the reference's own
  H2_3D_Compute applied to g (roles swapped, same points) to 1e-12.
- dL/d(positions) is the exact derivative of the float64 FMM: it matches
  central finite differences (h = 1e-6) of the forward FMM to 1e-6 relative,
  on coordinates whose move crosses no leaf boundary.
- Against direct sums (K^T g and the analytic position gradient) the
  agreement is the FMM's own approximation error."""
import numpy as np
import pytest

import oracle
import pbbfmm3d_b200 as fmm
from helpers import make_tree, rel

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _t(a):
    return torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda")


def _tree(kernel, param, level, order, eps, cheb):
    t = make_tree(kernel, param, 1.0, level, order, eps, cheb)
    t.buildFMMTree()
    return t


def _fwd(t, T, S, W, C, prec=fmm.PREC_FP64):
    out = torch.zeros(C, T.shape[0], dtype=torch.float64, device="cuda")
    fmm.compute_device(t, _t(T), _t(S), _t(W), C, out, precision=prec)
    return out.cpu().numpy()


def _adj(t, T, S, W, G, C, prec=fmm.PREC_FP64, want=("w", "s", "t")):
    gw = torch.zeros(C, S.shape[0], dtype=torch.float64, device="cuda") if "w" in want else None
    gs = torch.zeros(S.shape[0], 3, dtype=torch.float64, device="cuda") if "s" in want else None
    gt = torch.zeros(T.shape[0], 3, dtype=torch.float64, device="cuda") if "t" in want else None
    fmm.compute_adjoint_device(t, _t(T), _t(S), _t(W), _t(G), C, grad_weight=gw, grad_source=gs,
                               grad_target=gt, precision=prec)
    torch.cuda.synchronize()
    return [None if x is None else x.cpu().numpy() for x in (gw, gs, gt)]


CASES = [
    # kernel, param, level, order, eps, cheb, ncols
    ("Laplacian", 0.0, 4, 5, 1e-7, 1, 2),
    ("GaussSigma", 0.1, 4, 5, 1e-6, 1, 2),   # per-level operators
    ("ExpCov", 0.3, 4, 4, 1e-5, 0, 3),       # uniform, FFT M2L
    ("OneOverR2", 0.0, 3, 4, 1e-5, 1, 1),
]
IDS = [f"{c[0]}{'C' if c[5] else 'U'}" for c in CASES]


def _points(rng, nt=4000, ns=3500):
    T = rng.uniform(-0.5, 0.5, (nt, 3))
    S = rng.uniform(-0.45, 0.45, (ns, 3))  # inside bbox(T): well-defined binning
    return T, S


@pytest.mark.parametrize("case", CASES, ids=IDS)
def test_adjoint_is_exact_transpose(case):
    kernel, param, level, order, eps, cheb, C = case
    rng = np.random.default_rng(3)
    T, S = _points(rng)
    W = rng.standard_normal((C, S.shape[0]))
    G = rng.standard_normal((C, T.shape[0]))
    t = _tree(kernel, param, level, order, eps, cheb)
    f = _fwd(t, T, S, W, C)
    gw, _, _ = _adj(t, T, S, W, G, C, want=("w",))
    lhs, rhs = float((G * f).sum()), float((gw * W).sum())
    assert abs(lhs - rhs) <= 1e-11 * abs(lhs) + 1e-13 * np.abs(G * f).sum(), (lhs, rhs)
    # and K^T g against the direct transposed sum (approximation level)
    d = oracle.direct(kernel, [param], S, T, G.ravel(), C)
    assert rel(gw.ravel(), d) < 1e-3


def test_adjoint_matches_reference_with_roles_swapped():
    """S = T, uniform interpolation: K^T g from the adjoint pass equals the
    reference's H2_3D_Compute on (T, T, g)."""
    rng = np.random.default_rng(5)
    T = rng.uniform(-0.5, 0.5, (3000, 3))
    C = 2
    G = rng.standard_normal((C, 3000))
    W = rng.standard_normal((C, 3000))
    t = _tree("ExpCov", 0.3, 4, 4, 1e-5, 0)
    gw, _, _ = _adj(t, T, T, W, G, C, want=("w",))
    ref, _, _ = oracle.run_reference("ExpCov", 0.3, 1.0, 4, 4, 1e-5, 0, T, G.ravel(), C,
                                     threads=1)
    assert rel(gw.ravel(), ref) < 1e-12


def _safe_coords(P, ctr, level, rng, k, exclude=()):
    """k (point, dim) pairs whose +-1e-6 move stays inside its leaf."""
    w = 1.0 / (1 << level)
    u = (P - (ctr - 0.5)) / w
    frac = u - np.floor(u)
    ok = (np.minimum(frac, 1 - frac) > 1e-3)
    for i in exclude:
        ok[i, :] = False
    cand = np.argwhere(ok)
    return cand[rng.choice(len(cand), k, replace=False)]


@pytest.mark.parametrize("case", CASES[:3], ids=IDS[:3])
def test_position_gradients_match_finite_differences(case):
    kernel, param, level, order, eps, cheb, C = case
    rng = np.random.default_rng(11)
    T, S = _points(rng, 2500, 2000)
    W = rng.standard_normal((C, S.shape[0]))
    G = rng.standard_normal((C, T.shape[0]))
    t = _tree(kernel, param, level, order, eps, cheb)
    _, gs, gt = _adj(t, T, S, W, G, C)
    ctr = 0.5 * (T.min(0) + T.max(0))
    h = 1e-6

    def loss(Tm, Sm):
        return float((G * _fwd(t, Tm, Sm, W, C)).sum())

    fd, an = [], []
    for j, d in _safe_coords(S, ctr, level, rng, 12):
        Sp, Sm = S.copy(), S.copy()
        Sp[j, d] += h
        Sm[j, d] -= h
        fd.append((loss(T, Sp) - loss(T, Sm)) / (2 * h))
        an.append(gs[j, d])
    # targets: keep the bounding box (and so the tree) fixed
    ext = set(np.argmin(T, 0)) | set(np.argmax(T, 0))
    for i, d in _safe_coords(T, ctr, level, rng, 12, exclude=ext):
        Tp, Tm = T.copy(), T.copy()
        Tp[i, d] += h
        Tm[i, d] -= h
        fd.append((loss(Tp, S) - loss(Tm, S)) / (2 * h))
        an.append(gt[i, d])
    fd, an = np.array(fd), np.array(an)
    assert rel(an, fd) < 1e-6, np.c_[an, fd]


def test_position_gradients_against_direct_sums():
    """Laplacian and Gaussian: analytic gradients of the direct sums, within
    the approximation error of the differentiated interpolation."""
    rng = np.random.default_rng(12)
    T, S = _points(rng, 3000, 2500)
    C = 2
    W = rng.standard_normal((C, S.shape[0]))
    G = rng.standard_normal((C, T.shape[0]))
    for kernel, param, cheb in (("Laplacian", 0.0, 1), ("GaussSigma", 0.1, 1)):
        t = _tree(kernel, param, 4, 5, 1e-7, cheb)
        gw, gs, gt = _adj(t, T, S, W, G, C)
        # the same case's potential error (K^T g against the direct sum)
        e_pot = rel(gw.ravel(), oracle.direct(kernel, [param], S, T, G.ravel(), C))
        D = S[None, :, :] - T[:, None, :]  # d = y - x, (Nf, Ns, 3)
        r2 = (D ** 2).sum(-1)
        if kernel == "Laplacian":
            dk = -D / np.where(r2 > 0, r2, np.inf)[..., None] ** 1.5  # dK/dd
        else:
            s2 = 2 * param ** 2
            dk = (-2.0 / s2) * D * np.exp(-r2 / s2)[..., None]
        A = np.einsum("ci,cj->ij", G, W)  # sum_c g_ic w_jc
        gs_ref = np.einsum("ij,ijd->jd", A, dk)    # d/dy = +dK/dd
        gt_ref = -np.einsum("ij,ijd->id", A, dk)   # d/dx = -dK/dd
        # derivatives of the interpolant carry about one order more
        # approximation error than the potential (measured: 1/r 1.5e-4,
        # exp(-r^2 / 0.02) 2e-3 at n = 5)
        bound = max(30 * e_pot, 1e-6)
        assert rel(gs, gs_ref) < bound, (kernel, rel(gs, gs_ref), e_pot)
        assert rel(gt, gt_ref) < bound, (kernel, rel(gt, gt_ref), e_pot)


@pytest.mark.parametrize("case", CASES[:3], ids=IDS[:3])
def test_mixed_adjoint_close_to_fp64(case):
    kernel, param, level, order, eps, cheb, C = case
    rng = np.random.default_rng(21)
    T, S = _points(rng, 6000, 5000)
    W = rng.standard_normal((C, S.shape[0]))
    G = rng.standard_normal((C, T.shape[0]))
    t = _tree(kernel, param, level, order, eps, cheb)
    a64 = _adj(t, T, S, W, G, C)
    a32 = _adj(t, T, S, W, G, C, prec=fmm.PREC_MIXED)
    for x64, x32 in zip(a64, a32):
        assert rel(x32, x64) < 1e-5


def test_autograd_function():
    from pbbfmm3d_b200.autograd import fmm_matvec

    rng = np.random.default_rng(31)
    T, S = _points(rng, 3000, 2000)
    C = 2
    W = rng.standard_normal((C, S.shape[0]))
    G = rng.standard_normal((C, T.shape[0]))
    t = _tree("GaussSigma", 0.1, 4, 5, 1e-6, 1)
    tt, ss, ww = (_t(x).requires_grad_(True) for x in (T, S, W))
    out = fmm_matvec(t, tt, ss, ww)
    assert np.allclose(out.detach().cpu().numpy(), _fwd(t, T, S, W, C), rtol=0, atol=1e-12)
    (out * _t(G)).sum().backward()
    gw, gs, gt = _adj(t, T, S, W, G, C)
    assert rel(ww.grad.cpu().numpy(), gw) < 1e-14
    assert rel(ss.grad.cpu().numpy(), gs) < 1e-14
    assert rel(tt.grad.cpu().numpy(), gt) < 1e-14


def test_adjoint_matches_reference_union_with_roles_swapped():
    """S != T: the reference's H2_3D_Compute on the union S + T, with weights
    g on the targets and 0 on the sources, read at the sources, is K^T g on
    the same tree when bbox(T) = bbox(S + T) (T holds the corners; the
    reference bins everything with the targets' box).  Uniform interpolation
    (operators recomputed exactly): agreement to 1e-12."""
    rng = np.random.default_rng(41)
    T = rng.uniform(-0.5, 0.5, (2500, 3))
    T[:8] = np.array([[x, y, z] for x in (-0.5, 0.5) for y in (-0.5, 0.5) for z in (-0.5, 0.5)])
    S = rng.uniform(-0.5, 0.5, (2000, 3))
    C = 2
    G = rng.standard_normal((C, T.shape[0]))
    W = rng.standard_normal((C, S.shape[0]))
    t = _tree("ExpCov", 0.3, 4, 4, 1e-5, 0)
    gw, _, _ = _adj(t, T, S, W, G, C, want=("w",))
    U = np.vstack([T, S])
    Wu = np.hstack([G, np.zeros((C, S.shape[0]))])
    out, _, _ = oracle.run_reference("ExpCov", 0.3, 1.0, 4, 4, 1e-5, 0, U, Wu.ravel(), C,
                                     threads=1)
    ref = out.reshape(C, U.shape[0])[:, T.shape[0]:]
    assert rel(gw, ref) < 1e-12
