"""Shared test helpers: golden-case loading, operator plumbing, error norms."""
from __future__ import annotations

import glob
import json
import os

import numpy as np

import oracle
import pbbfmm3d_b200 as fmm

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

CLASSES = {
    "Laplacian": fmm.kernel_Laplacian, "OneOverR2": fmm.kernel_OneOverR2,
    "OneOverR4": fmm.kernel_OneOverR4, "Gaussian": fmm.kernel_Gaussian,
    "Logarithm": fmm.kernel_Logarithm, "Quadric": fmm.kernel_Quadric,
    "InverseQuadric": fmm.kernel_InverseQuadric, "ThinPlateSpline": fmm.kernel_ThinPlateSpline,
    "AnisoExp": fmm.kernel_AnisoExp,
}


def golden_names():
    return sorted(os.path.basename(p)[5:-4] for p in glob.glob(os.path.join(GOLDEN, "case_*.npz")))


def load_case(name):
    z = np.load(os.path.join(GOLDEN, "case_%s.npz" % name))
    meta = json.loads(str(z["meta"]))
    case = {k: z[k] for k in z.files if k != "meta"}
    case["meta"] = meta
    if "source" not in case:
        case["source"] = case["target"]
    return case


def make_tree(kernel, param, box, level, order, eps, cheb, device=0):
    if kernel == "ExpCov":
        return fmm.kernel_ExpCov(box, level, order, eps, cheb, ell=param, device=device)
    if kernel == "GaussSigma":
        return fmm.kernel_GaussSigma(box, level, order, eps, cheb, sigma=param, device=device)
    return CLASSES[kernel](box, level, order, eps, cheb, device=device)


def case_ops(case):
    """The reference's operators stored with a case (or the case it names)."""
    meta = case["meta"]
    src = case
    if not meta.get("has_ops"):
        if meta.get("ops_from"):
            src = load_case(meta["ops_from"])
        else:
            return None
    ops = {"cheb": meta["cheb"], "rf": src["meta"]["rf"], "rs": src["meta"]["rs"],
           "nlev_ops": src["meta"]["nlev_ops"], "K": src["K"]}
    if meta["cheb"]:
        ops["U"], ops["VT"] = src["U"], src["VT"]
    return ops


def host_ops(kernel, param, box, level, order, eps, cheb):
    """Operators from this library's own float64 precompute (host-only tree)."""
    t = make_tree(kernel, param, box, level, order, eps, cheb, device=-1)
    t.buildFMMTree()
    ops = t.get_operators()
    t.close()
    return ops


def oracle_ops(ops, meta):
    d = dict(ops)
    d.update(kernel=meta["kernel"], n=meta["order"], L=meta["level"], box=meta["box"],
             kparam=[meta["param"]], cheb=meta["cheb"])
    return d


def rel(a, b):
    a, b = np.asarray(a).ravel(), np.asarray(b).ravel()
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
