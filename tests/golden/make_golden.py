"""Generate the golden fixtures in tests/golden/ by running the UNMODIFIED
reference (compiled by oracle/ref/Makefile into oracle/_ref/ref_fmm).

Run here, where the reference sources exist:

    make -C oracle/ref && python tests/golden/make_golden.py

Each case_*.npz holds seeded inputs, the reference's output of
H2_3D_Compute (column-major Nf x nCols), and -- where they are small -- the
reference's own operator-cache contents (the K/U/V files of buildFMMTree), so
that parity can be checked on identical operators.  For S != T the reference is
run on the union S u T with zero weights on the target-only points (the
reference bins targets only and reuses that binning for sources,
include/compute.hpp:1191-1196), and outputs are read at the target rows.

The reference runs with ONE OpenMP thread here: its upward pass lets sibling
tasks add into the parent's moments without synchronisation
(include/compute.hpp:247-278), and multi-threaded runs occasionally lose an
update (observed: 1 run in 12 off by 4.5e-2 relative on case 9).
"""
from __future__ import annotations

import json
import os
import shutil
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle  # noqa: E402

# the reference checkout (read-only) is named by PBBFMM_REF_DIR; its input/
# fixture is used when present
REF_INPUT = os.path.join(os.environ.get("PBBFMM_REF_DIR", ""), "input")


def run_case(name, kernel, param, box, level, order, eps, cheb, target, weight, ncols,
             source=None, keep_ops=True, note="", ops_from=None):
    wd = os.path.join("/tmp", "golden_" + name)
    shutil.rmtree(wd, ignore_errors=True)
    if source is None:
        out, timing, wd = oracle.run_reference(kernel, param, box, level, order, eps, cheb, target,
                                               weight, ncols, workdir=wd, threads=1)
        meta_src = "same"
    else:
        # union trick: X = T u S, weights zero on the T part
        X = np.concatenate([target, source], axis=0)
        Nf, Ns = target.shape[0], source.shape[0]
        wu = np.zeros((ncols, Nf + Ns))
        wu[:, Nf:] = weight.reshape(ncols, Ns)
        outu, timing, wd = oracle.run_reference(kernel, param, box, level, order, eps, cheb, X,
                                                wu.ravel(), ncols, workdir=wd, threads=1)
        out = outu.reshape(ncols, Nf + Ns)[:, :Nf].ravel()
        meta_src = "distinct"
    kid, hom = oracle.KERNELS[kernel]
    ops = oracle.read_reference_cache(os.path.join(wd, "output"),
                                      oracle.kernel_type_name(kernel, param), order, cheb, level,
                                      abs(hom) > 0.1)
    meta = dict(name=name, kernel=kernel, param=param, box=box, level=level, order=order, eps=eps,
                cheb=cheb, ncols=ncols, source=meta_src, rf=ops["rf"], rs=ops["rs"],
                nlev_ops=ops["nlev_ops"], homogen=hom, note=note, has_ops=bool(keep_ops),
                ops_from=ops_from)
    arrays = dict(meta=np.array(json.dumps(meta)), target=target, weight=weight, output=out)
    if source is not None:
        arrays["source"] = source
    if keep_ops:
        arrays["K"] = ops["K"]
        if cheb:
            arrays["U"] = ops["U"]
            arrays["VT"] = ops["VT"]
    path = os.path.join(HERE, "case_%s.npz" % name)
    np.savez_compressed(path, **arrays)
    shutil.rmtree(wd, ignore_errors=True)
    print("%-28s N=%d C=%d rf=%d ops=%s -> %.1f KB" % (name, target.shape[0], ncols, ops["rf"],
                                                      keep_ops, os.path.getsize(path) / 1024))


def main():
    rng = np.random.default_rng(20240607)
    # 1. Laplacian, Chebyshev n=3, 3 levels, uniform cube (config-1 kernel, smaller)
    p = rng.uniform(-0.5, 0.5, (3000, 3))
    run_case("lap_cheb3", "Laplacian", 0.0, 1.0, 3, 3, 1e-4, 1, p, rng.uniform(-1, 1, 3000), 1)
    # 2. exponential covariance exp(-r/0.3), uniform grid n=4 (FFT M2L), 2 columns
    p = rng.uniform(-0.5, 0.5, (3000, 3))
    run_case("expcov_unif4", "ExpCov", 0.3, 1.0, 3, 4, 1e-5, 0, p, rng.standard_normal(6000), 2)
    # 3. Gaussian exp(-r^2), Chebyshev n=3, non-homogeneous (per-level operators), box 2
    p = rng.uniform(-1.0, 1.0, (2000, 3))
    run_case("gauss_cheb3", "Gaussian", 0.0, 2.0, 3, 3, 1e-3, 1, p, rng.uniform(-1, 1, 2000), 1)
    # 4. sources != targets (union trick), Laplacian uniform n=3
    #    T holds the corners of bbox(S u T), so the reference's recentring on
    #    its (union) targets equals recentring on T alone and the trees match
    t = rng.uniform(-0.5, 0.5, (1500, 3))
    s = rng.uniform(-0.5, 0.5, (1500, 3))
    x = np.concatenate([t, s])
    t[0], t[1] = x.min(axis=0), x.max(axis=0)
    run_case("lap_unif3_st", "Laplacian", 0.0, 1.0, 3, 3, 1e-5, 0, t, rng.uniform(-1, 1, 1500), 1,
             source=s, note="reference run on S u T with zero weights on T; bbox(T) = bbox(S u T)")
    # 5. the reference's own input fixture (input/*.bin, metadata 1,4,5000,5000,1,3),
    #    Laplacian Chebyshev n=4, eps 1e-5 -- outputs only (operators are 5.8 MB)
    if os.path.isdir(REF_INPUT):
        N = 5000
        pts = np.fromfile(os.path.join(REF_INPUT, "field_test.bin")).reshape(3, N).T.copy()
        w = np.fromfile(os.path.join(REF_INPUT, "charge_test.bin"))[:N].copy()
        run_case("ref_fixture_lap_cheb4", "Laplacian", 0.0, 1.0, 3, 4, 1e-5, 1, pts, w, 1,
                 keep_ops=False, note="reference input/field_test.bin + charge_test.bin")
    # 6. 1/r^2, uniform n=4, 4 levels (homogeneous, one operator level)
    p = rng.uniform(-0.5, 0.5, (4000, 3))
    run_case("r2_unif4_l4", "OneOverR2", 0.0, 1.0, 4, 4, 1e-5, 0, p, rng.uniform(-1, 1, 4000), 1,
             keep_ops=False, note="uniform operators are recomputed exactly")
    # 7. clustered points with many empty cells (two tight blobs + a few strays)
    a = rng.normal([-0.25, -0.2, -0.3], 0.03, (900, 3))
    b = rng.normal([0.3, 0.25, 0.2], 0.02, (900, 3))
    c = rng.uniform(-0.5, 0.5, (200, 3))
    p = np.clip(np.concatenate([a, b, c]), -0.5, 0.5)
    run_case("lap_cheb3_clustered", "Laplacian", 0.0, 1.0, 4, 3, 1e-4, 1, p,
             rng.uniform(-1, 1, 2000), 1, keep_ops=False, ops_from="lap_cheb3")
    # 8. anisotropic exp kernel of the python binding, uniform n=3, 3 columns
    p = rng.uniform(-0.5, 0.5, (2500, 3))
    run_case("aniso_unif3", "AnisoExp", 0.0, 1.0, 3, 3, 1e-5, 0, p, rng.standard_normal(7500), 3,
             keep_ops=False, note="uniform operators are recomputed exactly")
    # 9. thin-plate spline, Chebyshev n=3, points partly outside the box (box 0.8)
    p = rng.uniform(-0.5, 0.5, (2000, 3))
    run_case("tps_cheb3_outside", "ThinPlateSpline", 0.0, 0.8, 3, 3, 1e-3, 1, p,
             rng.uniform(-1, 1, 2000), 1, note="box smaller than the point cloud")


if __name__ == "__main__":
    main()
