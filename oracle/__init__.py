"""Test oracle for the PBBFMM3D matvec (H2_3D_Compute<T>, include/compute.hpp).

TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
cpu_baseline / reference legs of bench.py may import this package, and only as
the checker or the timed CPU baseline, never as the thing measured or shipped.

Two independent CPU oracles live here:

* ``run_reference``: the UNMODIFIED reference sources compiled by
  oracle/ref/Makefile into oracle/_ref/ref_fmm (FFTW/BLAS shims of our own,
  LAPACK dgesvd_ from the image's OpenBLAS).  It bins targets only and reuses
  that binning for sources (include/compute.hpp:1191-1196), so it is only
  meaningful for S == T; for S != T use the union trick (reference run on
  S u T with zero weights on target-only points).
* ``matvec``: the plain-C FP64 restatement in fmm_oracle.c (oracle/_build),
  which takes the operator tables as arguments so the GPU path and the oracle
  can be fed identical operators.  It is pinned against ``run_reference`` and
  against the golden vectors in tests/golden/.
"""
from __future__ import annotations

import ctypes
import json
import os
import struct
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_BIN = os.path.join(HERE, "_ref", "ref_fmm")
LIB_PATH = os.path.join(HERE, "_build", "libfmm_oracle.so")

# kernel ids (same numbering as the product's C-ABI)
KERNELS = {
    "Laplacian": (0, -1.0),
    "OneOverR2": (1, -2.0),
    "OneOverR4": (2, -4.0),
    "Gaussian": (3, 0.0),
    "Logarithm": (4, 0.0),
    "Quadric": (5, 0.0),
    "InverseQuadric": (6, 0.0),
    "ThinPlateSpline": (7, 0.0),
    "ExpCov": (8, 0.0),
    "GaussSigma": (9, 0.0),
    "AnisoExp": (10, 0.0),
}


def kernel_type_name(kernel: str, param: float = 0.0) -> str:
    """kernelType string the reference uses for its operator-cache file names
    (src/kernel_Types.cpp SetKernelProperty; user kernels of ref_driver.cpp)."""
    if kernel == "ExpCov":
        return "ExpCov%g" % param
    if kernel == "GaussSigma":
        return "GaussS%g" % param
    return kernel


class _Params(ctypes.Structure):
    _fields_ = [
        ("n", ctypes.c_int),
        ("L", ctypes.c_int),
        ("box", ctypes.c_double),
        ("cheb", ctypes.c_int),
        ("kernel", ctypes.c_int),
        ("kparam", ctypes.c_double * 4),
        ("homogen", ctypes.c_double),
        ("rf", ctypes.c_int),
        ("rs", ctypes.c_int),
        ("nlev_ops", ctypes.c_int),
        ("K", ctypes.c_void_p),
        ("U", ctypes.c_void_p),
        ("VT", ctypes.c_void_p),
    ]


_lib = None


def build() -> None:
    """Compile the C restatement (and, where the reference tree is present,
    the reference itself).  Building the checker is not using it."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    ref = os.environ.get("PBBFMM_REF_DIR")
    if ref and os.path.isdir(ref):
        subprocess.run(["make", "-s", "-C", os.path.join(HERE, "ref"), "REF=" + ref], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        dp = ctypes.POINTER(ctypes.c_double)
        L.orc_matvec.argtypes = [ctypes.POINTER(_Params), dp, ctypes.c_int64, dp, ctypes.c_int64,
                                 dp, ctypes.c_int, dp]
        L.orc_matvec.restype = ctypes.c_int
        L.orc_dump.argtypes = [ctypes.c_int, ctypes.c_int, dp]
        L.orc_dump.restype = ctypes.c_int64
        L.orc_direct_rows.argtypes = [ctypes.c_int, dp, dp, ctypes.POINTER(ctypes.c_int64),
                                      ctypes.c_int64, dp, ctypes.c_int64, dp, ctypes.c_int, dp]
        L.orc_direct_rows.restype = None
        L.orc_compute_weights.argtypes = [ctypes.c_int, ctypes.c_int, dp, dp, dp,
                                          ctypes.POINTER(ctypes.c_int)]
        L.orc_kernel.argtypes = [ctypes.c_int, dp, dp, dp]
        L.orc_kernel.restype = ctypes.c_double
        _lib = L
    return _lib


def _dp(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def compute_weights(n: int, cheb: int):
    """Tkz (n*n), Kweights (n^3), Cweights (2n^2), Ktable (343)."""
    Tkz = np.zeros(n * n)
    Kw = np.zeros(n ** 3)
    Cw = np.zeros(2 * n * n)
    Kt = np.zeros(343, dtype=np.int32)
    lib().orc_compute_weights(n, cheb, _dp(Tkz), _dp(Kw), _dp(Cw),
                              Kt.ctypes.data_as(ctypes.POINTER(ctypes.c_int)))
    return Tkz, Kw, Cw, Kt


def matvec(ops: dict, target: np.ndarray, source: np.ndarray, weight: np.ndarray, ncols: int,
           out: np.ndarray | None = None) -> np.ndarray:
    """FP64 restated matvec.  target/source (N,3) float64, weight column-major
    (Ns*ncols,), returns column-major (Nf*ncols,) accumulated into ``out``."""
    target = np.ascontiguousarray(target, dtype=np.float64)
    source = np.ascontiguousarray(source, dtype=np.float64)
    weight = np.ascontiguousarray(weight, dtype=np.float64).ravel()
    Nf, Ns = target.shape[0], source.shape[0]
    if out is None:
        out = np.zeros(Nf * ncols)
    kid, hom = KERNELS[ops["kernel"]]
    p = _Params()
    p.n, p.L, p.box, p.cheb, p.kernel = ops["n"], ops["L"], ops["box"], ops["cheb"], kid
    for i, v in enumerate(ops.get("kparam", [0.0])):
        p.kparam[i] = v
    p.homogen = ops.get("homogen", hom)
    keep = []
    if ops["cheb"]:
        K = np.ascontiguousarray(ops["K"], dtype=np.float64)
        U = np.ascontiguousarray(ops["U"], dtype=np.float64)
        VT = np.ascontiguousarray(ops["VT"], dtype=np.float64)
        keep += [K, U, VT]
        p.rf, p.rs = ops["rf"], ops["rs"]
        p.K, p.U, p.VT = K.ctypes.data, U.ctypes.data, VT.ctypes.data
    else:
        K = np.ascontiguousarray(ops["K"], dtype=np.float64)
        keep.append(K)
        p.K = K.ctypes.data
    p.nlev_ops = ops["nlev_ops"]
    rc = lib().orc_matvec(ctypes.byref(p), _dp(target), Nf, _dp(source), Ns, _dp(weight), ncols,
                          _dp(out))
    if rc != 0:
        raise RuntimeError("orc_matvec failed (%d)" % rc)
    return out


def dump(what: int, level: int) -> np.ndarray:
    n = lib().orc_dump(what, level, None)
    if n < 0:
        raise RuntimeError("nothing to dump")
    a = np.zeros(n)
    lib().orc_dump(what, level, _dp(a))
    return a


def direct(kernel: str, kparam, target, source, weight, ncols, rows=None) -> np.ndarray:
    """FP64 direct sum (include/test.hpp:19-34, inf -> 0) on ``rows`` of the
    targets (all rows if None); column-major (len(rows)*ncols,)."""
    target = np.ascontiguousarray(target, dtype=np.float64)
    source = np.ascontiguousarray(source, dtype=np.float64)
    weight = np.ascontiguousarray(weight, dtype=np.float64).ravel()
    kid, _ = KERNELS[kernel]
    kp = np.zeros(4)
    kp[: len(kparam)] = kparam
    if rows is None:
        rows = np.arange(target.shape[0], dtype=np.int64)
    rows = np.ascontiguousarray(rows, dtype=np.int64)
    out = np.zeros(len(rows) * ncols)
    lib().orc_direct_rows(kid, _dp(kp), _dp(target),
                          rows.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), len(rows),
                          _dp(source), source.shape[0], _dp(weight), ncols, _dp(out))
    return out


# ------------------------------------------------------------ reference cache


def read_reference_cache(outdir: str, kernel_type: str, n: int, cheb: int, L: int,
                         homogeneous: bool) -> dict:
    """Read the operator cache the reference writes (src/H2_3D_Tree.cpp:
    138-239): K = [double box][int level] + nlev blocks, U/V = [int cutoff] +
    nlev blocks.  nlev = 1 for homogeneous kernels, else L-1."""
    nlev = 1 if homogeneous else L - 1
    n3 = n ** 3
    if cheb:
        with open(os.path.join(outdir, "%sChebU%d.bin" % (kernel_type, n)), "rb") as f:
            rf = struct.unpack("i", f.read(4))[0]
            U = np.frombuffer(f.read(8 * n3 * rf * nlev), dtype=np.float64).copy()
        with open(os.path.join(outdir, "%sChebV%d.bin" % (kernel_type, n)), "rb") as f:
            rs = struct.unpack("i", f.read(4))[0]
            VT = np.frombuffer(f.read(8 * n3 * rs * nlev), dtype=np.float64).copy()
        with open(os.path.join(outdir, "%sChebK%d.bin" % (kernel_type, n)), "rb") as f:
            f.read(12)
            K = np.frombuffer(f.read(8 * 316 * rf * rs * nlev), dtype=np.float64).copy()
        return {"cheb": 1, "rf": rf, "rs": rs, "K": K, "U": U, "VT": VT, "nlev_ops": nlev}
    P = (2 * n - 1) ** 3
    with open(os.path.join(outdir, "%sUnifK%d.bin" % (kernel_type, n)), "rb") as f:
        f.read(12)
        K = np.frombuffer(f.read(8 * 316 * P * nlev), dtype=np.float64).copy()
    return {"cheb": 0, "rf": n3, "rs": n3, "K": K, "nlev_ops": nlev}


# --------------------------------------------------------- reference runner


def write_points(path: str, pts: np.ndarray) -> None:
    """Column-wise binary layout of the reference readers (README.md:318-351)."""
    np.ascontiguousarray(np.asarray(pts, dtype=np.float64).T).tofile(path)


def run_reference(kernel: str, param: float, box: float, level: int, order: int, eps: float,
                  cheb: int, points: np.ndarray, weight: np.ndarray, ncols: int,
                  workdir: str | None = None, repeat: int = 1, threads: int | None = None,
                  source: np.ndarray | None = None) -> tuple[np.ndarray, dict, str]:
    """Run the compiled reference (oracle/_ref/ref_fmm) on ``points`` (targets;
    sources = ``source`` or the same set) and return (output, timing, workdir).
    The operator cache lands in <workdir>/output/."""
    if not os.path.exists(REF_BIN):
        raise FileNotFoundError(REF_BIN)
    wd = workdir or tempfile.mkdtemp(prefix="refwd_")
    os.makedirs(wd, exist_ok=True)
    tp, wp = os.path.join(wd, "tgt.bin"), os.path.join(wd, "w.bin")
    op, tm = os.path.join(wd, "out.bin"), os.path.join(wd, "timing.json")
    write_points(tp, points)
    np.ascontiguousarray(weight, dtype=np.float64).ravel().tofile(wp)
    cmd = [REF_BIN, "--kernel", kernel, "--param", repr(param), "--L", repr(box), "--level",
           str(level), "--order", str(order), "--eps", repr(eps), "--cheb", str(cheb), "--ncols",
           str(ncols), "--nf", str(points.shape[0]), "--target", tp, "--weight", wp, "--out", op,
           "--timing", tm, "--workdir", wd, "--repeat", str(repeat)]
    if source is not None:
        sp = os.path.join(wd, "src.bin")
        write_points(sp, source)
        cmd += ["--source", sp, "--ns", str(source.shape[0])]
    env = dict(os.environ)
    env["OPENBLAS_NUM_THREADS"] = "1"
    if threads:
        env["OMP_NUM_THREADS"] = str(threads)
    subprocess.run(cmd, check=True, env=env, stdout=subprocess.DEVNULL)
    out = np.fromfile(op, dtype=np.float64)
    with open(tm) as f:
        timing = json.load(f)
    return out, timing, wd
