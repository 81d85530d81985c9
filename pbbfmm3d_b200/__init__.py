"""pbbfmm3d_b200: B200-native black-box FMM matvec, drop-in for PBBFMM3D's
``H2_3D_Compute`` hot path.

The Python surface mirrors the reference's C++ API (README.md:76-122 of the
reference; include/compute.hpp:20, src/H2_3D_Tree.cpp:12-66,
src/kernel_Types.cpp):

    tree = kernel_Laplacian(L, tree_level, interpolation_order, epsilon, use_chebyshev)
    tree.buildFMMTree()
    H2_3D_Compute(tree, target, source, weight, nCols, output)   # output += K @ weight

with ``target``/``source`` shaped (N, 3) float64, ``weight`` column-major
(Ns * nCols,) and ``output`` column-major (Nf * nCols,) accumulated in place,
exactly the reference's layouts.  ``compute_device`` runs the same matvec on
CUDA tensors without host copies.  All arithmetic happens in the CUDA library
``libpbbfmm3d_b200.so``; there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
from typing import Optional

import numpy as np

from . import _lib
from ._lib import FMMError, PREC_FP64, PREC_MIXED

__all__ = [
    "H2_3D_Tree", "H2_3D_Compute", "compute_device", "FMMError", "PREC_FP64", "PREC_MIXED",
    "kernel_Laplacian", "kernel_OneOverR2", "kernel_OneOverR4", "kernel_Gaussian",
    "kernel_Logarithm", "kernel_Quadric", "kernel_InverseQuadric", "kernel_ThinPlateSpline",
    "kernel_ExpCov", "kernel_GaussSigma", "kernel_AnisoExp", "KERNEL_IDS",
]

KERNEL_IDS = {
    "Laplacian": 0, "OneOverR2": 1, "OneOverR4": 2, "Gaussian": 3, "Logarithm": 4,
    "Quadric": 5, "InverseQuadric": 6, "ThinPlateSpline": 7, "ExpCov": 8, "GaussSigma": 9,
    "AnisoExp": 10,
}
# SetKernelProperty's homogen per kernel (src/kernel_Types.cpp)
HOMOGEN = {0: -1.0, 1: -2.0, 2: -4.0}


def _dp(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


_TC_FORMATS = {"f16": _lib.TC_F16, "tf32": _lib.TC_TF32}

class H2_3D_Tree:
    """FMM tree: box, levels, interpolation order and kernel (H2_3D_Tree,
    include/H2_3D_Tree.hpp:16-116).  Subclasses fix the kernel like the
    reference's ``kernel_*`` classes.  ``device=-1`` gives a host-only tree
    (operator precompute only)."""

    kernel_name = "Laplacian"

    def __init__(self, L: float, tree_level: int, interpolation_order: int, epsilon: float,
                 use_chebyshev: int, device: int = 0, kernel_param=(0.0,)):
        self.L = float(L)
        self.tree_level = int(tree_level)
        self.interpolation_order = int(interpolation_order)
        self.epsilon = float(epsilon)
        self.use_chebyshev = int(use_chebyshev)
        self.device = int(device)
        self.kernel_id = KERNEL_IDS[self.kernel_name]
        self.kernel_param = tuple(float(x) for x in kernel_param) + (0.0,) * (4 - len(kernel_param))
        self.homogen = HOMOGEN.get(self.kernel_id, 0.0)
        self.precision = PREC_FP64
        p = _lib.TreeParams()
        p.L, p.tree_level, p.interpolation_order = self.L, self.tree_level, self.interpolation_order
        p.epsilon, p.use_chebyshev, p.kernel = self.epsilon, self.use_chebyshev, self.kernel_id
        for i in range(4):
            p.kernel_param[i] = self.kernel_param[i]
        h = ctypes.c_void_p()
        _lib.check(_lib.lib().pbbfmm_tree_create(ctypes.byref(p), self.device, ctypes.byref(h)))
        self._h = h
        self.built = False

    # -- reference API --------------------------------------------------
    def buildFMMTree(self, cache_dir: Optional[str] = None) -> None:
        """Precompute interpolation weights and M2L operators (float64, host)
        and upload them (src/H2_3D_Tree.cpp:40-66).  ``cache_dir`` reads or
        writes operator files in the reference's format and names."""
        _lib.check(_lib.lib().pbbfmm_tree_build(
            self._h, cache_dir.encode() if cache_dir else None))
        self.built = True

    # -- extensions -----------------------------------------------------
    @property
    def nlev_ops(self) -> int:
        return 1 if abs(self.homogen) > 0.1 else self.tree_level - 1

    def set_operators(self, K: np.ndarray, U: Optional[np.ndarray] = None,
                      VT: Optional[np.ndarray] = None, rf: int = 0, rs: int = 0) -> None:
        """Install operators in FMMReadMatrices' layout (e.g. the reference's
        own cache files) instead of precomputing them."""
        K = np.ascontiguousarray(K, dtype=np.float64)
        U = None if U is None else np.ascontiguousarray(U, dtype=np.float64)
        VT = None if VT is None else np.ascontiguousarray(VT, dtype=np.float64)
        Up = _dp(U) if U is not None else None
        Vp = _dp(VT) if VT is not None else None
        _lib.check(_lib.lib().pbbfmm_tree_set_operators(self._h, int(rf), int(rs), self.nlev_ops,
                                                        _dp(K), Up, Vp))
        self.built = True

    def get_operators(self) -> dict:
        rf, rs, nl = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        L = _lib.lib()
        _lib.check(L.pbbfmm_tree_get_operators(self._h, ctypes.byref(rf), ctypes.byref(rs),
                                               ctypes.byref(nl), None, None, None))
        n3 = self.interpolation_order ** 3
        P = (2 * self.interpolation_order - 1) ** 3
        if self.use_chebyshev:
            K = np.zeros(nl.value * 316 * rf.value * rs.value)
            U = np.zeros(nl.value * n3 * rf.value)
            VT = np.zeros(nl.value * rs.value * n3)
            _lib.check(L.pbbfmm_tree_get_operators(self._h, None, None, None, _dp(K), _dp(U), _dp(VT)))
            return {"cheb": 1, "rf": rf.value, "rs": rs.value, "nlev_ops": nl.value, "K": K, "U": U,
                    "VT": VT}
        K = np.zeros(nl.value * 316 * P)
        _lib.check(L.pbbfmm_tree_get_operators(self._h, None, None, None, _dp(K), None, None))
        return {"cheb": 0, "rf": n3, "rs": n3, "nlev_ops": nl.value, "K": K}

    def get_weights(self):
        n = self.interpolation_order
        Tkz, Kw, Cw = np.zeros(n * n), np.zeros(n ** 3), np.zeros(2 * n * n)
        Kt = np.zeros(343, dtype=np.int32)
        _lib.check(_lib.lib().pbbfmm_tree_get_weights(
            self._h, _dp(Tkz), _dp(Kw), _dp(Cw), Kt.ctypes.data_as(ctypes.POINTER(ctypes.c_int))))
        return Tkz, Kw, Cw, Kt

    def set_precision(self, precision: int) -> None:
        _lib.check(_lib.lib().pbbfmm_set_precision(self._h, int(precision)))
        self.precision = int(precision)

    def set_tensor_cores(self, enable: bool = True, fmt: str = "f16") -> None:
        """Chebyshev M2L of the mixed path on tcgen05 or, with enable=False,
        on the CUDA cores in float32.  fmt: "f16" (power-of-two scaled F16
        hi / lo operands, the default) or "tf32" (3xTF32)."""
        if fmt not in _TC_FORMATS:
            raise ValueError("fmt must be 'f16' or 'tf32'")
        mode = _TC_FORMATS[fmt] if enable else _lib.TC_OFF
        _lib.check(_lib.lib().pbbfmm_set_tensor_cores(self._h, mode))

    def tensor_core_m2l(self) -> bool:
        """True when a mixed Chebyshev compute of this tree runs its M2L on tcgen05."""
        return bool(_lib.lib().pbbfmm_tensor_core_m2l(self._h))

    def tensor_core_format(self):
        """"f16" or "tf32": the operand format of the tensor-core M2L a mixed
        Chebyshev compute of this tree runs with; None on the CUDA cores."""
        m = _lib.lib().pbbfmm_tensor_core_m2l(self._h)
        return {v: k for k, v in _TC_FORMATS.items()}.get(m)

    def set_timing(self, enable: bool = True) -> None:
        _lib.check(_lib.lib().pbbfmm_set_timing(self._h, 1 if enable else 0))

    def phase_times(self) -> dict:
        ms = (ctypes.c_float * 16)()
        nph = ctypes.c_int()
        names = ctypes.c_char_p()
        _lib.check(_lib.lib().pbbfmm_get_phase_times(self._h, ms, 16, ctypes.byref(nph),
                                                     ctypes.byref(names)))
        return dict(zip(names.value.decode().split(","), [ms[i] for i in range(nph.value)]))

    def reset_kernel_times(self) -> None:
        _lib.check(_lib.lib().pbbfmm_reset_kernel_times(self._h))

    def kernel_times(self) -> dict:
        """{slot: (ms, launches)} summed since the last reset (timing on)."""
        ms = (ctypes.c_float * 32)()
        cnt = (ctypes.c_int * 32)()
        ns = ctypes.c_int()
        names = ctypes.c_char_p()
        _lib.check(_lib.lib().pbbfmm_get_kernel_times(self._h, ms, cnt, 32, ctypes.byref(ns),
                                                      ctypes.byref(names)))
        keys = names.value.decode().split(",")
        return {k: (ms[i], cnt[i]) for i, k in enumerate(keys[:ns.value])}

    def debug_copy(self, what: int, level: int = 0) -> np.ndarray:
        n = ctypes.c_int64()
        L = _lib.lib()
        _lib.check(L.pbbfmm_debug_copy(self._h, what, level, None, 0, ctypes.byref(n)))
        out = np.zeros(n.value)
        _lib.check(L.pbbfmm_debug_copy(self._h, what, level, _dp(out), n.value, ctypes.byref(n)))
        return out

    def close(self) -> None:
        if getattr(self, "_h", None):
            _lib.lib().pbbfmm_tree_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _kernel_class(name: str, doc: str):
    return type("kernel_" + name, (H2_3D_Tree,), {"kernel_name": name, "__doc__": doc})


kernel_Laplacian = _kernel_class("Laplacian", "1/r (src/kernel_Types.cpp:7-28)")
kernel_OneOverR2 = _kernel_class("OneOverR2", "1/r^2 (src/kernel_Types.cpp:101-120)")
kernel_OneOverR4 = _kernel_class("OneOverR4", "1/r^4 (src/kernel_Types.cpp:34-53)")
kernel_Gaussian = _kernel_class("Gaussian", "exp(-r^2) (src/kernel_Types.cpp:56-74)")
kernel_Logarithm = _kernel_class("Logarithm", "0.5 log r^2 (src/kernel_Types.cpp:77-99)")
kernel_Quadric = _kernel_class("Quadric", "1 + r^2 (src/kernel_Types.cpp:123-138)")
kernel_InverseQuadric = _kernel_class("InverseQuadric", "1/(1+r^2) (src/kernel_Types.cpp:140-155)")
kernel_ThinPlateSpline = _kernel_class("ThinPlateSpline",
                                       "0.5 r^2 log r^2 (src/kernel_Types.cpp:157-178)")
kernel_AnisoExp = _kernel_class("AnisoExp",
                                "0.75 exp(-sqrt(dx^2/100+dy^2/100+dz^2/2.25)) (python/mykernel_python.hpp:10-18)")


class kernel_ExpCov(H2_3D_Tree):
    """exp(-r / ell): the exponential covariance kernel (user kernel)."""
    kernel_name = "ExpCov"

    def __init__(self, L, tree_level, interpolation_order, epsilon, use_chebyshev, ell=1.0,
                 device=0):
        super().__init__(L, tree_level, interpolation_order, epsilon, use_chebyshev, device,
                         kernel_param=(ell,))


class kernel_GaussSigma(H2_3D_Tree):
    """exp(-r^2 / (2 sigma^2)) (user kernel)."""
    kernel_name = "GaussSigma"

    def __init__(self, L, tree_level, interpolation_order, epsilon, use_chebyshev, sigma=1.0,
                 device=0):
        super().__init__(L, tree_level, interpolation_order, epsilon, use_chebyshev, device,
                         kernel_param=(sigma,))


def H2_3D_Compute(tree: H2_3D_Tree, target, source, weight, nCols: int, output) -> np.ndarray:
    """``output += K(target, source) @ weight`` through the host-buffer C-ABI
    entry (include/compute.hpp:67-149 semantics).  ``target``/``source`` are
    (N, 3) float64 (vector3 AoS), ``weight`` column-major (Ns*nCols,), and
    ``output`` column-major (Nf*nCols,) float64, updated in place."""
    if not tree.built:
        raise FMMError(_lib.ERR_STATE, "call buildFMMTree() first")
    t = np.ascontiguousarray(target, dtype=np.float64).reshape(-1, 3)
    same = source is target
    s = t if same else np.ascontiguousarray(source, dtype=np.float64).reshape(-1, 3)
    w = np.ascontiguousarray(weight, dtype=np.float64).ravel()
    if not isinstance(output, np.ndarray) or output.dtype != np.float64 or not output.flags.c_contiguous:
        raise TypeError("output must be a C-contiguous float64 numpy array")
    Nf, Ns = t.shape[0], s.shape[0]
    if w.size != Ns * nCols or output.size != Nf * nCols:
        raise ValueError("weight must hold Ns*nCols and output Nf*nCols values")
    _lib.check(_lib.lib().pbbfmm_compute(tree._h, _dp(t), Nf, _dp(s), Ns, _dp(w), int(nCols),
                                         _dp(output)))
    return output


def launch_count() -> int:
    """Kernel launches issued by the library so far in this process."""
    return int(_lib.lib().pbbfmm_launch_count())


def measure_fma_peak(device: int = 0, precision: int = PREC_FP64) -> float:
    """Measured FMA throughput (TFLOP/s) of the FP64 or FP32 pipes."""
    v = ctypes.c_double()
    _lib.check(_lib.lib().pbbfmm_measure_fma_peak(int(device), int(precision), ctypes.byref(v)))
    return v.value


def compute_device(tree: H2_3D_Tree, target, source, weight, nCols: int, output,
                   precision: Optional[int] = None, stream=None):
    """Device-buffer matvec on torch CUDA tensors (float64, contiguous):
    target/source (N, 3), weight (nCols, Ns) or flat column-major, output
    (nCols, Nf) or flat, accumulated.  Runs on ``stream`` (default: torch's
    current stream) without synchronising."""
    import torch

    for name, x in (("target", target), ("source", source), ("weight", weight), ("output", output)):
        if not (isinstance(x, torch.Tensor) and x.is_cuda and x.dtype == torch.float64
                and x.is_contiguous()):
            raise TypeError(name + " must be a contiguous float64 CUDA tensor")
    Nf, Ns = target.numel() // 3, source.numel() // 3
    if weight.numel() != Ns * nCols or output.numel() != Nf * nCols:
        raise ValueError("weight must hold Ns*nCols and output Nf*nCols values")
    if stream is None:
        stream = torch.cuda.current_stream(target.device).cuda_stream
    prec = tree.precision if precision is None else int(precision)
    _lib.check(_lib.lib().pbbfmm_compute_device(
        tree._h, target.data_ptr(), Nf, source.data_ptr(), Ns, weight.data_ptr(), int(nCols),
        output.data_ptr(), prec, ctypes.c_void_p(stream)))
    return output


def compute_adjoint_device(tree: H2_3D_Tree, target, source, weight, g, nCols: int,
                           grad_weight=None, grad_source=None, grad_target=None,
                           precision: Optional[int] = None, stream=None):
    """Adjoint of ``compute_device`` on torch CUDA tensors (float64,
    contiguous): given g = dL/d(output) (nCols, Nf), accumulate
    grad_weight (nCols, Ns) += K^T g, grad_source (Ns, 3) += dL/d(source) and
    grad_target (Nf, 3) += dL/d(target), each when given.  ``weight`` is
    needed for the position gradients.  No synchronisation."""
    import torch

    def ok(x):
        return (isinstance(x, torch.Tensor) and x.is_cuda and x.dtype == torch.float64
                and x.is_contiguous())

    for name, x in (("target", target), ("source", source), ("g", g)):
        if not ok(x):
            raise TypeError(name + " must be a contiguous float64 CUDA tensor")
    for name, x in (("weight", weight), ("grad_weight", grad_weight),
                    ("grad_source", grad_source), ("grad_target", grad_target)):
        if x is not None and not ok(x):
            raise TypeError(name + " must be a contiguous float64 CUDA tensor")
    Nf, Ns = target.numel() // 3, source.numel() // 3
    if g.numel() != Nf * nCols:
        raise ValueError("g must hold Nf*nCols values")
    if grad_weight is not None and grad_weight.numel() != Ns * nCols:
        raise ValueError("grad_weight must hold Ns*nCols values")
    if grad_source is not None and grad_source.numel() != Ns * 3:
        raise ValueError("grad_source must hold Ns*3 values")
    if grad_target is not None and grad_target.numel() != Nf * 3:
        raise ValueError("grad_target must hold Nf*3 values")
    if stream is None:
        stream = torch.cuda.current_stream(target.device).cuda_stream
    prec = tree.precision if precision is None else int(precision)

    def ptr(x):
        return None if x is None else x.data_ptr()

    _lib.check(_lib.lib().pbbfmm_compute_adjoint_device(
        tree._h, target.data_ptr(), Nf, source.data_ptr(), Ns, ptr(weight), g.data_ptr(),
        int(nCols), ptr(grad_weight), ptr(grad_source), ptr(grad_target), prec,
        ctypes.c_void_p(stream)))
