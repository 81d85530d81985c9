"""Host-side logic of the product (no GPU): the C-ABI library loads and exports
every declared symbol, the float64 operator precompute reproduces the
reference's, the reference cache format round-trips, and bad arguments are
rejected with status codes instead of crashing."""
import ctypes
import os
import re

import numpy as np
import pytest

import oracle
import pbbfmm3d_b200 as fmm
from pbbfmm3d_b200 import _lib
from helpers import load_case, make_tree, rel

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    src = open(os.path.join(ROOT, "include", "pbbfmm3d_b200.h")).read()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(pbbfmm_\w+)\s*\(", src, re.M)))


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    names = declared_functions()
    assert len(names) >= 14
    for n in names:
        assert hasattr(L, n), n
    assert set(names) <= set(_lib.EXPORTS), set(names) - set(_lib.EXPORTS)
    assert b"sm_100a" in L.pbbfmm_version()


def test_weights_match_oracle():
    for n in (3, 4, 5, 6):
        for cheb in (0, 1):
            t = fmm.kernel_Laplacian(1.0, 3, n, 1e-5, cheb, device=-1)
            a = t.get_weights()
            b = oracle.compute_weights(n, cheb)
            for x, y in zip(a, b):
                if cheb == 0 and x is a[1]:
                    continue  # Kweights unused for uniform grids
                assert np.array_equal(x, y)
            t.close()


def test_uniform_precompute_matches_reference_operators():
    case = load_case("expcov_unif4")
    m = case["meta"]
    t = make_tree(m["kernel"], m["param"], m["box"], m["level"], m["order"], m["eps"], 0, device=-1)
    t.buildFMMTree()
    ops = t.get_operators()
    assert ops["nlev_ops"] == m["nlev_ops"] == 2
    assert rel(ops["K"], case["K"]) < 1e-12


@pytest.mark.parametrize("name", ["lap_cheb3", "gauss_cheb3", "tps_cheb3_outside"])
def test_chebyshev_precompute_cutoffs_and_operator_range(name):
    """Same SVD cutoffs as the reference; the compressed operators U E_i V^T
    agree up to the truncation level (the kept subspace is only defined up to
    degenerate singular values, so bitwise agreement is not expected)."""
    case = load_case(name)
    m = case["meta"]
    t = make_tree(m["kernel"], m["param"], m["box"], m["level"], m["order"], m["eps"], 1, device=-1)
    t.buildFMMTree()
    ops = t.get_operators()
    assert (ops["rf"], ops["rs"], ops["nlev_ops"]) == (m["rf"], m["rs"], m["nlev_ops"])
    n3 = m["order"] ** 3

    def recon(o, lvl):
        rf, rs = o["rf"], o["rs"]
        U = o["U"][lvl * n3 * rf:(lvl + 1) * n3 * rf].reshape(rf, n3).T
        VT = o["VT"][lvl * rs * n3:(lvl + 1) * rs * n3].reshape(n3, rs).T
        E = o["K"][lvl * 316 * rf * rs:(lvl + 1) * 316 * rf * rs].reshape(316, rs, rf).transpose(0, 2, 1)
        return np.einsum("ia,kab,bj->kij", U, E, VT)

    ref = {"rf": m["rf"], "rs": m["rs"], "U": case["U"], "VT": case["VT"], "K": case["K"]}
    for lvl in range(m["nlev_ops"]):
        assert rel(recon(ops, lvl), recon(ref, lvl)) < 10 * m["eps"]


def test_cache_roundtrip_reference_format(tmp_path):
    t = fmm.kernel_Laplacian(1.0, 3, 3, 1e-4, 1, device=-1)
    t.buildFMMTree(str(tmp_path))
    files = sorted(os.listdir(tmp_path))
    assert files == ["LaplacianChebK3.bin", "LaplacianChebU3.bin", "LaplacianChebV3.bin"]
    a = t.get_operators()
    # the oracle's reader (reference layout) reads what we wrote
    b = oracle.read_reference_cache(str(tmp_path), "Laplacian", 3, 1, 3, True)
    assert a["rf"] == b["rf"] and np.array_equal(a["K"], b["K"]) and np.array_equal(a["U"], b["U"])
    # a second tree reads the cache instead of recomputing
    t2 = fmm.kernel_Laplacian(1.0, 3, 3, 1e-4, 1, device=-1)
    t2.buildFMMTree(str(tmp_path))
    c = t2.get_operators()
    assert np.array_equal(a["K"], c["K"]) and np.array_equal(a["VT"], c["VT"])


def test_nonhomogeneous_cache_is_keyed_on_box_and_level(tmp_path):
    t = fmm.kernel_ExpCov(1.0, 3, 3, 1e-5, 0, ell=0.3, device=-1)
    t.buildFMMTree(str(tmp_path))
    t2 = fmm.kernel_ExpCov(2.0, 3, 3, 1e-5, 0, ell=0.3, device=-1)  # different box: stale
    t2.buildFMMTree(str(tmp_path))
    t3 = fmm.kernel_ExpCov(2.0, 3, 3, 1e-5, 0, ell=0.3, device=-1)
    t3.buildFMMTree()
    assert rel(t2.get_operators()["K"], t3.get_operators()["K"]) < 1e-14


def test_bad_arguments_return_status():
    with pytest.raises(fmm.FMMError) as e:
        fmm.kernel_Laplacian(1.0, 1, 4, 1e-5, 1, device=-1)
    assert e.value.code == _lib.ERR_ARG
    with pytest.raises(fmm.FMMError):
        fmm.kernel_Laplacian(-1.0, 3, 4, 1e-5, 1, device=-1)
    with pytest.raises(fmm.FMMError):
        fmm.kernel_Laplacian(1.0, 3, 11, 1e-5, 1, device=-1)
    with pytest.raises(fmm.FMMError):
        fmm.kernel_ExpCov(1.0, 3, 4, 1e-5, 0, ell=0.0, device=-1)
    t = fmm.kernel_Laplacian(1.0, 3, 3, 1e-4, 1, device=-1)
    with pytest.raises(fmm.FMMError) as e:  # compute before build
        fmm.H2_3D_Compute(t, np.zeros((4, 3)), np.zeros((4, 3)), np.zeros(4), 1, np.zeros(4))
    assert e.value.code == _lib.ERR_STATE
    t.buildFMMTree()
    with pytest.raises(fmm.FMMError) as e:  # host-only tree cannot compute
        fmm.H2_3D_Compute(t, np.zeros((4, 3)), np.zeros((4, 3)), np.zeros(4), 1, np.zeros(4))
    assert e.value.code == _lib.ERR_STATE
    with pytest.raises(ValueError):
        fmm.H2_3D_Compute(t, np.zeros((4, 3)), np.zeros((4, 3)), np.zeros(3), 1, np.zeros(4))
    # wrong operator level count (homogeneous kernel: one level)
    z = np.zeros(5 * 316 * 27 * 27)
    with pytest.raises(fmm.FMMError) as e:
        _lib.check(
            _lib.lib().pbbfmm_tree_set_operators(t._h, 27, 27, 5, fmm._dp(z), fmm._dp(z), fmm._dp(z)))
    assert e.value.code == _lib.ERR_ARG


def test_tensor_core_mode_switch_on_host_tree():
    """pbbfmm_set_tensor_cores takes PBBFMM_TC_OFF / _F16 / _TF32 (1 still
    means on) and refuses other values; a host-only tree has no tensor-core
    operators, so the query reports the CUDA-core path."""
    t = fmm.kernel_Laplacian(1.0, 3, 4, 1e-5, 1, device=-1)
    t.buildFMMTree()
    L = _lib.lib()
    for mode in (_lib.TC_OFF, _lib.TC_F16, _lib.TC_TF32, 1):
        assert L.pbbfmm_set_tensor_cores(t._h, mode) == _lib.OK
    for mode in (-1, 3, 7):
        assert L.pbbfmm_set_tensor_cores(t._h, mode) == _lib.ERR_ARG
    t.set_tensor_cores(True, "tf32")
    t.set_tensor_cores(True, "f16")
    with pytest.raises(ValueError):
        t.set_tensor_cores(True, "bf16")
    assert not t.tensor_core_m2l() and t.tensor_core_format() is None
    # the header's constants are the binding's
    hdr = open(os.path.join(os.path.dirname(__file__), "..", "include", "pbbfmm3d_b200.h")).read()
    for name, val in (("PBBFMM_TC_OFF", _lib.TC_OFF), ("PBBFMM_TC_F16", _lib.TC_F16),
                      ("PBBFMM_TC_TF32", _lib.TC_TF32)):
        assert "#define %s %d" % (name, val) in hdr


def test_operator_cache_failures_return_io_status(tmp_path):
    """The reference exits on operator-file errors (H2_3D_Tree.hpp READ_CHECK);
    here they are statuses: an unwritable cache directory and a truncated
    cache file both give PBBFMM_ERR_IO, and the tree stays usable."""
    t = fmm.kernel_Laplacian(1.0, 3, 3, 1e-4, 1, device=-1)
    with pytest.raises(fmm.FMMError) as e:
        t.buildFMMTree(str(tmp_path / "missing" / "dir"))
    assert e.value.code == _lib.ERR_IO
    (tmp_path / "LaplacianChebK3.bin").write_bytes(b"\x00\x01")  # truncated
    t2 = fmm.kernel_Laplacian(1.0, 3, 3, 1e-4, 1, device=-1)
    with pytest.raises(fmm.FMMError) as e:
        t2.buildFMMTree(str(tmp_path))
    assert e.value.code == _lib.ERR_IO
    t2.buildFMMTree()  # without the cache: computed
    assert t2.get_operators()["rf"] > 0


_EVAL = ctypes.CFUNCTYPE(ctypes.c_double, ctypes.POINTER(ctypes.c_double),
                         ctypes.POINTER(ctypes.c_double), ctypes.c_void_p)
_LAUNCH = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p)


class _UserKernel(ctypes.Structure):
    """pbbfmm_user_kernel (include/pbbfmm3d_b200.h)."""
    _fields_ = [
        ("kernel_type", ctypes.c_char_p),
        ("homogen", ctypes.c_double),
        ("symmetry", ctypes.c_int),
        ("evaluate", _EVAL),
        ("launch_leaf", _LAUNCH),
        ("has_gradient", ctypes.c_int),
        ("ctx", ctypes.c_void_p),
    ]


def _user_tree(kernel, homogen, L=1.0, level=3, order=4, eps=1e-5, cheb=1):
    p = _lib.TreeParams()
    p.L, p.tree_level, p.interpolation_order, p.epsilon, p.use_chebyshev = L, level, order, eps, cheb
    h = ctypes.c_void_p()
    rc = _lib.lib().pbbfmm_tree_create_user(ctypes.byref(p), ctypes.cast(ctypes.byref(kernel),
                                                                        ctypes.c_void_p),
                                            -1, ctypes.byref(h))
    return rc, h


def test_user_kernel_host_precompute_equals_builtin():
    """A user-defined kernel's float64 operators come from its host
    EvaluateKernel (here the Laplacian written in Python through the C ABI's
    evaluate callback): on a host-only tree they equal the built-in
    Laplacian's, since homogen, symmetry and the kernel values agree."""
    import math

    calls = [0]

    def lap(t, s, ctx):
        calls[0] += 1
        dx, dy, dz = s[0] - t[0], s[1] - t[1], s[2] - t[2]
        r = math.sqrt(dx * dx + dy * dy + dz * dz)
        return 1.0 / r if r > 0 else math.inf

    k = _UserKernel()
    k.kernel_type = b"myLaplacian"
    k.homogen, k.symmetry = -1.0, 1
    k.evaluate = _EVAL(lap)
    k.launch_leaf = _LAUNCH(lambda a, s: 0)
    k.has_gradient = 0
    for cheb in (1, 0):
        rc, h = _user_tree(k, -1.0, cheb=cheb)
        assert rc == _lib.OK
        _lib.check(_lib.lib().pbbfmm_tree_build(h, None))
        b = fmm.kernel_Laplacian(1.0, 3, 4, 1e-5, cheb, device=-1)
        b.buildFMMTree()
        ref = b.get_operators()
        u = fmm.H2_3D_Tree.__new__(fmm.H2_3D_Tree)
        u._h, u.interpolation_order, u.use_chebyshev = h, 4, cheb
        ops = u.get_operators()
        assert ops["rf"] == ref["rf"] and ops["nlev_ops"] == ref["nlev_ops"] == 1
        assert np.array_equal(ops["K"], ref["K"])
        u.close()
        b.close()
    assert calls[0] > 0


def test_user_kernel_rejected_without_its_functions():
    k = _UserKernel()
    k.kernel_type = b"x"
    k.homogen, k.symmetry = 0.0, 1
    rc, _ = _user_tree(k, 0.0)  # no evaluate / launch_leaf
    assert rc == _lib.ERR_ARG
    k.evaluate = _EVAL(lambda t, s, c: 1.0)
    k.launch_leaf = _LAUNCH(lambda a, s: 0)
    k.symmetry = 2
    rc, _ = _user_tree(k, 0.0)
    assert rc == _lib.ERR_ARG
