"""The C++ front door (include/pbbfmm3d_b200.hpp): the reference's call
sequence -- kernel_X tree(...); tree.buildFMMTree(); H2_3D_Compute(tree,
target, source, weight, nCols, output) -- compiled with g++ against the
library.  CPU: it compiles and links.  GPU: it runs and agrees with the
float64 direct sum (tolerance 1e-4, the FMM's approximation level)."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "pbbfmm3d_b200")


def _build(tmp_path):
    exe = str(tmp_path / "front_door")
    cmd = ["g++", "-std=c++17", "-O2", os.path.join(ROOT, "tests", "cpp", "front_door.cpp"),
           "-I", os.path.join(ROOT, "include"), "-L", LIBDIR, "-lpbbfmm3d_b200",
           "-Wl,-rpath," + LIBDIR, "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_front_door_compiles_and_links(tmp_path):
    if not os.path.exists(os.path.join(LIBDIR, "libpbbfmm3d_b200.so")):
        pytest.skip("library not built")
    exe = _build(tmp_path)
    r = subprocess.run([exe, "--no-run"], capture_output=True, text=True)
    assert r.returncode == 0 and "linked pbbfmm3d_b200" in r.stdout, r.stdout + r.stderr


@pytest.mark.gpu
def test_front_door_runs(tmp_path):
    exe = _build(tmp_path)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0 and "OK" in r.stdout, r.stdout + r.stderr
