"""VTK output against the reference's own files.

CPU: the library's writer (host build, tests/vtk_harness.cpp) fed the fields the reference
wrote its last files from must write the same files (on the cavity cases byte for byte;
elsewhere values of round-off size around zero differ with the summation order).
GPU:
The reference (oracle/_ref/ho2d_ref --solve: solve_vorticity_streamfunction with its VTK
writers, direct Poisson solve) and ho2d_solve with an output directory run the same golden
case; both write vorticity<p>_K<K>_<step>.vtk and problem<p>_K<K>_<step>.vtk at the dump
steps. The files must have the same lines and words; numbers agree to the printed six
significant digits (relative 2e-5, plus 1e-8 of the file's largest value for values that
are round-off around zero).
"""

import ctypes
import os
import shutil
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, REPO

REF = os.path.join(REPO, "oracle", "_ref", "ho2d_ref")


def _num(t):
    try:
        return float(t)
    except ValueError:
        return None


def compare_vtk(a_path, b_path):
    a = open(a_path).read().split("\n")
    b = open(b_path).read().split("\n")
    assert len(a) == len(b), (a_path, len(a), len(b))
    vals = [abs(x) for line in a for t in line.split() if (x := _num(t)) is not None and np.isfinite(x)]
    scale = max(vals) if vals else 1.0
    worst = 0.0
    for la, lb in zip(a, b):
        ta, tb = la.split(), lb.split()
        assert len(ta) == len(tb), (la, lb)
        for x, y in zip(ta, tb):
            fx, fy = _num(x), _num(y)
            if fx is None or fy is None:
                assert x == y, (la, lb)
            else:
                d = abs(fx - fy)
                assert d <= 2e-5 * max(abs(fx), abs(fy)) + 1e-8 * scale, (la, lb)
                worst = max(worst, d / (abs(fx) + 1e-8 * scale))
    return worst


def _dp(a):
    return np.ascontiguousarray(a, dtype=np.float64).ctypes.data_as(ctypes.POINTER(ctypes.c_double))


@pytest.fixture(scope="module")
def vtk_harness(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    csrc = os.path.join(REPO, "ho-cxx_b200", "csrc")
    out = str(tmp_path_factory.mktemp("vtk_harness") / "libvtk_harness.so")
    srcs = [os.path.join(REPO, "tests", "vtk_harness.cpp")] + [os.path.join(csrc, f) for f in
                                                                ("output_host.cpp", "host_io.cpp", "host_setup.cpp")]
    subprocess.run(["g++", "-O1", "-std=c++17", "-shared", "-fPIC", "-I", csrc, "-I", os.path.join(REPO, "include"),
                    *srcs, "-o", out], check=True, capture_output=True, text=True)
    return ctypes.CDLL(out)


@pytest.mark.parametrize("case", ["cav4_rk4", "cav4_euler_k3", "bfs2_rk4", "cyl4x8_rk4"])
def test_vtk_writer_reproduces_reference_files(tmp_path, vtk_harness, case):
    """The library's writer, given the fields the reference wrote its last files from,
    writes the same files (host build; the reference run on the CPU)."""
    if not os.path.exists(REF):
        pytest.skip("oracle/_ref/ho2d_ref not built")
    d = tmp_path / "case"
    shutil.copytree(os.path.join(GOLDEN, case), d)
    env = dict(os.environ, HO_SHIM_SOLVER="direct")
    subprocess.run([REF, str(d / "input.dat"), str(tmp_path / "fields"), "--solve"], check=True, env=env,
                   stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
    f = {k: np.load(tmp_path / "fields" / f"solve_{k}.npy") for k in
         ("vorticity", "psi", "vel", "rhs_diff", "rhs_adv", "bc_w", "bc_nv", "bc_pv")}
    lines = open(d / "input.dat").read().split("\n")
    knod, ptype, nsteps = int(lines[3]), int(lines[25]), int(lines[27])
    ours = tmp_path / "ours"
    ours.mkdir()
    rc = vtk_harness.write_vtk_host(str(d / "mesh.msh").encode(), 0, knod, ptype, _dp(f["vorticity"]),
                                    _dp(f["psi"]), _dp(f["vel"][..., 0]), _dp(f["vel"][..., 1]), _dp(f["rhs_diff"]),
                                    _dp(f["rhs_adv"]), _dp(f["bc_w"]), _dp(f["bc_nv"]), _dp(f["bc_pv"]), nsteps, -1,
                                    str(ours).encode())
    assert rc == 0
    files = sorted(os.listdir(ours))
    assert files == [f"problem{ptype}_K{knod}_{nsteps:05d}.vtk", f"vorticity{ptype}_K{knod}_{nsteps:05d}.vtk"]
    for fn in files:  # identical except for round-off around zero (summation order)
        compare_vtk(str(ours / fn), str(d / fn))


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["cav4_rk4", "bfs2_rk4", "cyl4x8_rk4"])
def test_vtk_files_match_reference(tmp_path, case):
    if not os.path.exists(REF):
        pytest.skip("oracle/_ref/ho2d_ref not built")
    from ho2d import HO_2D

    d = tmp_path / "case"
    shutil.copytree(os.path.join(GOLDEN, case), d)
    env = dict(os.environ, HO_SHIM_SOLVER="direct")
    subprocess.run([REF, str(d / "input.dat"), str(tmp_path / "refout"), "--solve"], check=True, env=env,
                   stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
    ref_files = sorted(f for f in os.listdir(d) if f.endswith(".vtk"))
    assert len(ref_files) >= 4
    ours = tmp_path / "ours"
    ours.mkdir()
    s = HO_2D()
    s.read_input_file(str(d / "input.dat"))
    s.set_poisson_tolerance(1e-14, 2000)
    s.setup()
    s.set_output_dir(str(ours))
    s.solve_vorticity_streamfunction()
    assert sorted(os.listdir(ours)) == ref_files
    for f in ref_files:
        compare_vtk(str(ours / f), str(d / f))
