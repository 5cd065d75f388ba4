"""VTK and sample-point output against the reference's own files.

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

from conftest import GOLDEN, REPO, reference_root

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
                                                                ("output_host.cpp", "host_io.cpp", "host_setup.cpp",
                                                                 "host_samples.cpp", "host_kron.cpp")]
    subprocess.run(["g++", "-O1", "-std=c++17", "-shared", "-fPIC", "-I", csrc, "-I", os.path.join(REPO, "include"),
                    *srcs, "-o", out], check=True, capture_output=True, text=True)
    lib = ctypes.CDLL(out)
    lib.sample_points_host.restype = ctypes.c_long
    return lib


@pytest.mark.parametrize("case", ["cav4_rk4", "cav4_euler_k3", "bfs2_rk4", "cyl4x8_rk4", "cavq3_rk4"])
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
                                    str(ours).encode(), b"")
    assert rc == 0
    files = sorted(os.listdir(ours))
    assert files == [f"problem{ptype}_K{knod}_{nsteps:05d}.vtk", f"vorticity{ptype}_K{knod}_{nsteps:05d}.vtk"]
    for fn in files:  # identical except for round-off around zero (summation order)
        compare_vtk(str(ours / fn), str(d / fn))
    # the time loop's dumps go through VtkQueue's thread: the same bytes, for two dumps in a row
    queued = tmp_path / "queued"
    queued.mkdir()
    rc = vtk_harness.write_vtk_queued_host(str(d / "mesh.msh").encode(), 0, knod, ptype, _dp(f["vorticity"]),
                                           _dp(f["psi"]), _dp(f["vel"][..., 0]), _dp(f["vel"][..., 1]),
                                           _dp(f["rhs_diff"]), _dp(f["rhs_adv"]), _dp(f["bc_w"]), _dp(f["bc_nv"]),
                                           _dp(f["bc_pv"]), nsteps, str(queued).encode(), b"")
    assert rc == 0
    assert sorted(os.listdir(queued)) == sorted(files + [fn.replace(f"{nsteps:05d}", f"{nsteps + 1:05d}")
                                                         for fn in files])
    for fn in os.listdir(queued):
        src = fn.replace(f"{nsteps + 1:05d}", f"{nsteps:05d}")
        assert open(queued / fn).read() == open(ours / src).read(), fn


def q2_cavity(n=3, amp=0.04):
    from ho2d import meshgen

    return meshgen.cavity_q2(n, amp)


def msh_nodes(path):
    """Node coordinates of a Gmsh 4.1 file written by meshgen or the golden generator."""
    lines = open(path).read().split("\n")
    i = lines.index("$Nodes")
    nb, n = int(lines[i + 1].split()[0]), int(lines[i + 1].split()[1])
    k, xy = i + 2, []
    for _ in range(nb):
        cnt = int(lines[k].split()[3])
        xy += [[float(t) for t in lines[k + 1 + cnt + a].split()[:2]] for a in range(cnt)]
        k += 1 + 2 * cnt
    assert len(xy) == n
    return np.array(xy)


@pytest.mark.parametrize("case", ["cav4_rk4", "bfs2_rk4", "cyl4x8_rk4", "q2_cavity"])
def test_sample_point_file_matches_reference(tmp_path, vtk_harness, case):
    """read_process_sample_points + the sample-point file of save_smooth_vtk: 40 seeded
    points in the mesh's bounding box, some outside the domain (the BFS step, the cylinder,
    the box corners), so that both the polygon search and the nearest-node fallback run.
    The reference (--solve --samples) and the library's writer, given the fields the
    reference wrote from, must write the same file (values to the printed six digits), and
    every point's shape functions must sum to one."""
    if not os.path.exists(REF):
        pytest.skip("oracle/_ref/ho2d_ref not built")
    from ho2d import meshgen

    d = tmp_path / "case"
    if case == "q2_cavity":
        d.mkdir()
        meshgen.write_msh(q2_cavity(), str(d / "mesh.msh"))
        meshgen.write_input_dat(str(d / "input.dat"), "mesh.msh", knod=4, reyn=100.0, dt=1e-3, num_steps=2,
                                problem_type=1, lnod_in=2)
    else:
        shutil.copytree(os.path.join(GOLDEN, case), d)
    lines = open(d / "input.dat").read().split("\n")
    assert lines[-3] == "sample_points file"
    lines[-2] = "samples.dat"
    open(d / "input.dat", "w").write("\n".join(lines))
    xy = msh_nodes(str(d / "mesh.msh"))
    lo, hi = xy.min(axis=0), xy.max(axis=0)
    rng = np.random.Generator(np.random.PCG64(7))
    pts = lo - 0.02 * (hi - lo) + rng.random((40, 2)) * 1.04 * (hi - lo)
    with open(d / "samples.dat", "w") as f:
        for x, y in pts:
            f.write(f"{x:.17g} {y:.17g}\n")
    env = dict(os.environ, HO_SHIM_SOLVER="direct")
    subprocess.run([REF, str(d / "input.dat"), str(tmp_path / "fields"), "--solve", "--samples"], check=True, env=env,
                   stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL, timeout=300)
    f = {k: np.load(tmp_path / "fields" / f"solve_{k}.npy") for k in
         ("vorticity", "psi", "vel", "rhs_diff", "rhs_adv", "bc_w", "bc_nv", "bc_pv")}
    knod, lnod_in, ptype, nsteps = int(lines[3]), int(lines[5]), int(lines[25]), int(lines[27])
    ours = tmp_path / "ours"
    ours.mkdir()
    rc = vtk_harness.write_vtk_host(str(d / "mesh.msh").encode(), 0, knod, ptype, _dp(f["vorticity"]),
                                    _dp(f["psi"]), _dp(f["vel"][..., 0]), _dp(f["vel"][..., 1]), _dp(f["rhs_diff"]),
                                    _dp(f["rhs_adv"]), _dp(f["bc_w"]), _dp(f["bc_nv"]), _dp(f["bc_pv"]), nsteps, -1,
                                    str(ours).encode(), str(d / "samples.dat").encode())
    assert rc == 0
    name = f"sampling_points{ptype}_K{knod}_L{lnod_in + 1}_{nsteps:05d}.dat"
    assert os.path.exists(d / name) and os.path.exists(ours / name)
    compare_vtk(str(ours / name), str(d / name))
    assert len(open(ours / name).read().split("\n")) == len(pts) + 1
    # the points outside the domain took the nearest-node fallback
    L2 = (lnod_in + 1) ** 2
    elem, shape = np.zeros(64, np.int32), np.zeros(64 * L2)
    n = vtk_harness.sample_points_host(str(d / "mesh.msh").encode(), 0, str(d / "samples.dat").encode(),
                                       elem.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), _dp(shape), 64)
    assert n == len(pts)
    sh = shape[: n * L2].reshape(n, L2)
    np.testing.assert_allclose(sh.sum(axis=1), 1.0, atol=1e-12)  # a partition of unity
    assert elem[:n].min() >= 0


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


def test_sample_points_of_the_shipped_cavity(tmp_path, vtk_harness):
    """The reference's shipped cavity input (2,895 quadratic quads) with its own
    sample-points file (input/sample_points.dat, points on the centrelines; read where they
    lie, skipped without them), two time steps: the library's writer reproduces the
    reference's sampling_points file and both VTK files from the fields the reference wrote
    them from."""
    src = os.path.join(reference_root(), "input")
    if not (os.path.isdir(src) and os.path.exists(REF)):
        pytest.skip("the reference's input/ directory or oracle/_ref/ho2d_ref is not available")
    d = tmp_path / "case"
    d.mkdir()
    lines = open(os.path.join(src, "input_cavity.dat")).read().split("\n")
    for f in (lines[7].strip(), "sample_points.dat"):
        shutil.copy(os.path.join(src, f), d)
    lines[27], lines[31] = "2", "2"  # two steps, files at steps 0 and 2
    open(d / "input.dat", "w").write("\n".join(lines))
    env = dict(os.environ, HO_SHIM_SOLVER="direct")
    subprocess.run([REF, str(d / "input.dat"), str(tmp_path / "fields"), "--solve", "--samples"], check=True, env=env,
                   stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL, timeout=600)
    f = {k: np.load(tmp_path / "fields" / f"solve_{k}.npy") for k in
         ("vorticity", "psi", "vel", "rhs_diff", "rhs_adv", "bc_w", "bc_nv", "bc_pv")}
    knod, ptype = int(lines[3]), int(lines[25])
    ours = tmp_path / "ours"
    ours.mkdir()
    rc = vtk_harness.write_vtk_host(str(d / lines[7].strip()).encode(), int(lines[9]), knod, ptype,
                                    _dp(f["vorticity"]), _dp(f["psi"]), _dp(f["vel"][..., 0]), _dp(f["vel"][..., 1]),
                                    _dp(f["rhs_diff"]), _dp(f["rhs_adv"]), _dp(f["bc_w"]), _dp(f["bc_nv"]),
                                    _dp(f["bc_pv"]), 2, -1, str(ours).encode(), str(d / "sample_points.dat").encode())
    assert rc == 0
    names = [n for n in os.listdir(d) if n.startswith("sampling_points") and n.endswith("_00002.dat")]
    assert len(names) == 1, os.listdir(d)
    compare_vtk(str(ours / names[0]), str(d / names[0]))
    assert len(open(ours / names[0]).read().split()) == 5 * 14  # 14 points, 5 values each
    for vtk in (f"problem{ptype}_K{knod}_00002.vtk", f"vorticity{ptype}_K{knod}_00002.vtk"):  # 9-node quads
        compare_vtk(str(ours / vtk), str(d / vtk))


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["cavq3_rk4", "bfs2_rk4", "cyl4x8_rk4"])
def test_device_node_values_write_the_host_files(tmp_path, case, monkeypatch):
    """The smooth file's node averages and sample values made on the device (the default)
    give byte-identical files to the host writer's (HO2D_HOST_OUTPUT=1), sample points
    included; the vorticity file is written from the same fields either way."""
    from ho2d import HO_2D

    d = tmp_path / "case"
    shutil.copytree(os.path.join(GOLDEN, case), d)
    lines = open(d / "input.dat").read().split("\n")
    idx = next(i for i, ln in enumerate(lines) if ln.startswith("sample_points file"))
    lines[idx + 1] = "samples.dat"
    open(d / "input.dat", "w").write("\n".join(lines))
    rng = np.random.Generator(np.random.PCG64(9))
    pts = rng.uniform(-0.2, 1.2, size=(12, 2))  # some outside the domain: the nearest-node fallback
    np.savetxt(d / "samples.dat", pts)
    out = {}
    for host in ("0", "1"):
        monkeypatch.setenv("HO2D_HOST_OUTPUT", host)
        o = tmp_path / f"out{host}"
        o.mkdir()
        s = HO_2D()
        s.read_input_file(str(d / "input.dat"))
        s.setup()
        s.set_output_dir(str(o))
        s.solve_vorticity_streamfunction()
        s.trigger_write(99, 1, str(o))
        s.close()
        out[host] = o
    names = sorted(os.listdir(out["0"]))
    assert names == sorted(os.listdir(out["1"]))
    assert any(n.startswith("sampling_points") for n in names) and any(n.startswith("problem") for n in names)
    for n in names:
        assert open(out["0"] / n, "rb").read() == open(out["1"] / n, "rb").read(), n
