"""CPU checks of the discrete adjoint's element bodies (no GPU).

The bodies of ho-cxx_b200/csrc/adjoint_chain.cuh are compiled for the host by
tests/adjoint_harness.cpp (one thread per element, the GPU launch order) and compared
with the oracle:
  * the transposed Poisson operator against the transpose of the oracle's assembled
    matrix (which is pinned to the reference's own matrix);
  * the adjoint of one stage by the dot-product test <lam_k, J v> = <J^T lam_k, v>, with
    J v the complex-step derivative of the oracle's stage (ho2d_cs) and the transposed
    Poisson solve done by the oracle's LU. The stage is taken at a random vorticity so
    that every face flux and both upwind branches are exercised, for both advection
    schemes (type 1, discontinuous flux; type 2, continuous volumetric flux).
"""

import ctypes
import os
import shutil
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, REPO

import ho2d_cs as CS
import ho2d_oracle as O

CSRC = os.path.join(REPO, "ho-cxx_b200", "csrc")
CASES = ["cav4_rk4", "cav4_euler_k3", "bfs2_rk4", "cyl4x8_rk4"]  # advection type 1
CASES_ADV2 = ["cavj6_adv2", "cyl4x8_rk2_adv2"]  # advection type 2 (continuous volumetric flux)


def _cuda_include():
    for c in (os.environ.get("CUDA_HOME"), "/usr/local/cuda"):
        if c and os.path.isfile(os.path.join(c, "include", "cuda_runtime.h")):
            return os.path.join(c, "include")
    pytest.skip("cuda_runtime.h not found (the harness includes the device structs)")


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    out = str(tmp_path_factory.mktemp("adjoint_harness") / "libadjoint_harness.so")
    src = os.path.join(REPO, "tests", "adjoint_harness.cpp")
    subprocess.run(["g++", "-O1", "-std=c++17", "-shared", "-fPIC", "-I", _cuda_include(), "-I", CSRC, src, "-o", out],
                   check=True, capture_output=True, text=True)
    return ctypes.CDLL(out)


def _p(a, t=ctypes.c_double):
    return a.ctypes.data_as(ctypes.POINTER(t))


class Geom:
    """The oracle case's geometry in the device layout (FrGeom, DevBases)."""

    def __init__(self, c: O.Case):
        K, N, M = c.K, c.N, c.M
        self.K, self.N, self.neb = K, N, c.neb
        self.face_nb = np.ascontiguousarray(np.where(c.f_nbr >= 0, c.f_nbr, -(c.f_bidx + 1)), dtype=np.int32)
        self.face_nijp = np.ascontiguousarray(c.f_nijp, dtype=np.int32)
        self.met = np.concatenate([M[k].ravel() for k in ("xxi", "xeta", "yxi", "yeta", "J")])
        self.fmet = np.concatenate([M[k].ravel() for k in ("fA", "fB", "fJ", "fAn")])
        grp = np.zeros(c.neb, dtype=np.int32)
        for g, (_, ed) in enumerate(c.mesh.groups):
            grp[np.asarray(ed, dtype=int)] = g
        self.be_group = grp
        self.sw_p = np.ascontiguousarray(c.sw_p, dtype=np.int32)
        self.sw_d = np.ascontiguousarray(c.sw_d, dtype=np.int32)
        self.noslip = np.ascontiguousarray(c.noslip, dtype=np.int32)
        B = c.B
        bases = np.zeros(64 + 16 * 4 + 2)
        bases[:K * K] = B.D.ravel()
        for off, arr in ((64, B.sbb), (80, B.sbgb), (96, B.R), (112, B.gR)):
            bases[off:off + 2 * K] = arr.ravel()
        bases[128:130] = B.gp
        self.bases = bases

    def args(self):
        i32 = ctypes.c_int
        return [self.K, self.N, self.neb, _p(self.face_nb, i32), _p(self.face_nijp, i32), _p(self.met), _p(self.fmet),
                _p(self.be_group, i32), _p(self.sw_p, i32), _p(self.sw_d, i32), _p(self.noslip, i32), _p(self.bases)]


def case_of(name):
    return O.Case(os.path.join(GOLDEN, name, "input.dat"))


@pytest.mark.parametrize("name", CASES)
def test_poisson_transpose_matches_assembled_matrix(harness, name):
    c = case_of(name)
    g = Geom(c)
    rng = np.random.default_rng(3)
    x = rng.standard_normal(c.N * c.K * c.K)
    y = np.zeros_like(x)
    assert harness.poisson_transpose_host(*g.args(), _p(x), _p(y)) == 0
    ref = c.A.T @ x
    assert np.linalg.norm(y - ref) <= 1e-12 * np.linalg.norm(ref)


def stage_adjoint(harness, c, g, w, lam_k, coeff=0.0):
    """J^T lam_k of one stage at stage input w: (lam of w, lam of BC_parl_vel)."""
    st = CS.stage_forward_state(c, w, coeff)
    nv = c.N * c.K * c.K
    lw = np.zeros(nv)
    lpsi = np.zeros(nv)
    lpv = np.zeros((c.neb, c.K))
    u, v = np.ascontiguousarray(st["u"]), np.ascontiguousarray(st["v"])
    bw, bnv = np.ascontiguousarray(st["bc_w"]), np.ascontiguousarray(st["bc_nv"])
    wc, lk = np.ascontiguousarray(w, dtype=float), np.ascontiguousarray(lam_k, dtype=float)
    rc = harness.stage_adjoint_host(*g.args(), _p(wc), _p(u), _p(v), _p(bw), _p(bnv), _p(lk),
                                    ctypes.c_double(c.dt), ctypes.c_double(c.re_inv), _p(lw), _p(lpsi), _p(lpv),
                                    ctypes.c_int(c.adv_type))
    assert rc == 0
    mu = c.lu.solve(lpsi, trans="T")  # psi = A^-1 (-J omega - ...): lam_omega -= J A^-T lam_psi
    return lw - c.M["J"].ravel() * mu, lpv


@pytest.mark.parametrize("name", CASES + CASES_ADV2)
def test_stage_adjoint_dot_product(harness, name):
    c = case_of(name)
    g = Geom(c)
    rng = np.random.default_rng(11)
    shape = (c.N, c.K, c.K)
    w = rng.standard_normal(shape)
    lam_k = rng.standard_normal(shape)
    gw, gpv = stage_adjoint(harness, c, g, w, lam_k)
    for trial in range(3):
        dw = rng.standard_normal(shape)
        dpv = rng.standard_normal((c.neb, c.K))
        _, dk = CS.stage_jvp(c, w, dw, dpv)
        lhs = float(np.vdot(lam_k.ravel(), dk.ravel()))
        rhs = float(np.vdot(gw, dw.ravel()) + np.vdot(gpv.ravel(), dpv.ravel()))
        scale = np.linalg.norm(lam_k) * np.linalg.norm(dk) + 1e-300
        assert abs(lhs - rhs) <= 1e-11 * scale, (trial, lhs, rhs)


def test_complex_step_matches_central_differences():
    """The oracle's complex-step tangent agrees with central differences of its stage."""
    c = case_of("cav4_rk4")
    rng = np.random.default_rng(5)
    shape = (c.N, c.K, c.K)
    w = 0.1 * rng.standard_normal(shape)
    dw = rng.standard_normal(shape)
    _, dk = CS.stage_jvp(c, w, dw)
    h = 1e-6
    kp = CS.stage_forward_state(c, w + h * dw)["k"]
    km = CS.stage_forward_state(c, w - h * dw)["k"]
    fd = (kp - km) / (2 * h)
    assert np.linalg.norm(fd - dk) <= 1e-6 * np.linalg.norm(dk)


_SANITIZED_RUN = """
import ctypes, sys
import numpy as np
sys.path[:0] = sys.argv[2:]
import test_adjoint_cpu as T
H = ctypes.CDLL(sys.argv[1])
for name in T.CASES + T.CASES_ADV2:
    c = T.case_of(name)
    g = T.Geom(c)
    rng = np.random.default_rng(11)
    w, lk = rng.standard_normal((c.N, c.K, c.K)), rng.standard_normal((c.N, c.K, c.K))
    for coeff in (0.0, 0.5):
        T.stage_adjoint(H, c, g, w, lk, coeff)
    x = rng.standard_normal(c.N * c.K * c.K)
    y = np.zeros_like(x)
    assert H.poisson_transpose_host(*g.args(), T._p(x), T._p(y)) == 0
print("clean")
"""


def test_element_bodies_under_sanitizers(tmp_path):
    """The adjoint's element bodies (the source the device kernels are compiled from) under
    AddressSanitizer and UBSan on every case of both advection schemes: the stage adjoint at
    two stage coefficients and the transposed Poisson operator. Any report fails the run."""
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    import sys

    so = str(tmp_path / "libadjoint_sanitized.so")
    r = subprocess.run(["g++", "-O1", "-g", "-std=c++17", "-shared", "-fPIC", "-fsanitize=address,undefined",
                        "-fno-omit-frame-pointer", "-I", _cuda_include(), "-I", CSRC,
                        os.path.join(REPO, "tests", "adjoint_harness.cpp"), "-o", so], capture_output=True, text=True)
    if r.returncode != 0 and "sanitize" in r.stderr:
        pytest.skip("sanitizer runtimes not available")
    assert r.returncode == 0, r.stderr[-2000:]
    libs = [subprocess.run(["g++", f"-print-file-name={n}"], capture_output=True, text=True).stdout.strip()
            for n in ("libasan.so", "libubsan.so")]
    if not all(os.path.isabs(p) and os.path.exists(p) for p in libs):
        pytest.skip("sanitizer runtimes not found")
    env = dict(os.environ, LD_PRELOAD=":".join(libs), ASAN_OPTIONS="detect_leaks=0:halt_on_error=1",
               UBSAN_OPTIONS="print_stacktrace=1:halt_on_error=1")
    paths = [os.path.join(REPO, d) for d in ("tests", "oracle", "ho-cxx_b200")]
    r = subprocess.run([sys.executable, "-c", _SANITIZED_RUN, so, *paths], capture_output=True, text=True, env=env,
                       timeout=900)
    assert r.returncode == 0 and "clean" in r.stdout and "runtime error" not in r.stderr, r.stderr[-3000:]
