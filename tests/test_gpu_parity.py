"""CUDA path (through the C ABI) against the reference's golden vectors and the oracle."""

import json
import os

import numpy as np
import pytest

from conftest import GOLDEN, GOLDEN_CASES

from ho2d import FP64, MIXED, MIXED_KRYLOV, HO_2D, capi, meshgen

import ho2d_oracle as O

pytestmark = pytest.mark.gpu

# FP64 device path vs FP64 reference: the Poisson solve is converged to 1e-14 relative
# residual, so results agree to solver round-off times the operator's conditioning.
TOL64 = 1e-9


def rel(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(b).max(), 1e-300))


def solver_for(inp, precision=FP64, tol=1e-14, max_iter=2000):
    s = HO_2D()
    s.read_input_file(inp)
    s.set_precision(precision)
    s.set_poisson_tolerance(tol, max_iter)
    s.setup()
    return s


def golden(case):
    d = os.path.join(GOLDEN, case)
    return os.path.join(d, "input.dat"), dict(np.load(os.path.join(d, "ref.npz"))), json.load(
        open(os.path.join(d, "meta.json")))


@pytest.mark.parametrize("case", GOLDEN_CASES)
def test_poisson_operator_matches_reference_matrix(case):
    """The matrix-free device operator reproduces the reference's assembled matrix."""
    import scipy.sparse as sp

    inp, ref, _ = golden(case)
    s = solver_for(inp)
    n = s.N_el * s.Knod ** 2
    A = sp.csr_matrix((ref["A_val"], ref["A_col"], ref["A_ptr"][: n + 1]), shape=(n, n))
    rng = np.random.Generator(np.random.PCG64(5))
    for _ in range(3):
        x = rng.standard_normal(n)
        y = s.apply_poisson(x.reshape(s.N_el, s.Knod, s.Knod)).ravel()
        ya = A @ x
        # the reference drops |a| <= 1e-14 entries; everything else is round-off
        assert np.abs(y - ya).max() <= 1e-12 * np.abs(ya).max()


@pytest.mark.parametrize("case", GOLDEN_CASES)
def test_stage_matches_reference(case):
    inp, ref, meta = golden(case)
    s = solver_for(inp)
    s.set_vorticity(ref["w0"])
    k = s.Euler_time_integrate(meta["stage_coeff"])
    it, res = s.poisson_stats()
    assert res < 1e-13
    checks = [
        (s.get_streamfunction(), "stage_psi"),
        (s.get_velocity(), "stage_vel"),
        (s.get_field(capi.FIELD_RHS_DIFFUSIVE), "stage_rhs_diff"),
        (s.get_field(capi.FIELD_RHS_ADVECTIVE), "stage_rhs_adv"),
        (k, "stage_k"),
        (s.get_boundary(capi.BC_VORTICITY), "stage_BC_vorticity"),
        (s.get_boundary(capi.BC_VELOCITY_JUMP), "stage_velocity_jump"),
        (s.get_boundary(capi.BC_DIFFUSION), "stage_BC_diffusion"),
        (s.get_boundary(capi.BC_ADVECTION), "stage_BC_advection"),
        (s.get_boundary(capi.BC_NORMAL_VEL), "stage_BC_normal_vel"),
    ]
    for mine, nm in checks:
        scale = max(np.abs(ref[nm]).max(), 1e-12)
        assert np.abs(mine - ref[nm]).max() <= TOL64 * scale, (nm, rel(mine, ref[nm]))


@pytest.mark.parametrize("case", GOLDEN_CASES)
def test_trajectory_matches_reference(case):
    inp, ref, meta = golden(case)
    s = solver_for(inp)
    s.set_vorticity(ref["w0"])
    for step in range(1, meta["steps"] + 1):
        s.solve_advection_diffusion(1)
        assert rel(s.get_vorticity(), ref[f"traj_vort_{step}"]) < TOL64, step
        assert rel(s.get_streamfunction(), ref[f"traj_psi_{step}"]) < TOL64, step
    t, dt = s.time()
    assert abs(t - meta["steps"] * dt) < 1e-12


def test_solve_and_solveto_match_steps():
    inp, ref, meta = golden("cav4_rk4")
    s = solver_for(inp)
    s.set_vorticity(ref["w0"])
    s.solve_vorticity_streamfunction()  # num_time_steps = 3 from input.dat
    assert rel(s.get_vorticity(), ref["traj_vort_3"]) < TOL64
    s2 = solver_for(inp)
    s2.set_vorticity(ref["w0"])
    _, dt = s2.time()
    s2.solveto_d(3 * dt, 3, 4, 100.0)
    assert rel(s2.get_vorticity(), ref["traj_vort_3"]) < TOL64


# K = 2..8: the reference stops at K = 5 (src/HO_2D.cpp:522-525), the oracle does not; K < 4
# runs the operator's general form, K >= 4 the register-resident one, K = 8 is the maximum
@pytest.mark.parametrize("name,knod,steps,kw", [
    ("cavityj10", 5, 4, {}),
    ("cyl6x12", 4, 4, {"advection_type": 2}),
    ("bfs3", 3, 3, {"x_out": 4.0}),
    ("cavityj8", 2, 3, {}),
    ("cyl6x12", 6, 2, {}),
    ("cavityj8", 7, 2, {"advection_type": 2}),
    ("cavityj6", 8, 2, {}),
])
def test_against_oracle(tmp_path, name, knod, steps, kw):
    inp = meshgen.make_case(name, str(tmp_path), knod=knod, steps=steps, **kw)
    c = O.Case(inp)
    rng = np.random.Generator(np.random.PCG64(11))
    w0 = rng.standard_normal((c.N, c.K, c.K))
    c.omega = w0.copy()
    c.run(steps)
    s = solver_for(inp)
    s.set_vorticity(w0)
    s.solve_advection_diffusion(steps)
    assert rel(s.get_vorticity(), c.omega) < TOL64
    assert rel(s.get_streamfunction(), c.psi) < TOL64
    assert rel(s.get_velocity(), c.vel) < TOL64


def test_mixed_precision_close_to_fp64(tmp_path):
    inp = meshgen.make_case("cavityj8", str(tmp_path), knod=4, steps=5)
    ref = solver_for(inp)
    mix = solver_for(inp, precision=MIXED, tol=1e-12)
    ref.solve_advection_diffusion(20)
    mix.solve_advection_diffusion(20)
    w64, w32 = ref.get_vorticity(), mix.get_vorticity()
    err = np.linalg.norm(w32 - w64) / np.linalg.norm(w64)
    assert err < 1e-4, err
    it, res = mix.poisson_stats()
    assert res < 1e-11


def test_mixed_krylov_matches_fp64(tmp_path):
    # FP64 FR stage with the FP32 Krylov inside FP64 refinement: the only difference from
    # FP64 is the Poisson solve's round-off below its 1e-12 tolerance
    inp = meshgen.make_case("cavityj8", str(tmp_path), knod=4, steps=5)
    ref = solver_for(inp, tol=1e-12)
    mix = solver_for(inp, precision=MIXED_KRYLOV, tol=1e-12)
    ref.solve_advection_diffusion(20)
    mix.solve_advection_diffusion(20)
    w64, w32 = ref.get_vorticity(), mix.get_vorticity()
    err = np.linalg.norm(w32 - w64) / np.linalg.norm(w64)
    assert err < 1e-9, err
    assert mix.poisson_stats()[1] < 1e-11


def test_nonfinite_vorticity_rejected(tmp_path):
    inp = meshgen.make_case("cavity4", str(tmp_path), knod=3, steps=1)
    s = solver_for(inp)
    w = np.zeros((s.N_el, s.Knod, s.Knod))
    w[0, 0, 0] = np.nan
    with pytest.raises(capi.HO2DError) as e:
        s.set_vorticity(w)
    assert e.value.code == 7


# every shape of the coarse hierarchy -- P0 + dense level (default), a dense P0 level,
# three levels with a grid-wide up step -- and plain block-Jacobi converge to the same
# streamfunction (3,600 elements)
@pytest.mark.parametrize("env", [{}, {"HO2D_DENSE_MAX": "100"}, {"HO2D_DENSE_MAX": "5000"},
                                 {"HO2D_PRECOND": "bj"}])
def test_preconditioner_layouts_agree_with_oracle(tmp_path, monkeypatch, env):
    for k, v in env.items():
        monkeypatch.setenv(k, v)
    inp = meshgen.make_case("cavityj60", str(tmp_path), knod=3, steps=2)
    c = O.Case(inp)
    rng = np.random.Generator(np.random.PCG64(5))
    w0 = rng.standard_normal((c.N, c.K, c.K))
    c.omega = w0.copy()
    c.run(2)
    s = solver_for(inp, max_iter=5000)
    s.set_vorticity(w0)
    s.solve_advection_diffusion(2)
    assert rel(s.get_streamfunction(), c.psi) < TOL64
    assert rel(s.get_vorticity(), c.omega) < TOL64


def test_body_force_matches_restatement(tmp_path):
    # the device sum against the same force integral restated from the mesh geometry and the
    # exported boundary arrays; orientation here comes from the element centroid instead of
    # the element's counter-clockwise traversal used by the library
    inp = meshgen.make_case("cyl6x12", str(tmp_path), knod=4, steps=2)
    s = solver_for(inp)
    rng = np.random.Generator(np.random.PCG64(21))
    s.set_vorticity(rng.standard_normal((s.N_el, s.Knod, s.Knod)))
    s.solve_advection_diffusion(2)
    fx, fy = s.forces()
    c = O.Case(inp)
    K, L, B = c.K, c.L, c.B
    w_wall = s.get_boundary(capi.BC_VORTICITY).reshape(-1, K)
    dwdn = s.get_boundary(capi.BC_DIFFUSION).reshape(-1, K)
    gx = np.linspace(-1.0, 1.0, L)
    nu = 1.0 / 100.0
    ref = np.zeros(2)
    edges = dict(c.mesh.groups)["object"]
    for e in edges:
        el, side = int(c.mesh.be_el[e]), int(c.mesh.be_side[e])
        ijp = int(O.F2I[side])
        Xe = c.X[el]
        centroid = Xe.reshape(-1, 2).mean(0)
        for k in range(K):
            a = B.xs[k]
            xi, eta = {0: (-1.0, a), 1: (1.0, a), 2: (a, -1.0), 3: (a, 1.0)}[ijp]
            lx, dlx = O.lagrange(gx, [xi])
            ly, dly = O.lagrange(gx, [eta])
            pos = np.einsum("j,i,jic->c", ly[:, 0], lx[:, 0], Xe)
            if ijp < 2:
                tan = np.einsum("j,i,jic->c", dly[:, 0], lx[:, 0], Xe)
            else:
                tan = np.einsum("j,i,jic->c", ly[:, 0], dlx[:, 0], Xe)
            length = np.linalg.norm(tan)
            n = np.array([-tan[1], tan[0]]) / length
            if n @ (centroid - pos) < 0:
                n = -n
            t = np.array([-n[1], n[0]])  # z x n
            idx = (side // 2) * (K - 2 * k - 1) + k
            dn = (1.0 if ijp % 2 == 0 else -1.0) * dwdn[e, idx]
            om = w_wall[e, idx]
            ds = nu * B.w[k] * length
            ref += ds * np.array([pos[1] * dn + om * t[0], -pos[0] * dn + om * t[1]])
    scale = max(np.abs(ref).max(), 1e-300)
    assert abs(fx - ref[0]) <= 1e-10 * scale and abs(fy - ref[1]) <= 1e-10 * scale, (fx, fy, ref)
