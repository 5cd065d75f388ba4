"""GPU parity of the discrete adjoint, through the C ABI.

The reference has no adjoint; the adjoint is checked against derivatives of the oracle
(pinned to the reference's golden vectors) and of the device's own FP64 forward:
  * transposed Poisson operator = transpose of the oracle's assembled matrix;
  * one stage: dot-product test <lam_k, J v> = <J^T lam_k, v> with J v the complex-step
    derivative of the oracle's stage (ho2d_cs), in the stage input and in BC_parl_vel;
  * several time steps with checkpoint recomputation: the same test on the oracle's
    complex-step derivative of omega(T);
  * central finite differences (h = 1e-6) of J = 0.5 ||omega(T) - target||^2 on the
    device, along seeded directions in (omega0, lid coefficients), to 1e-5 relative;
  * checkpoint intervals, mixed precision, the torch.autograd wrapper, rejected cases.
"""

import os

import numpy as np
import pytest

from conftest import GOLDEN

from ho2d import FP64, MIXED, MIXED_KRYLOV, HO_2D, HO2DError, capi, meshgen

import ho2d_cs as CS
import ho2d_oracle as O

pytestmark = pytest.mark.gpu

CASES = ["cav4_rk4", "cav4_euler_k3", "bfs2_rk4", "cyl4x8_rk4"]  # advection type 1
CASES_ADV2 = ["cavj6_adv2", "cyl4x8_rk2_adv2"]  # advection type 2 (continuous volumetric flux)


def solver_for(inp, precision=FP64, tol=1e-14, max_iter=2000):
    s = HO_2D()
    s.read_input_file(inp)
    s.set_precision(precision)
    s.set_poisson_tolerance(tol, max_iter)
    s.setup()
    return s


def golden_input(name):
    return os.path.join(GOLDEN, name, "input.dat")


def rng_of(seed):
    return np.random.Generator(np.random.PCG64(seed))


@pytest.mark.parametrize("name", CASES)
def test_poisson_transpose_matches_oracle_matrix(name):
    inp = golden_input(name)
    s = solver_for(inp)
    c = O.Case(inp)
    x = rng_of(3).standard_normal(c.N * c.K * c.K)
    y = s.apply_poisson_transpose(x)
    ref = c.A.T @ x
    assert np.linalg.norm(y - ref) <= 1e-12 * np.linalg.norm(ref)


@pytest.mark.parametrize("name,coeff", [(n, 0.0) for n in CASES + CASES_ADV2] +
                         [("bfs2_rk4", 0.5), ("cyl4x8_rk4", 1.0), ("cyl4x8_rk2_adv2", 0.5)])
def test_stage_adjoint_dot_product(name, coeff):
    inp = golden_input(name)
    s = solver_for(inp)
    c = O.Case(inp)
    rng = rng_of(11)
    shape = (c.N, c.K, c.K)
    w = rng.standard_normal(shape)
    lam_k = rng.standard_normal(shape)
    s.setsolnvort_d(w)
    gw, gpv = s.stage_adjoint(coeff, lam_k)
    for trial in range(3):
        dw = rng.standard_normal(shape)
        dpv = rng.standard_normal((c.neb, c.K))
        _, dk = CS.stage_jvp(c, w, dw, dpv, coeff)
        lhs = float(np.vdot(lam_k, dk))
        rhs = float(np.vdot(gw, dw) + np.vdot(gpv, dpv))
        assert abs(lhs - rhs) <= 1e-9 * np.linalg.norm(lam_k) * np.linalg.norm(dk), (trial, lhs, rhs)


@pytest.mark.parametrize("name", CASES + CASES_ADV2)
def test_rollout_gradient_matches_complex_step(name):
    inp = golden_input(name)
    s = solver_for(inp)
    c = O.Case(inp)
    rng = rng_of(21)
    shape = (c.N, c.K, c.K)
    w0 = rng.standard_normal(shape)
    nsteps = 3
    s.setsolnvort_d(w0)
    s.adjoint_forward(nsteps, 2)  # two segments: one recomputed from the checkpoint at step 2
    wT = s.getallvorts_d()
    dJ = rng.standard_normal(shape)
    gw, gpv = s.adjoint_backward(dJ)
    np.testing.assert_array_equal(s.getallvorts_d(), wT)  # the solver is back at T
    assert abs(s.time()[0] - nsteps * c.dt) < 1e-12
    for trial in range(2):
        dw0 = rng.standard_normal(shape)
        dpv = rng.standard_normal((c.neb, c.K))
        wT_o, dwT = CS.run_jvp(c, w0, dw0, dpv, nsteps)
        if trial == 0:
            assert np.linalg.norm(wT - wT_o) <= 1e-10 * np.linalg.norm(wT_o)
        lhs = float(np.vdot(dJ, dwT))
        rhs = float(np.vdot(gw, dw0) + np.vdot(gpv, dpv))
        assert abs(lhs - rhs) <= 1e-8 * np.linalg.norm(dJ) * np.linalg.norm(dwT), (trial, lhs, rhs)


def test_checkpoint_interval_does_not_change_the_gradient():
    inp = golden_input("cav4_rk4")
    rng = rng_of(31)
    out = []
    for every in (1, 3, 5):
        s = solver_for(inp)
        w0 = rng_of(30).standard_normal((s.N_el, s.Knod, s.Knod))
        s.setsolnvort_d(w0)
        s.adjoint_forward(5, every)
        dJ = rng_of(32).standard_normal(w0.shape)
        out.append(s.adjoint_backward(dJ))
    for gw, gpv in out[1:]:
        assert np.linalg.norm(gw - out[0][0]) <= 1e-10 * np.linalg.norm(out[0][0])
        assert np.linalg.norm(gpv - out[0][1]) <= 1e-10 * np.linalg.norm(out[0][1])
    del rng


# HO2D_MIXED_KRYLOV: the same FP64 stages, Poisson round-off only; HO2D_MIXED: the FP32
# stage's trajectory (about 1e-8 from FP64 after 4 steps) as the linearisation point
@pytest.mark.parametrize("prec,tol", [(MIXED_KRYLOV, 1e-8), (MIXED, 1e-6)])
def test_mixed_adjoint_matches_fp64(prec, tol):
    inp = golden_input("bfs2_rk4")
    res = {}
    for p in (FP64, prec):
        s = solver_for(inp, precision=p, tol=1e-12)
        w0 = rng_of(40).standard_normal((s.N_el, s.Knod, s.Knod))
        s.setsolnvort_d(w0)
        s.adjoint_forward(4, 2)
        res[p] = s.adjoint_backward(rng_of(41).standard_normal(w0.shape))
    for a, b in zip(res[prec], res[FP64]):
        assert np.linalg.norm(a - b) <= tol * np.linalg.norm(b)


def test_fp32_state_storage_is_close_to_fp64():
    inp = golden_input("cav4_rk4")
    res = []
    for fp32 in (False, True):
        s = solver_for(inp)
        s.set_adjoint_storage(fp32)
        w0 = rng_of(50).standard_normal((s.N_el, s.Knod, s.Knod))
        s.setsolnvort_d(w0)
        s.adjoint_forward(6, 3)
        res.append(s.adjoint_backward(rng_of(51).standard_normal(w0.shape)))
    for a, b in zip(res[1], res[0]):
        assert np.linalg.norm(a - b) <= 1e-5 * np.linalg.norm(b)


def cavity_problem(tmp_path, n=12, knod=4, reyn=1000.0, steps=10, dt=2e-3):
    """A small version of the differentiation case: seeded sine-mode vorticity, lid
    u(x) = 1 + sum a_m sin(m pi x), target from a second seed."""
    inp = meshgen.make_case(f"cavity{n}", str(tmp_path), knod=knod, steps=steps, dt=dt, reyn=reyn)
    s = solver_for(inp, tol=1e-13)
    xy = s.getsolnpts_d()
    bp = s.get_boundary_points()
    top = s.get_boundary(capi.BC_PARL_VEL) == -1.0  # problem type 1: BC_parl_vel = -1 on the lid
    w0 = meshgen.sine_spectrum(xy, seed=4)
    target = meshgen.sine_spectrum(xy, seed=42)
    a = meshgen.lid_coefficients(seed=41)
    m = np.arange(1, len(a) + 1)
    dpv_da = np.where(top[..., None], -np.sin(np.pi * bp[..., 0, None] * m), 0.0)  # [N_eb][K][modes]

    def pv_of(av):
        return np.where(top, -meshgen.lid_velocity(bp[..., 0], av), 0.0)

    return s, w0, target, a, pv_of, dpv_da


def J_of(s, w0, pv, target, steps):
    s.set_time(0.0)
    s.set_boundary(capi.BC_PARL_VEL, pv)
    s.setsolnvort_d(w0)
    s.solve_advection_diffusion(steps)
    return 0.5 * float(np.sum((s.getallvorts_d() - target) ** 2))


def test_gradient_matches_central_differences(tmp_path):
    steps = 10
    s, w0, target, a, pv_of, dpv_da = cavity_problem(tmp_path, steps=steps)
    s.set_boundary(capi.BC_PARL_VEL, pv_of(a))
    s.setsolnvort_d(w0)
    s.adjoint_forward(steps, 4)
    wT = s.getallvorts_d()
    gw, gpv = s.adjoint_backward(wT - target)
    ga = np.einsum("ekm,ek->m", dpv_da, gpv)
    rng = rng_of(43)
    h = 1e-6
    for _ in range(3):
        dw = rng.standard_normal(w0.shape)
        da = rng.standard_normal(a.shape)
        jp = J_of(s, w0 + h * dw, pv_of(a + h * da), target, steps)
        jm = J_of(s, w0 - h * dw, pv_of(a - h * da), target, steps)
        fd = (jp - jm) / (2 * h)
        ad = float(np.vdot(gw, dw) + np.vdot(ga, da))
        assert abs(fd - ad) <= 1e-5 * abs(ad), (fd, ad)


def test_torch_rollout_matches_the_c_abi(tmp_path):
    torch = pytest.importorskip("torch")
    from ho2d.adjoint import rollout

    steps = 6
    s, w0, target, a, pv_of, _ = cavity_problem(tmp_path, steps=steps)
    pv = pv_of(a)
    w0t = torch.tensor(w0, requires_grad=True)
    pvt = torch.tensor(pv, requires_grad=True)
    wT = rollout(s, w0t, pvt, steps, 3)
    J = 0.5 * ((wT - torch.tensor(target)) ** 2).sum()
    J.backward()
    s.set_time(0.0)
    s.set_boundary(capi.BC_PARL_VEL, pv)
    s.setsolnvort_d(w0)
    s.adjoint_forward(steps, 3)
    gw, gpv = s.adjoint_backward(s.getallvorts_d() - target)
    np.testing.assert_allclose(w0t.grad.numpy(), gw, rtol=0, atol=1e-12 * np.abs(gw).max())
    np.testing.assert_allclose(pvt.grad.numpy(), gpv, rtol=0, atol=1e-12 * np.abs(gpv).max())


def test_adjoint_rejects_what_it_does_not_cover(tmp_path):
    s = solver_for(golden_input("cav4_rk4"))
    with pytest.raises(HO2DError) as e:
        s.adjoint_backward(np.zeros((s.N_el, s.Knod, s.Knod)))
    assert e.value.code == 1
    with pytest.raises(HO2DError) as e:
        s.adjoint_forward(-1, 1)
    assert e.value.code == 1
