"""The torch.autograd wrapper of the adjoint (ho2d.adjoint) on the CPU, with a stand-in
solver whose rollout is a known linear map omega(T) = A omega0 + B parl_vel and whose
adjoint_backward returns (A^T g, B^T g). Checks the wrapper's plumbing: the calls it makes
and their order, the gradients it returns (against A^T g, B^T g and torch's gradcheck),
that the output does not alias the solver's buffer, and that a second rollout on the same
solver invalidates the first one's backward. The GPU test compares the wrapper with the C
ABI on the real solver.
"""

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from ho2d import capi  # noqa: E402
from ho2d.adjoint import rollout  # noqa: E402


class LinearSolver:
    def __init__(self, N=3, K=2, neb=4, seed=0):
        rng = np.random.Generator(np.random.PCG64(seed))
        self.shape, self.pvshape = (N, K, K), (neb, K)
        n, m = N * K * K, neb * K
        self.A = rng.standard_normal((n, n))
        self.B = rng.standard_normal((n, m))
        self.calls = []
        self.wT = np.zeros(self.shape)

    def set_boundary(self, which, values):
        assert which == capi.BC_PARL_VEL and values.shape == self.pvshape and values.dtype == np.float64
        self.pv = values.copy()
        self.calls.append("set_boundary")

    def setsolnvort_d(self, w):
        assert w.shape == self.shape and w.dtype == np.float64
        self.w0 = w.copy()
        self.calls.append("setsolnvort_d")

    def adjoint_forward(self, nsteps, ckpt_every):
        self.calls.append(("adjoint_forward", nsteps, ckpt_every))
        self.wT[...] = (self.A @ self.w0.ravel() + self.B @ self.pv.ravel()).reshape(self.shape)

    def getallvorts_d(self):
        return self.wT  # the same buffer every time, as a device-backed copy could be

    def adjoint_backward(self, g):
        self.calls.append("adjoint_backward")
        g = np.asarray(g).ravel()
        return (self.A.T @ g).reshape(self.shape), (self.B.T @ g).reshape(self.pvshape)


def inputs(s, seed=1):
    rng = np.random.Generator(np.random.PCG64(seed))
    w0 = torch.tensor(rng.standard_normal(s.shape), requires_grad=True)
    pv = torch.tensor(rng.standard_normal(s.pvshape), requires_grad=True)
    return w0, pv


def test_gradients_are_the_adjoint_map():
    s = LinearSolver()
    w0, pv = inputs(s)
    wT = rollout(s, w0, pv, 7, 3)
    assert s.calls == ["set_boundary", "setsolnvort_d", ("adjoint_forward", 7, 3)]
    np.testing.assert_allclose(wT.detach().numpy(), s.wT)
    g = torch.tensor(np.random.Generator(np.random.PCG64(2)).standard_normal(s.shape))
    (wT * g).sum().backward()
    np.testing.assert_allclose(w0.grad.numpy(), (s.A.T @ g.numpy().ravel()).reshape(s.shape), rtol=1e-14)
    np.testing.assert_allclose(pv.grad.numpy(), (s.B.T @ g.numpy().ravel()).reshape(s.pvshape), rtol=1e-14)
    assert s.calls[-1] == "adjoint_backward"


def test_output_does_not_alias_the_solver_buffer():
    s = LinearSolver()
    w0, pv = inputs(s)
    wT = rollout(s, w0, pv, 1, 1)
    before = wT.detach().clone()
    s.wT[...] = 0.0
    assert torch.equal(wT.detach(), before)


def test_directional_derivative_matches_central_differences():
    """torch.autograd.gradcheck interleaves forward calls with the backward of an earlier
    forward, which the wrapper refuses by design (one rollout in flight per solver); the
    same check done in order: the differences first, then one rollout and its backward."""
    s = LinearSolver(N=2, K=2, neb=2)
    w0, pv = inputs(s, seed=3)
    rng = np.random.Generator(np.random.PCG64(4))
    g = torch.tensor(rng.standard_normal(s.shape))
    dw, dp = torch.tensor(rng.standard_normal(s.shape)), torch.tensor(rng.standard_normal(s.pvshape))
    h = 1e-6
    with torch.no_grad():
        jp = (g * rollout(s, w0 + h * dw, pv + h * dp, 2, 1)).sum()
        jm = (g * rollout(s, w0 - h * dw, pv - h * dp, 2, 1)).sum()
    (g * rollout(s, w0, pv, 2, 1)).sum().backward()
    fd = float((jp - jm) / (2 * h))
    ad = float((w0.grad * dw).sum() + (pv.grad * dp).sum())
    assert abs(fd - ad) <= 1e-8 * max(1.0, abs(ad)), (fd, ad)


def test_a_second_rollout_invalidates_the_first_backward():
    s = LinearSolver()
    w0, pv = inputs(s)
    first = rollout(s, w0, pv, 2, 1)
    rollout(s, w0.detach().clone().requires_grad_(), pv.detach().clone().requires_grad_(), 2, 1)
    with pytest.raises(RuntimeError, match="replaced the checkpoints"):
        first.sum().backward()
