"""Complex-step derivatives of the oracle's stage and time loop.

TEST INFRASTRUCTURE ONLY -- like ``ho2d_oracle``, this module is a checker; only
``tests/`` may use it. The reference has no adjoint, so the discrete adjoint is checked
against directional derivatives of the oracle (which is itself pinned to the reference's
golden vectors): for a real-analytic map F, Im F(x + i h v) / h equals F'(x) v to
rounding for tiny h (Squire & Trapp, SIAM Review 40, 1998; Martins, Sturdza & Alonso,
ACM TOMS 29, 2003), with no subtraction error. The oracle's stage is analytic in the
vorticity and the wall velocity away from the upwind switch |d omega| = 1e-4 and from a
zero wave speed, where it is piecewise linear; ``ho2d_oracle`` evaluates both tests on
the real part, so a complex argument follows the same branch as the real one.

A tangent u = F'(x) v and an adjoint a = F'(x)^T w pass the dot-product test when
<w, u> = <a, v> to rounding.
"""

from __future__ import annotations

import numpy as np

# Every array of the oracle's Case that a stage reads or writes.
_STATE = ("bc_p", "bc_nv", "bc_pv", "bc_d", "bc_w", "vjump", "bc_adv", "psi", "vel", "omega")
H = 1e-30


def _save(case) -> dict:
    s = {k: np.array(getattr(case, k), copy=True) for k in _STATE}
    s["t"] = case.t
    return s


def _restore(case, s: dict) -> None:
    for k in _STATE:
        setattr(case, k, s[k])
    case.t = s["t"]


def _complexify(case) -> None:
    for k in _STATE:
        setattr(case, k, np.asarray(getattr(case, k), dtype=complex))


def stage_jvp(case, w, dw, dpv=None, coeff: float = 0.0):
    """k and dk for one stage k = stage(w, coeff), in direction dw of the stage input and
    dpv of BC_parl_vel ([N_eb][K]). The case's state is left as it was."""
    saved = _save(case)
    try:
        _complexify(case)
        if dpv is not None:
            case.bc_pv = case.bc_pv + 1j * H * np.asarray(dpv)
        k = case.stage(np.asarray(w) + 1j * H * np.asarray(dw), coeff)
    finally:
        _restore(case, saved)
    return k.real, k.imag / H


def run_jvp(case, w0, dw0, dpv, nsteps: int):
    """omega(T) and its derivative after nsteps time steps from omega0 = w0, in direction
    dw0 of omega0 and dpv of BC_parl_vel. The case's state is left as it was."""
    saved = _save(case)
    try:
        _complexify(case)
        case.bc_pv = case.bc_pv + 1j * H * (np.zeros_like(case.bc_pv) if dpv is None else np.asarray(dpv))
        case.omega = np.asarray(w0, dtype=complex) + 1j * H * np.asarray(dw0)
        case.run(nsteps)
        wT = np.array(case.omega, copy=True)
    finally:
        _restore(case, saved)
    return wT.real, wT.imag / H


def stage_forward_state(case, w, coeff: float = 0.0) -> dict:
    """The stage's intermediate arrays at stage input w (psi, u, v, BC_vorticity,
    BC_normal_vel, ...), as the adjoint's linearisation point; state left as it was."""
    saved = _save(case)
    try:
        k = case.stage(np.asarray(w, dtype=float), coeff)
        out = dict(k=k, psi=case.psi.copy(), u=case.vel[..., 0].copy(), v=case.vel[..., 1].copy(),
                   bc_w=case.bc_w.copy(), bc_nv=case.bc_nv.copy(), bc_d=case.bc_d.copy())
    finally:
        _restore(case, saved)
    return out
