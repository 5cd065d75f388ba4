"""The CUDA path (through the C ABI) against the reference on the two benchmark
configurations the reference can run (golden vectors from tests/golden/make_config_golden.py):

* the 16 x 16 lid-driven cavity, K = 4, Re = 100, dt = 1e-3, from rest: vorticity and
  streamfunction after 1, 10, 100, 1000 and 2000 RK4 steps;
* the 14,625-element backward-facing step, K = 5, Re = 400, pulsatile inlet from t = 1.5:
  one stage and two RK4 steps from a seeded vorticity field, compared on 20,000 seeded
  points per field plus the field's L2 norm and sum.
"""

import json
import os
import sys

import numpy as np
import pytest

from conftest import GOLDEN

from ho2d import FP64, MIXED_KRYLOV, HO_2D, capi

sys.path.insert(0, GOLDEN)
import make_config_golden as CG  # noqa: E402

pytestmark = pytest.mark.gpu

# FP64 device path vs the reference with a direct Poisson solve: the device solve is
# converged to 1e-14 relative residual; differences are that round-off carried through
# the steps
TOL64 = 1e-9
# FP32 Krylov inside FP64 refinement (tolerance 1e-12) over the 2000-step run
TOL_MIXED = 1e-8


def _load(name):
    d = os.path.join(GOLDEN, name)
    return dict(np.load(os.path.join(d, "cfg.npz"))), json.load(open(os.path.join(d, "meta.json")))


def _case(name, tmp_path, meta):
    inp = CG.write_case(name, str(tmp_path / name))
    # the mesh and input the reference read, byte for byte
    assert CG.sha256(inp) == meta["input_sha256"]
    assert CG.sha256(os.path.join(os.path.dirname(inp), "mesh.msh")) == meta["mesh_sha256"]
    return inp


def _solver(inp, precision, tol):
    s = HO_2D()
    s.read_input_file(inp)
    s.set_precision(precision)
    s.set_poisson_tolerance(tol, 5000)
    s.setup()
    return s


def _rel_full(mine, ref):
    return float(np.abs(np.ravel(mine) - ref).max() / max(np.abs(ref).max(), 1e-300))


def _check_sampled(mine, ref, key, tol):
    a = np.ravel(mine)
    idx = ref[key + "__idx"]
    val = ref[key + "__val"]
    scale = max(np.abs(val).max(), 1e-300)
    assert np.abs(a[idx] - val).max() <= tol * scale, (key, np.abs(a[idx] - val).max() / scale)
    l2 = ref[key + "__l2"][0]
    assert abs(np.linalg.norm(a) - l2) <= tol * l2, key
    # the sum cancels: compare it against the field's L1 mass
    assert abs(a.sum() - ref[key + "__sum"][0]) <= tol * np.abs(a).sum(), key


@pytest.mark.parametrize("precision,tol", [(FP64, TOL64), (MIXED_KRYLOV, TOL_MIXED)])
def test_cavity16_2000_steps(tmp_path, precision, tol):
    ref, meta = _load("cfg1_cavity16")
    s = _solver(_case("cfg1_cavity16", tmp_path, meta), precision, 1e-14 if precision == FP64 else 1e-12)
    done = 0
    for step in meta["keep"]:
        s.solve_advection_diffusion(step - done)
        done = step
        assert _rel_full(s.get_vorticity(), ref[f"traj_vort_{step}"]) < tol, step
        assert _rel_full(s.get_streamfunction(), ref[f"traj_psi_{step}"]) < tol, step
    t, dt = s.time()
    assert abs(t - 2000 * dt) < 1e-9


def test_bfs14625_stage_and_steps(tmp_path):
    ref, meta = _load("cfg2_bfs")
    s = _solver(_case("cfg2_bfs", tmp_path, meta), FP64, 1e-14)
    w0 = np.random.Generator(np.random.PCG64(7)).standard_normal((s.N_el, s.Knod, s.Knod))
    s.set_time(meta["t0"])
    s.set_vorticity(w0)
    k = s.Euler_time_integrate(meta["stage_coeff"])
    assert s.poisson_stats()[1] < 1e-13
    for mine, key in [(s.get_streamfunction(), "stage_psi"), (s.get_velocity(), "stage_vel"),
                      (s.get_field(capi.FIELD_RHS_DIFFUSIVE), "stage_rhs_diff"),
                      (s.get_field(capi.FIELD_RHS_ADVECTIVE), "stage_rhs_adv"), (k, "stage_k")]:
        _check_sampled(mine, ref, key, TOL64)
    for which, key in [(capi.BC_VORTICITY, "stage_BC_vorticity"), (capi.BC_VELOCITY_JUMP, "stage_velocity_jump"),
                       (capi.BC_DIFFUSION, "stage_BC_diffusion"), (capi.BC_ADVECTION, "stage_BC_advection"),
                       (capi.BC_NORMAL_VEL, "stage_BC_normal_vel")]:
        assert _rel_full(s.get_boundary(which), ref[key]) < TOL64, key
    for step in meta["keep"]:
        s.solve_advection_diffusion(1)
        _check_sampled(s.get_vorticity(), ref, f"traj_vort_{step}", TOL64)
        _check_sampled(s.get_streamfunction(), ref, f"traj_psi_{step}", TOL64)
