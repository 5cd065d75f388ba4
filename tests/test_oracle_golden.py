"""The oracle (numpy restatement) against golden vectors produced by the reference itself."""

import json
import os

import numpy as np
import pytest
import scipy.sparse as sp

from conftest import GOLDEN, GOLDEN_CASES, reference_root

import ho2d_oracle as O

# FP64 restatement vs FP64 reference: only summation order differs
TOL = 1e-11


def rel(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(b).max(), 1e-300))


@pytest.fixture(scope="module", params=GOLDEN_CASES)
def golden(request):
    d = os.path.join(GOLDEN, request.param)
    ref = dict(np.load(os.path.join(d, "ref.npz")))
    meta = json.load(open(os.path.join(d, "meta.json")))
    case = O.Case(os.path.join(d, "input.dat"))
    return request.param, case, ref, meta


def test_mesh_tables(golden):
    _, c, ref, _ = golden
    assert np.array_equal(c.mesh.nbr, ref["elem_neighbor"])
    assert np.array_equal(c.mesh.nbr_side, ref["elem_neighbor_side"])
    assert np.array_equal(c.mesh.bidx, ref["elem_boundary_index"])
    assert np.array_equal(c.mesh.be_el, ref["bedge_element"])
    assert np.array_equal(c.mesh.be_side, ref["bedge_side"])


def test_bases_and_metrics(golden):
    _, c, ref, _ = golden
    assert rel(c.B.xs, ref["sps_local_coor"]) < 1e-14
    assert rel(c.B.w, ref["sps_weight"]) < 1e-14
    assert rel(c.B.D, ref["sps_sps_grad_basis"]) < 1e-13
    assert rel(c.B.gR, ref["sps_grad_radau"]) < 1e-13
    assert rel(c.B.R, ref["sps_radau"]) < 1e-13
    for mine, nm in [(c.M["J"], "vol_jac"), (c.M["G"], "G"), (c.M["GB"], "GB"), (c.M["fJ"], "face_jac"),
                     (c.M["fA"], "face_Acoef"), (c.M["fAn"], "face_Anorm")]:
        assert rel(mine, ref[nm]) < TOL, nm
    # face_Bcoef vanishes on affine meshes: compare absolutely against the face scale
    assert np.abs(c.M["fB"] - ref["face_Bcoef"]).max() <= TOL * np.abs(ref["face_Acoef"]).max()


def test_boundary_conditions(golden):
    _, c, ref, _ = golden
    assert np.array_equal(c.sw_p, ref["BC_switch_Poisson"])
    assert np.array_equal(c.sw_d, ref["BC_switch_diffusion"])
    for mine, nm in [(c.bc_p, "BC_Poisson"), (c.bc_nv, "BC_normal_vel"), (c.bc_pv, "BC_parl_vel"),
                     (c.bc_d, "BC_diffusion")]:
        assert np.abs(mine - ref[nm]).max() <= TOL * max(1.0, np.abs(ref[nm]).max()), nm


def test_poisson_operator(golden):
    _, c, ref, _ = golden
    n = c.N * c.K ** 2
    A = sp.csr_matrix((ref["A_val"], ref["A_col"], ref["A_ptr"][: n + 1]), shape=(n, n))
    assert A.nnz == c.A.nnz
    assert abs(A - c.A).max() <= 1e-13 * abs(A).max()
    assert rel(c.bsrc, ref["boundary_source"]) < 1e-13


def test_one_stage(golden):
    _, c, ref, meta = golden
    c.omega = ref["w0"].copy()
    c.t = 0.0
    k = c.stage(c.omega, meta["stage_coeff"])
    for mine, nm in [(c.psi, "stage_psi"), (c.vel, "stage_vel"), (c.rhs_diff, "stage_rhs_diff"),
                     (c.rhs_adv, "stage_rhs_adv"), (k, "stage_k"), (c.bc_w, "stage_BC_vorticity"),
                     (c.vjump, "stage_velocity_jump"), (c.bc_d, "stage_BC_diffusion"),
                     (c.bc_adv, "stage_BC_advection"), (c.bc_nv, "stage_BC_normal_vel")]:
        scale = max(np.abs(ref[nm]).max(), 1e-12)
        assert np.abs(mine - ref[nm]).max() <= TOL * scale, nm


def test_trajectory(golden):
    name, _, ref, meta = golden
    c = O.Case(os.path.join(GOLDEN, name, "input.dat"))
    c.omega = ref["w0"].copy()
    for s in range(1, meta["steps"] + 1):
        c.step()
        assert rel(c.omega, ref[f"traj_vort_{s}"]) < TOL, s
        assert rel(c.psi, ref[f"traj_psi_{s}"]) < TOL, s


@pytest.mark.parametrize("dat", ["input_cavity.dat", "input_bfs.dat", "input_cylinder.dat"])
def test_oracle_on_shipped_meshes(tmp_path, dat):
    """The reference's own fixtures (input/: quadratic cavity and step, OCC cylinder, K = 3;
    read where they lie, skipped without them): two time steps of the oracle against the
    reference's run (oracle/_ref/ho2d_ref, direct Poisson solve) from the same seeded
    vorticity."""
    import shutil
    import subprocess

    from conftest import REPO

    src = os.path.join(reference_root(), "input")
    ref_bin = os.path.join(REPO, "oracle", "_ref", "ho2d_ref")
    if not (os.path.isdir(src) and os.path.exists(ref_bin)):
        pytest.skip("the reference's input/ directory or oracle/_ref/ho2d_ref is not available")
    lines = open(os.path.join(src, dat)).read().split("\n")
    shutil.copy(os.path.join(src, lines[7].strip()), tmp_path)
    lines[27] = "2"
    inp = str(tmp_path / "input.dat")
    open(inp, "w").write("\n".join(lines))
    c = O.Case(inp)
    w0 = np.random.Generator(np.random.PCG64(7)).standard_normal((c.N, c.K, c.K))
    np.save(tmp_path / "w0.npy", w0)
    subprocess.run([ref_bin, inp, str(tmp_path / "o"), "--init-vort", str(tmp_path / "w0.npy"), "--steps", "2"],
                   check=True, env=dict(os.environ, HO_SHIM_SOLVER="direct"), stdout=subprocess.DEVNULL, timeout=600)
    c.omega = w0
    c.run(2)
    assert rel(c.omega, np.load(tmp_path / "o" / "traj_vort_2.npy")) < TOL
