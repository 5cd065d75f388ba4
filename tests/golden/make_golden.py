"""Generate the golden vectors in tests/golden/<case>/ from the reference itself.

The reference (src/HO_2D.cpp, src/Mesh.cpp, unmodified) is built by oracle/Makefile
against the oracle's Eigen/AMGCL API shim into oracle/_ref/ho2d_ref. This script writes
each synthetic case (mesh + input.dat, deterministic), runs the reference with the
shim's direct Poisson solver (HO_SHIM_SOLVER=direct, so psi is the converged discrete
solution) and stores, in ref.npz:

* setup tables: the assembled Poisson matrix (CSR), boundary_source, metrics, BC arrays
  and the mesh neighbour tables;
* one stage (Euler_time_integrate) from a seeded random vorticity field;
* a short trajectory (vorticity and psi after each step).

usage: python tests/golden/make_golden.py [--check-shipped] [case ...]
  case names restrict the run to those cases (default: all).
  --check-shipped additionally runs the oracle against the reference on the meshes
  shipped in the reference's input/ directory and prints the largest differences.
"""

from __future__ import annotations

import json
import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.abspath(os.path.join(HERE, "..", ".."))
sys.path.insert(0, os.path.join(REPO, "ho-cxx_b200"))
sys.path.insert(0, os.path.join(REPO, "oracle"))
from ho2d import meshgen  # noqa: E402

REF = os.path.join(REPO, "oracle", "_ref", "ho2d_ref")


def reference_root() -> str:
    """Root of the reference's sources: $HO2D_REFERENCE, else the build machine's checkout."""
    return os.environ.get("HO2D_REFERENCE") or "/root/reference"

# name: (meshgen case, keyword overrides, knod, steps)
CASES = {
    "cav4_rk4": ("cavity4", {}, 4, 3),
    "cav4_euler_k3": ("cavity4", {"time_integration": 1}, 3, 3),
    "cavj6_adv2": ("cavityj6", {"advection_type": 2}, 4, 3),
    "cyl4x8_rk4": ("cyl4x8", {}, 5, 3),
    "cyl4x8_rk2_adv2": ("cyl4x8", {"time_integration": 2, "advection_type": 2}, 5, 3),
    "bfs2_rk4": ("bfs2", {"x_out": 6.0}, 5, 3),
    "cavq3_rk4": ("cavityq3", {}, 4, 3),  # curved 9-node quads (input Lnod 2)
}
SEED = 7
SETUP_ARRAYS = ["A_ptr", "A_col", "A_val", "boundary_source", "vol_jac", "G", "GB", "face_Acoef", "face_Bcoef",
                "face_jac", "face_Anorm", "BC_Poisson", "BC_normal_vel", "BC_parl_vel", "BC_diffusion",
                "BC_switch_Poisson", "BC_switch_diffusion", "elem_neighbor", "elem_neighbor_side",
                "elem_boundary_index", "bedge_element", "bedge_side", "sps_local_coor", "sps_weight",
                "sps_radau", "sps_grad_radau", "sps_sps_grad_basis", "sps_boundary_basis",
                "sps_boundary_grad_basis"]
STAGE_ARRAYS = ["stage_psi", "stage_vel", "stage_rhs_diff", "stage_rhs_adv", "stage_k", "stage_BC_vorticity",
                "stage_velocity_jump", "stage_BC_diffusion", "stage_BC_advection", "stage_BC_normal_vel"]


def run_ref(inp, out, *args):
    env = dict(os.environ, HO_SHIM_SOLVER="direct")
    subprocess.run([REF, inp, out, *args], check=True, env=env, stdout=subprocess.DEVNULL)


def make_case(name: str) -> None:
    mcase, kw, knod, steps = CASES[name]
    cdir = os.path.join(HERE, name)
    if os.path.isdir(cdir):
        shutil.rmtree(cdir)
    inp = meshgen.make_case(mcase, cdir, knod=knod, steps=steps, **kw)
    with tempfile.TemporaryDirectory() as tmp:
        meta_dir = os.path.join(tmp, "setup")
        run_ref(inp, meta_dir, "--setup")
        meta = json.load(open(os.path.join(meta_dir, "meta.json")))
        n, k = meta["N_el"], meta["Knod"]
        w0 = np.random.Generator(np.random.PCG64(SEED)).standard_normal((n, k, k))
        w0_path = os.path.join(tmp, "w0.npy")
        np.save(w0_path, w0)
        stage_dir = os.path.join(tmp, "stage")
        run_ref(inp, stage_dir, "--init-vort", w0_path, "--stage", "0.5")
        traj_dir = os.path.join(tmp, "traj")
        run_ref(inp, traj_dir, "--init-vort", w0_path, "--steps", str(steps), "--every", "1")
        data = {"w0": w0}
        for a in SETUP_ARRAYS:
            p = os.path.join(meta_dir, a + ".npy")
            if os.path.exists(p):
                data[a] = np.load(p)
        for a in STAGE_ARRAYS:
            data[a] = np.load(os.path.join(stage_dir, a + ".npy"))
        for s in range(1, steps + 1):
            data[f"traj_vort_{s}"] = np.load(os.path.join(traj_dir, f"traj_vort_{s}.npy"))
            data[f"traj_psi_{s}"] = np.load(os.path.join(traj_dir, f"traj_psi_{s}.npy"))
        np.savez_compressed(os.path.join(cdir, "ref.npz"), **data)
        meta.pop("setup_seconds", None)
        meta.update(steps=steps, seed=SEED, stage_coeff=0.5)
        with open(os.path.join(cdir, "meta.json"), "w") as f:
            json.dump(meta, f, indent=1)
    print(f"{name}: N_el={n} K={k} -> {cdir}")


def check_shipped() -> None:
    import ho2d_oracle as O

    src_dir = os.path.join(reference_root(), "input")
    for dat in ("input_cavity.dat", "input_bfs.dat", "input_cylinder.dat"):
        with tempfile.TemporaryDirectory() as tmp:
            lines = open(os.path.join(src_dir, dat)).read().split("\n")
            shutil.copy(os.path.join(src_dir, lines[7].strip()), tmp)
            lines[3] = "2"
            lines[27] = "2"
            inp = os.path.join(tmp, "input.dat")
            open(inp, "w").write("\n".join(lines))
            c = O.Case(inp)
            w0 = np.random.Generator(np.random.PCG64(SEED)).standard_normal((c.N, c.K, c.K))
            np.save(os.path.join(tmp, "w0.npy"), w0)
            run_ref(inp, os.path.join(tmp, "o"), "--init-vort", os.path.join(tmp, "w0.npy"), "--steps", "2")
            c.omega = w0
            c.run(2)
            ref = np.load(os.path.join(tmp, "o", "traj_vort_2.npy"))
            print(f"{dat}: N_el={c.N} rel. max |omega - omega_ref| after 2 steps = "
                  f"{np.abs(c.omega - ref).max() / np.abs(ref).max():.2e}")


if __name__ == "__main__":
    if not os.path.exists(REF):
        sys.exit("oracle/_ref/ho2d_ref is missing: run `make -C oracle` first")
    names = [a for a in sys.argv[1:] if not a.startswith("--")] or list(CASES)
    for nm in names:
        make_case(nm)
    if "--check-shipped" in sys.argv:
        check_shipped()
