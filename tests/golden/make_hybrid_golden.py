"""Golden vectors of the reference's hybrid operation (problem type 11).

Writes ``tests/golden/hybrid/<case>/``: the driver's arrays (``spec.txt`` and ``*.npy``, the
input of ``oracle/_ref/ho2d_ref --hybrid``), ``hybrid_ref.npz``, the reference's own
results: the vorticity after each outer ``solveto_d`` step, the solution-point areas and
the open-boundary points, with the shim's direct Poisson solver (HO_SHIM_SOLVER=direct) so
that psi is the converged discrete solution; and ``hybrid_setup_ref.npz``, the reference's
state after ``process_mesh_input`` (mesh tables, Jacobians, boundary conditions: setup_*)
and its normal / parallel split of each open-boundary velocity (open_vel*_end_<step>). Run from the repository root after
``make -C oracle``:

    python tests/golden/make_hybrid_golden.py

Cases (bilinear quads, Knod = 3, RK2, advection type 2 = the hybrid defaults):
  annulus  O-grid r in [0.5, 1.5], 4 x 12 cells; "wall" inside, "open" outside. The driver
           gives potential-flow velocities and a vorticity profile on the open boundary
           (changing between outer steps), a smooth vorticity field to blend in, and
           particle-to-grid weights rising towards the open boundary.
  channel  [0, 3] x [0, 1], 6 x 2 cells; "wall" top and bottom, "inlet" left (normal
           velocity -1 per edge), "outlet" right (+1): psi from the inlet chain.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.abspath(os.path.join(HERE, "..", ".."))
REF = os.path.join(REPO, "oracle", "_ref", "ho2d_ref")
OUT = os.path.join(HERE, "hybrid")
KNOD = 3
GL = np.polynomial.legendre.leggauss(KNOD)[0]


def orient(quads, edges):
    """Each boundary edge as the side (q[s], q[s+1]) of the quad that owns it."""
    side = {}
    for q in quads:
        for s in range(4):
            side[frozenset((int(q[s]), int(q[(s + 1) % 4])))] = (int(q[s]), int(q[(s + 1) % 4]))
    return np.array([side[frozenset((int(a), int(b)))] for a, b in edges], dtype=np.int32)


def solution_points(xy, quads):
    """[el][j][i][x, y] of the bilinear map at the Gauss points (corners SW, SE, NE, NW)."""
    xi = GL[None, :]
    eta = GL[:, None]
    N = [(1 - xi) * (1 - eta) / 4, (1 + xi) * (1 - eta) / 4, (1 + xi) * (1 + eta) / 4, (1 - xi) * (1 + eta) / 4]
    c = xy[quads]  # [el, 4, 2]
    return sum(N[a][None, :, :, None] * c[:, a, None, None, :] for a in range(4))


def edge_points(xy, edges):
    """[edge][k][x, y] along each edge from its first to its second node."""
    t = GL[None, :, None]
    return (1 - t) / 2 * xy[edges[:, 0]][:, None, :] + (1 + t) / 2 * xy[edges[:, 1]][:, None, :]


def annulus():
    nr, nt, r0, r1 = 4, 12, 0.5, 1.5
    r = np.linspace(r0, r1, nr + 1)
    th = np.linspace(0.0, 2 * np.pi, nt, endpoint=False)
    xy = np.array([[ri * np.cos(t), ri * np.sin(t)] for ri in r for t in th])
    idx = lambda i, j: i * nt + (j % nt)  # noqa: E731
    # counter-clockwise: outward, then along increasing theta
    quads = np.array([[idx(i, j), idx(i + 1, j), idx(i + 1, j + 1), idx(i, j + 1)] for i in range(nr) for j in range(nt)],
                     dtype=np.int32)
    inner = orient(quads, [(idx(0, j), idx(0, j + 1)) for j in range(nt)])
    outer = orient(quads, [(idx(nr, j), idx(nr, j + 1)) for j in range(nt)])
    sp = solution_points(xy, quads)
    rr = np.hypot(sp[..., 0], sp[..., 1])
    data = {"nodes": xy.ravel(), "elems": quads.ravel(), "wall": inner.ravel(), "open": outer.ravel(),
            "ptog": np.clip((rr - 1.1) / 0.4, 0.0, 1.0).ravel()}
    op = edge_points(xy, outer)
    ox, oy = op[..., 0], op[..., 1]
    orr2 = ox ** 2 + oy ** 2
    for s in (-1, 0, 1):
        U = 1.0 + 0.1 * (s + 1)
        u = U * (1 - 0.25 * (ox ** 2 - oy ** 2) / orr2 ** 2)
        v = -U * 0.5 * ox * oy / orr2 ** 2
        data[f"openvel_{s}"] = np.stack([u, v], -1).ravel()
        data[f"openvort_{s}"] = (0.2 * (s + 2) * np.sin(np.arctan2(oy, ox))).ravel()
        data[f"vort_{s}"] = (0.5 * (s + 2) * np.sin(2 * sp[..., 0]) * np.cos(sp[..., 1])).ravel()
    spec = {"knod": KNOD, "iorder": 1, "nouter": 2, "numstep": 3, "outerdt": 0.006, "integ": 2, "reyn": 100.0}
    return data, spec


def channel():
    nx, ny, L, H = 6, 2, 3.0, 1.0
    xs, ys = np.linspace(0, L, nx + 1), np.linspace(0, H, ny + 1)
    xy = np.array([[x, y] for y in ys for x in xs])
    idx = lambda i, j: j * (nx + 1) + i  # noqa: E731
    quads = np.array([[idx(i, j), idx(i + 1, j), idx(i + 1, j + 1), idx(i, j + 1)] for j in range(ny) for i in range(nx)],
                     dtype=np.int32)
    bottom = [(idx(i, 0), idx(i + 1, 0)) for i in range(nx)]
    top = [(idx(i + 1, ny), idx(i, ny)) for i in range(nx)]
    left = [(idx(0, j + 1), idx(0, j)) for j in range(ny)]
    right = [(idx(nx, j), idx(nx, j + 1)) for j in range(ny)]
    data = {"nodes": xy.ravel(), "elems": quads.ravel(), "wall": orient(quads, bottom + top).ravel(),
            "inlet": orient(quads, left).ravel(), "inletvel": -np.ones(ny), "outlet": orient(quads, right).ravel(),
            "outletvel": np.ones(ny)}
    spec = {"knod": KNOD, "iorder": 1, "nouter": 2, "numstep": 4, "outerdt": 0.01, "integ": 2, "reyn": 50.0}
    return data, spec


CASES = {"annulus": annulus, "channel": channel}


def write_spec(d, data, spec):
    os.makedirs(d, exist_ok=True)
    with open(os.path.join(d, "spec.txt"), "w") as f:
        for k, v in spec.items():
            f.write(f"{k} {v}\n")
    for k, v in data.items():
        arr = np.ascontiguousarray(v, dtype=np.int32 if k in ("elems", "wall", "open", "inlet", "outlet") else np.float64)
        np.save(os.path.join(d, k + ".npy"), arr)


def make(name):
    data, spec = CASES[name]()
    d = os.path.join(OUT, name)
    if os.path.isdir(d):
        shutil.rmtree(d)
    write_spec(d, data, spec)
    with tempfile.TemporaryDirectory() as tmp:
        # the shim's direct Poisson solver: psi is the converged discrete solution
        env = dict(os.environ, HO_SHIM_SOLVER="direct")
        subprocess.run([REF, "--hybrid", d, tmp], check=True, env=env, stdout=subprocess.DEVNULL)
        out = {f[:-4]: np.load(os.path.join(tmp, f)) for f in os.listdir(tmp) if f.endswith(".npy")}
    setup = {k: v for k, v in out.items() if k.startswith(("setup_", "open_"))}
    run = {k: v for k, v in out.items() if k not in setup}
    np.savez_compressed(os.path.join(d, "hybrid_ref.npz"), **run)
    np.savez_compressed(os.path.join(d, "hybrid_setup_ref.npz"), **setup)
    print(name, {k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    if not os.path.exists(REF):
        sys.exit("oracle/_ref/ho2d_ref is missing: run `make -C oracle` first")
    for nm in CASES:
        make(nm)
