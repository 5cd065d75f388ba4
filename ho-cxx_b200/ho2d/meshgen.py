"""Synthetic quad meshes in Gmsh 4.1 ASCII, and HO-CXX ``input.dat`` files.

The reference reads every case from a ``.msh`` file (its built-in mesher returns an
error, src/Mesh.cpp:836 with src/main.cpp:49-53), so the seeded benchmark and test
geometries are written here in the subset of Gmsh 4.1 that ``Mesh::read_msh_file``
accepts (src/Mesh.cpp:93-340):

* ``$PhysicalNames`` with dimension-1 names only (the reader mis-parses any other
  dimension, src/Mesh.cpp:126-127);
* ``$Entities`` with one curve per named boundary (tag, bounding box, one physical
  tag), src/Mesh.cpp:141-152;
* ``$Nodes``: one block, tags 1..N;
* ``$Elements``: 2-node lines (type 1) per boundary curve and 4-node quads (type 3)
  listed counter-clockwise, so the reader needs no OCC reorientation (flag 0); or, for
  quadratic geometry (input.dat Lnod 2), 3-node lines (type 8: ends, then midpoint) and
  9-node quads (type 10: corners, edge midpoints, centre).

Physical names follow the problem types of src/HO_2D.cpp:675-1238: cavity
(``bottom_wall, right_wall, top, left_wall``), backward-facing step
(``inlet, outlet, top, bottom``) and flow over a cylinder
(``object, inlet, outlet``). Random jitter uses ``numpy.random.Generator(PCG64(seed))``
on interior nodes only.
"""

from __future__ import annotations

import math
import os
from dataclasses import dataclass, field

import numpy as np


@dataclass
class QuadMesh:
    xy: np.ndarray  # [n_nodes, 2]
    quads: np.ndarray  # [n_el, 4] node indices, counter-clockwise (or [n_el, 9], Gmsh order)
    boundaries: dict = field(default_factory=dict)  # name -> [n_edges, 2] node indices (or [n_edges, 3])

    @property
    def n_el(self) -> int:
        return int(self.quads.shape[0])


def _grid_block(nx: int, ny: int, fx, fy):
    """Node coordinates of an (nx+1) x (ny+1) logical grid, x = fx(i), y = fy(j)."""
    ii, jj = np.meshgrid(np.arange(nx + 1), np.arange(ny + 1), indexing="xy")
    return np.stack([fx(ii), fy(jj)], axis=-1)  # [ny+1, nx+1, 2]


def _quads_of_block(ids: np.ndarray) -> np.ndarray:
    """CCW quads (SW, SE, NE, NW) from a [ny+1, nx+1] node-id array."""
    sw = ids[:-1, :-1]
    se = ids[:-1, 1:]
    ne = ids[1:, 1:]
    nw = ids[1:, :-1]
    return np.stack([sw, se, ne, nw], axis=-1).reshape(-1, 4)


def _jitter(xy: np.ndarray, interior: np.ndarray, amp: float, seed: int | None) -> np.ndarray:
    if amp <= 0.0:
        return xy
    rng = np.random.Generator(np.random.PCG64(seed))
    out = xy.copy()
    d = rng.uniform(-amp, amp, size=xy.shape)
    out[interior] += d[interior]
    return out


def cavity(n: int, jitter: float = 0.0, seed: int | None = None) -> QuadMesh:
    """Unit-square lid-driven cavity, n x n uniform quads, interior jitter +/- jitter*h."""
    h = 1.0 / n
    g = _grid_block(n, n, lambda i: i * h, lambda j: j * h)
    ids = np.arange((n + 1) * (n + 1)).reshape(n + 1, n + 1)
    xy = g.reshape(-1, 2)
    interior = np.zeros(len(xy), dtype=bool)
    interior[ids[1:-1, 1:-1].ravel()] = True
    xy = _jitter(xy, interior, jitter * h, seed)
    quads = _quads_of_block(ids)
    bnd = {
        "bottom_wall": np.stack([ids[0, :-1], ids[0, 1:]], axis=1),
        "right_wall": np.stack([ids[:-1, -1], ids[1:, -1]], axis=1),
        "top": np.stack([ids[-1, 1:], ids[-1, :-1]], axis=1)[::-1],
        "left_wall": np.stack([ids[1:, 0], ids[:-1, 0]], axis=1)[::-1],
    }
    return QuadMesh(xy, quads, bnd)


def cavity_q2(n: int, amp: float = 0.04) -> QuadMesh:
    """Unit-square cavity of n x n 9-node (quadratic) quads whose interior is bent by
    (x, y) += amp sin(pi x) sin(2 pi y) (1, 0.5): curved interior edges, straight walls.
    Nodes in Gmsh order per quad (corners SW, SE, NE, NW, the edge midpoints, the centre);
    boundary edges as (end, end, midpoint)."""
    m = 2 * n + 1
    g = np.linspace(0.0, 1.0, m)
    X, Y = np.meshgrid(g, g)  # [j][i]
    b = amp * np.sin(np.pi * X) * np.sin(2 * np.pi * Y)
    xy = np.stack([(X + b).ravel(), (Y + 0.5 * b).ravel()], -1)

    def nid(i, j):
        return j * m + i

    quads = []
    for j in range(n):
        for i in range(n):
            a, c = 2 * i, 2 * j
            quads.append([nid(a, c), nid(a + 2, c), nid(a + 2, c + 2), nid(a, c + 2), nid(a + 1, c), nid(a + 2, c + 1),
                          nid(a + 1, c + 2), nid(a, c + 1), nid(a + 1, c + 1)])
    bnd = {"bottom_wall": [[nid(2 * i, 0), nid(2 * i + 2, 0), nid(2 * i + 1, 0)] for i in range(n)],
           "right_wall": [[nid(m - 1, 2 * j), nid(m - 1, 2 * j + 2), nid(m - 1, 2 * j + 1)] for j in range(n)],
           "top": [[nid(2 * i + 2, m - 1), nid(2 * i, m - 1), nid(2 * i + 1, m - 1)] for i in range(n)],
           "left_wall": [[nid(0, 2 * j + 2), nid(0, 2 * j), nid(0, 2 * j + 1)] for j in range(n)]}
    return QuadMesh(xy, np.array(quads), {k: np.array(v) for k, v in bnd.items()})


def backward_facing_step(h: float = 1.0 / 15.0, jitter: float = 0.15, seed: int | None = 2,
                         x_in: float = -5.0, x_out: float = 30.0) -> QuadMesh:
    """Backward-facing step: step height 1, expansion ratio 2.

    Upstream channel x in [x_in, 0], y in [0, 1]; downstream x in [0, x_out],
    y in [-1, 1]. With h = 1/15: 75x15 + 450x30 = 14,625 quads. Names follow
    problem_type 2: inlet (x = x_in), outlet (x = x_out), top (y = 1), bottom (the
    upstream floor, the step face and the downstream floor).
    """
    nu_x = int(round(-x_in / h))
    nd_x = int(round(x_out / h))
    n1 = int(round(1.0 / h))
    up = _grid_block(nu_x, n1, lambda i: x_in + i * h, lambda j: j * h)
    dn = _grid_block(nd_x, 2 * n1, lambda i: i * h, lambda j: -1.0 + j * h)
    up_ids = np.arange((n1 + 1) * (nu_x + 1)).reshape(n1 + 1, nu_x + 1)
    base = up_ids.size
    dn_ids = np.full((2 * n1 + 1, nd_x + 1), -1, dtype=np.int64)
    # downstream column i=0, rows j >= n1 coincide with upstream column nu_x
    dn_ids[n1:, 0] = up_ids[:, nu_x]
    fresh = dn_ids < 0
    dn_ids[fresh] = base + np.arange(int(fresh.sum()))
    xy = np.zeros((base + int(fresh.sum()), 2))
    xy[up_ids.ravel()] = up.reshape(-1, 2)
    xy[dn_ids[fresh]] = dn[fresh]
    boundary_nodes = np.zeros(len(xy), dtype=bool)
    for arr in (up_ids[0, :], up_ids[-1, :], up_ids[:, 0], dn_ids[0, :], dn_ids[-1, :], dn_ids[:, -1],
                dn_ids[: n1 + 1, 0]):
        boundary_nodes[arr] = True
    xy = _jitter(xy, ~boundary_nodes, jitter * h, seed)
    quads = np.concatenate([_quads_of_block(up_ids), _quads_of_block(dn_ids)])
    bottom = np.concatenate([
        np.stack([up_ids[0, :-1], up_ids[0, 1:]], axis=1),                    # upstream floor, +x
        np.stack([dn_ids[1: n1 + 1, 0], dn_ids[:n1, 0]], axis=1)[::-1],       # step face, -y
        np.stack([dn_ids[0, :-1], dn_ids[0, 1:]], axis=1),                    # downstream floor, +x
    ])
    top = np.concatenate([
        np.stack([dn_ids[-1, 1:], dn_ids[-1, :-1]], axis=1)[::-1],
        np.stack([up_ids[-1, 1:], up_ids[-1, :-1]], axis=1)[::-1],
    ])
    bnd = {
        "inlet": np.stack([up_ids[1:, 0], up_ids[:-1, 0]], axis=1)[::-1],
        "outlet": np.stack([dn_ids[:-1, -1], dn_ids[1:, -1]], axis=1),
        "top": top,
        "bottom": bottom,
    }
    return QuadMesh(xy, quads, bnd)


def cylinder_ogrid(n_r: int = 256, n_theta: int = 512, r0: float = 0.5, r1: float = 20.0,
                   stretch: float = 1.02, square: bool = False) -> QuadMesh:
    """O-grid around a cylinder: radial spacing dr_k = dr0 * stretch**k from r0 to r1.

    Names follow problem_type 3: ``object`` (r = r0), ``inlet`` (outer arc, edge
    midpoint x < 0) and ``outlet`` (outer arc, x >= 0).

    With ``square`` the rings blend from the circle at r0 to the square of half-width r1
    (weight ((r - r0) / (r1 - r0))^2 on the square's radial scaling), so the outer boundary
    is the box [-r1, r1]^2 with its sides named as problem type 3's channel expects:
    ``inlet`` (x = -r1), ``outlet`` (x = r1), ``top`` and ``bottom``. n_theta must be a
    multiple of 8 (box corners on nodes).
    """
    if square and n_theta % 8:
        raise ValueError("square outer boundary needs n_theta divisible by 8")
    if abs(stretch - 1.0) < 1e-14:
        radii = np.linspace(r0, r1, n_r + 1)
    else:
        dr0 = (r1 - r0) * (stretch - 1.0) / (stretch ** n_r - 1.0)
        radii = r0 + dr0 * (stretch ** np.arange(n_r + 1) - 1.0) / (stretch - 1.0)
        radii[-1] = r1
    theta = 2.0 * np.pi * np.arange(n_theta) / n_theta
    # ids[j, i]: j radial ring, i azimuth (periodic)
    ids = np.arange((n_r + 1) * n_theta).reshape(n_r + 1, n_theta)
    rr, tt = np.meshgrid(radii, theta, indexing="ij")
    scale = np.ones_like(rr)
    if square:
        w = ((rr - r0) / (r1 - r0)) ** 2
        scale = (1.0 - w) + w / np.maximum(np.abs(np.cos(tt)), np.abs(np.sin(tt)))
    xy = np.stack([rr * scale * np.cos(tt), rr * scale * np.sin(tt)], axis=-1).reshape(-1, 2)
    idsp = np.concatenate([ids, ids[:, :1]], axis=1)  # wrap in azimuth
    # azimuth increases CCW: (i along theta) x (j along r) would be clockwise, so use
    # xi = radial, eta = azimuthal: SW=(j,i), SE=(j+1,i), NE=(j+1,i+1), NW=(j,i+1)
    sw = idsp[:-1, :-1]
    se = idsp[1:, :-1]
    ne = idsp[1:, 1:]
    nw = idsp[:-1, 1:]
    quads = np.stack([sw, se, ne, nw], axis=-1).reshape(-1, 4)
    inner = np.stack([idsp[0, 1:], idsp[0, :-1]], axis=1)      # domain on the left when walking
    outer = np.stack([idsp[-1, :-1], idsp[-1, 1:]], axis=1)
    mid_x = 0.5 * (xy[outer[:, 0], 0] + xy[outer[:, 1], 0])
    if not square:
        bnd = {"object": inner, "inlet": outer[mid_x < 0.0], "outlet": outer[mid_x >= 0.0]}
        return QuadMesh(xy, quads, bnd)
    mid_y = 0.5 * (xy[outer[:, 0], 1] + xy[outer[:, 1], 1])
    side = np.abs(mid_x) >= np.abs(mid_y)
    bnd = {"object": inner, "inlet": outer[side & (mid_x < 0.0)], "outlet": outer[side & (mid_x >= 0.0)],
           "top": outer[~side & (mid_y > 0.0)], "bottom": outer[~side & (mid_y <= 0.0)]}
    return QuadMesh(xy, quads, bnd)


def cylinder_channel(n_r: int = 48, n_theta: int = 96, r0: float = 0.5, x_in: float = -15.0, x_out: float = 45.0,
                     half_h: float = 15.0, stretch: float = 1.04) -> QuadMesh:
    """O-grid from a cylinder at the origin (radius r0) out to the channel
    [x_in, x_out] x [-half_h, half_h], at uniform azimuth (as ``cylinder_ogrid``). x_in
    and x_out are moved to the nearest values that put the channel's corners on azimuthal
    nodes, so every boundary edge lies on one side. Ring j sits at r_j along each ray,
    blended from the circle to the channel boundary with weight ((r_j - r0) / (R - r0))^2,
    R = half_h, r_j growing geometrically by ``stretch``. Names follow problem type 3's
    channel: ``object``, ``inlet`` (x = x_in), ``outlet`` (x = x_out), ``top``,
    ``bottom``."""
    dth = 2.0 * np.pi / n_theta
    k_out = max(1, int(round(math.atan2(half_h, x_out) / dth)))
    k_in = max(1, int(round(math.atan2(half_h, -x_in) / dth)))
    x_out = half_h / math.tan(k_out * dth)
    x_in = -half_h / math.tan(k_in * dth)
    theta = dth * np.arange(n_theta)
    c, sn = np.cos(theta), np.sin(theta)
    with np.errstate(divide="ignore"):
        tx = np.where(c > 0, x_out / np.where(c > 0, c, 1.0), np.where(c < 0, x_in / np.where(c < 0, c, 1.0), np.inf))
        ty = np.where(sn != 0, half_h / np.abs(np.where(sn != 0, sn, 1.0)), np.inf)
    dist = np.minimum(tx, ty)  # distance from the centre to the channel boundary along each ray
    R = half_h
    dr0 = (R - r0) * (stretch - 1.0) / (stretch ** n_r - 1.0)
    radii = r0 + dr0 * (stretch ** np.arange(n_r + 1) - 1.0) / (stretch - 1.0)
    radii[-1] = R
    w = ((radii - r0) / (R - r0)) ** 2
    rr = radii[:, None] * ((1.0 - w)[:, None] + w[:, None] * (dist / R)[None, :])
    xy = np.stack([rr * c[None, :], rr * sn[None, :]], axis=-1).reshape(-1, 2)
    ids = np.arange((n_r + 1) * n_theta).reshape(n_r + 1, n_theta)
    idsp = np.concatenate([ids, ids[:, :1]], axis=1)
    quads = np.stack([idsp[:-1, :-1], idsp[1:, :-1], idsp[1:, 1:], idsp[:-1, 1:]], axis=-1).reshape(-1, 4)
    inner = np.stack([idsp[0, 1:], idsp[0, :-1]], axis=1)
    outer = np.stack([idsp[-1, :-1], idsp[-1, 1:]], axis=1)
    mid = 0.5 * (xy[outer[:, 0]] + xy[outer[:, 1]])
    tol = 1e-9 * max(abs(x_in), x_out, half_h)
    bnd = {"object": inner, "inlet": outer[np.abs(mid[:, 0] - x_in) < tol],
           "outlet": outer[np.abs(mid[:, 0] - x_out) < tol], "top": outer[np.abs(mid[:, 1] - half_h) < tol],
           "bottom": outer[np.abs(mid[:, 1] + half_h) < tol]}
    return QuadMesh(xy, quads, bnd)


def write_msh(mesh: QuadMesh, path: str) -> None:
    """Write ``mesh`` as Gmsh 4.1 ASCII readable by the reference's reader."""
    names = list(mesh.boundaries.keys())
    n_nodes = len(mesh.xy)
    lines = ["$MeshFormat", "4.1 0 8", "$EndMeshFormat", "$PhysicalNames", str(len(names))]
    for g, nm in enumerate(names):
        lines.append(f'1 {g + 1} "{nm}"')
    lines += ["$EndPhysicalNames", "$Entities", f"0 {len(names)} 1 0"]
    for g, nm in enumerate(names):
        e = mesh.boundaries[nm]
        p = mesh.xy[np.unique(e.ravel())]
        lo, hi = p.min(axis=0), p.max(axis=0)
        lines.append(f"{g + 1} {lo[0]:.17g} {lo[1]:.17g} 0 {hi[0]:.17g} {hi[1]:.17g} 0 1 {g + 1} 0")
    lo, hi = mesh.xy.min(axis=0), mesh.xy.max(axis=0)
    lines.append(f"1 {lo[0]:.17g} {lo[1]:.17g} 0 {hi[0]:.17g} {hi[1]:.17g} 0 0 0")
    lines += ["$EndEntities", "$Nodes", f"1 {n_nodes} 1 {n_nodes}", f"2 1 0 {n_nodes}"]
    lines += [str(i + 1) for i in range(n_nodes)]
    lines += [f"{x:.17g} {y:.17g} 0" for x, y in mesh.xy]
    n_edges = sum(len(v) for v in mesh.boundaries.values())
    n_elem = n_edges + mesh.n_el
    lines += ["$EndNodes", "$Elements", f"{len(names) + 1} {n_elem} 1 {n_elem}"]
    quadratic = mesh.quads.shape[1] == 9
    tag = 1
    for g, nm in enumerate(names):
        e = mesh.boundaries[nm]
        lines.append(f"1 {g + 1} {8 if quadratic else 1} {len(e)}")
        for ed in e:
            lines.append(f"{tag} " + " ".join(str(int(a) + 1) for a in ed))
            tag += 1
    lines.append(f"2 1 {10 if quadratic else 3} {mesh.n_el}")
    for q in mesh.quads:
        lines.append(f"{tag} " + " ".join(str(int(a) + 1) for a in q))
        tag += 1
    lines.append("$EndElements")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def write_input_dat(path: str, mesh_file: str, knod: int, reyn: float, dt: float, num_steps: int,
                    problem_type: int, time_integration: int = 4, advection_type: int = 1,
                    dump_frequency: int | None = None, occ: int = 0, lhs_type: int = 3,
                    sample_points: str = "none", lnod_in: int = 1) -> None:
    """Write the 17-field positional ``input.dat`` (src/HO_2D.cpp:213-317); ``lnod_in`` is
    the geometry order (1 bilinear, 2 quadratic)."""
    if dump_frequency is None:
        dump_frequency = max(num_steps, 1)
    fields = [
        ("Nel_i , Nel_j:", "1, 1"),
        ("Knod quantity:", str(knod)),
        ("Lnod:", str(lnod_in)),
        ("mesh file name:", mesh_file),
        ("if the file is written in OCC format or original gmsh format. zero means original, 1 means OCC format",
         str(occ)),
    ]
    body = []
    for c, v in fields:
        body += [c, v]
    body += ["Exact", "false"]
    rest = [
        ("Reyn", repr(float(reyn))),
        ("dx ratio : expanding mesh ratio. For Gmsh reading option it is not used.", "1."),
        ("fac:  multiplier to make grids randomly non-uniform; uniform: fac=0", "0."),
        ("Huyn solver: for now only the option 2 is used which is the DG equivalence", "2"),
        ("time integration: 1: explicit Euler, 2: explicit RK2, 4: explicit RK4", str(time_integration)),
        ("advection scheme: 1: original discontinuous, 2: continuous mass flux term", str(advection_type)),
        ("problem type. 1 is lid-driven cavity, 2 is BFS, 3 is flow over cylinder", str(problem_type)),
        ("number of time steps", str(num_steps)),
        ("dt: time step size", repr(float(dt))),
        ("dumpfreq: how many time steps are the results saved", str(dump_frequency)),
        ("fast: if it uses large stencil or compact stencil. fast-true means compact. It is not setup yet in the code",
         "0"),
        ("linear solver type: 1:Eigen, 2: Hypre, 3: AMGCL. The HYPRE is not setup yet.", str(lhs_type)),
        ("sample_points file", sample_points),
    ]
    for c, v in rest:
        body += [c, v]
    with open(path, "w") as f:
        f.write("\n".join(body) + "\n")


def min_edge_length(mesh: QuadMesh) -> float:
    q = mesh.quads
    d = [np.linalg.norm(mesh.xy[q[:, (k + 1) % 4]] - mesh.xy[q[:, k]], axis=1) for k in range(4)]
    return float(np.min(d))


def cfl_dt(mesh: QuadMesh, knod: int, u_max: float, cfl: float = 0.5) -> float:
    """dt = cfl * h_min / (u_max * K^2): the explicit FR step bound used for the benchmark cases."""
    return cfl * min_edge_length(mesh) / (u_max * knod * knod)


def viscous_dt(mesh: QuadMesh, knod: int, reyn: float, c: float = 1.5) -> float:
    """dt = c * h_min^2 * Re / K^4: the diffusive bound of explicit RK4 on the FR Laplacian.

    On strongly stretched meshes (the cylinder O-grid's first radial cell is h/2500) it is
    far below the CFL bound; measured on the 256 x 512 O-grid at K = 6, Re = 100, steps up
    to about 3x this value are stable and 6x blow up."""
    h = min_edge_length(mesh)
    return c * h * h * reyn / float(knod) ** 4


# Named cases: (mesh builder, problem_type, Re, velocity scale for the CFL dt)
def sine_spectrum(xy: np.ndarray, seed: int, modes: int = 4) -> np.ndarray:
    """Seeded smooth cavity vorticity: sum_{m,n=1..modes} c_mn sin(m pi x) sin(n pi y) with
    c_mn ~ N(0, 1) / (m^2 + n^2), evaluated at points xy[..., 2] of the unit square (the
    sine modes vanish on its walls)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    m = np.arange(1, modes + 1)
    c = rng.standard_normal((modes, modes)) / (m[:, None] ** 2 + m[None, :] ** 2)
    sx = np.sin(np.pi * xy[..., 0, None] * m)  # [..., modes]
    sy = np.sin(np.pi * xy[..., 1, None] * m)
    return np.einsum("...m,...n,mn->...", sx, sy, c)


def lid_coefficients(seed: int, modes: int = 4, sigma: float = 0.05) -> np.ndarray:
    """a_m ~ N(0, sigma^2) of the lid profile u(x) = 1 + sum_m a_m sin(m pi x)."""
    return np.random.Generator(np.random.PCG64(seed)).normal(0.0, sigma, modes)


def lid_velocity(x: np.ndarray, a: np.ndarray) -> np.ndarray:
    """u(x) = 1 + sum_m a_m sin(m pi x)."""
    m = np.arange(1, len(a) + 1)
    return 1.0 + np.sin(np.pi * np.asarray(x)[..., None] * m) @ np.asarray(a)


def make_case(name: str, outdir: str, knod: int | None = None, steps: int = 10, dt: float | None = None,
              **kw) -> str:
    """Write ``<outdir>/input.dat`` and its mesh for a named synthetic case; returns the input path.

    Cases: ``cavity<N>`` (uniform N x N cavity, Re=100, K=4, dt=1e-3), ``cavityq<N>``
    (N x N curved 9-node quads, cavity_q2),
    ``cavityj<N>`` (jittered +/-0.1h), ``bfs`` (the 14,625-quad step, K=5, Re=400,
    CFL-0.5 dt), ``bfs<m>`` (step with h = 1/m), ``cyl<nr>x<nt>`` (O-grid, K=5, Re=100).
    The step is the smaller of the CFL and the viscous bound (cfl_dt, viscous_dt).
    """
    os.makedirs(outdir, exist_ok=True)
    if name.startswith("cavityq"):
        n = int(name[7:])
        mesh = cavity_q2(n, amp=kw.get("amp", 0.04))
        ptype, reyn, k = 1, kw.get("reyn", 100.0), knod or 4
        dt = dt or 1e-3
    elif name.startswith("cavityj"):
        n = int(name[7:])
        mesh = cavity(n, jitter=kw.get("jitter", 0.1), seed=kw.get("seed", 5))
        ptype, reyn, k = 1, kw.get("reyn", 100.0), knod or 4
        dt = dt or 1e-3
    elif name.startswith("cavity"):
        n = int(name[6:])
        mesh = cavity(n)
        ptype, reyn, k = 1, kw.get("reyn", 100.0), knod or 4
        dt = dt or 1e-3
    elif name.startswith("bfs"):
        m = int(name[3:]) if len(name) > 3 else 15
        mesh = backward_facing_step(h=1.0 / m, jitter=kw.get("jitter", 0.15), seed=kw.get("seed", 2),
                                    x_out=kw.get("x_out", 30.0), x_in=kw.get("x_in", -5.0))
        ptype, reyn, k = 2, kw.get("reyn", 400.0), knod or 5
        dt = dt or min(cfl_dt(mesh, k, 1.5), viscous_dt(mesh, k, reyn))
    elif name.startswith("cyl"):
        nr, nt = (int(v) for v in name[3:].split("x"))
        mesh = cylinder_ogrid(nr, nt, stretch=kw.get("stretch", 1.02))
        ptype, reyn, k = 3, kw.get("reyn", 100.0), knod or 5
        dt = dt or min(cfl_dt(mesh, k, 2.0), viscous_dt(mesh, k, reyn))
    else:
        raise ValueError(f"unknown case {name!r}")
    write_msh(mesh, os.path.join(outdir, "mesh.msh"))
    path = os.path.join(outdir, "input.dat")
    write_input_dat(path, "mesh.msh", k, reyn, dt, steps, ptype,
                    advection_type=kw.get("advection_type", 1),
                    time_integration=kw.get("time_integration", 4),
                    lnod_in=2 if mesh.quads.shape[1] == 9 else 1)
    return path
