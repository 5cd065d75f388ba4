"""CPU restatement (numpy) of HO-CXX's vorticity-streamfunction FR time step.

TEST INFRASTRUCTURE ONLY -- this module is the parity checker. It may be imported by
``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg, never by the
product. It restates, vectorised over elements, the reference's algorithm (citations
are to the reference's ``src/`` files):

* input reader ............................. src/HO_2D.cpp:213-317
* Gmsh 4.1 reader + mesh processing ........ src/Mesh.cpp:93-340, 342-487 (hash-based
  neighbour search with the same results as the O(N^2) scan)
* bases ..................................... src/HO_2D.cpp:486-673
* metrics ................................... src/HO_2D.cpp:1240-1388
* initial/boundary conditions ............... src/HO_2D.cpp:675-1238 (problem types 1, 2, 3)
* Poisson operator assembly ................. src/HO_2D.cpp:1533-1804, CSR filter 3023-3062
* time loop: RK driver ...................... src/HO_2D.cpp:1465-1531
* stage ..................................... src/HO_2D.cpp:1806-1839
* Poisson RHS / solve ....................... src/HO_2D.cpp:1841-1977 (scipy SuperLU, exact)
* BC refresh ................................ src/HO_2D.cpp:1979-2217
* velocity from psi ......................... src/HO_2D.cpp:3174-3366
* diffusion BC / residual ................... src/HO_2D.cpp:2647-2664, 2666-2927
* advection BC / residual (types 1 and 2) ... src/HO_2D.cpp:2219-2243, 2245-2437, 2439-2645

Pinned against golden vectors produced by the reference itself (built from its own
sources against the oracle's Eigen/AMGCL API shim): ``tests/golden``.

Array layout follows the reference: volume fields ``[el][j=eta][i=xi]``, face traces
``[el][ijp][k]`` with ijp 0=W (xi=-1), 1=E, 2=S (eta=-1), 3=N, boundary-edge arrays
``[edge][k]`` in edge (counter-clockwise) order.
"""

from __future__ import annotations

import math
import os
from dataclasses import dataclass

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

DIRICHLET, NEUMANN = 0, 1
SOUTH, EAST, NORTH, WEST = 0, 1, 2, 3
I2F = np.array([WEST, EAST, SOUTH, NORTH])  # ijp -> element side
F2I = np.array([2, 1, 3, 0])  # element side -> ijp
SGN = np.array([-1.0, 1.0, -1.0, 1.0])
EDGE_NODES = {1: 2, 8: 3, 26: 4, 27: 5, 28: 6}
FACE_NODES = {3: 4, 10: 9, 16: 8, 36: 16, 37: 25}
FACE_EDGE_NODES = {3: 2, 10: 3, 16: 3, 36: 4, 37: 5}


# ----------------------------------------------------------------------------- input
def read_input(path: str) -> dict:
    """Positional input.dat: each value follows one comment line (src/HO_2D.cpp:228-303)."""
    with open(path) as f:
        lines = f.read().split("\n")
    vals = []
    i = 0
    # 5 (comment, value) pairs, 2 ignored lines, then 13 more pairs
    order = ["nel", "knod", "lnod", "mesh", "occ", None, "reyn", "dxr", "fac", "huynh", "ti", "adv",
             "ptype", "nsteps", "dt", "dump", "fast", "lhs", "sample"]
    out = {}
    for key in order:
        if key is None:
            i += 2
            continue
        i += 1
        out[key] = lines[i].strip()
        i += 1
    out["knod"] = int(out["knod"].split()[0])
    out["occ"] = int(out["occ"].split()[0])
    reyn = float(out["reyn"].split()[0])
    out["reyn_inv"] = 1.0 / reyn if reyn > 1e-3 else -1.0
    for k in ("huynh", "ti", "adv", "ptype", "nsteps", "dump", "lhs"):
        out[k] = int(out[k].split()[0])
    out["dt"] = float(out["dt"].split()[0])
    out["mesh"] = out["mesh"].split()[0]
    return out


# ----------------------------------------------------------------------------- mesh
def tensor2fem(i: int, j: int, lnod_in: int) -> int:
    """Tensor (i, j) -> Gmsh node slot (src/Mesh.cpp:34-91)."""
    if lnod_in == 1:
        return i + 3 * j - 2 * i * j
    if lnod_in == 2:
        return [[0, 4, 1], [7, 8, 5], [3, 6, 2]][j][i]
    if lnod_in == 3:
        return [[0, 4, 5, 1], [11, 12, 13, 6], [10, 15, 14, 7], [3, 9, 8, 2]][j][i]
    raise ValueError("only up to cubic geometry is supported")


def tensor2fem_1d(i: int, lnod_in: int) -> int:
    return 0 if i == 0 else (1 if i == lnod_in else i + 1)


@dataclass
class Mesh:
    xy: np.ndarray  # node coordinates
    elem_nodes: list  # per element: Gmsh node list (after OCC reorientation)
    edge_nodes: list  # per edge: node list (boundary edges first, in file order)
    groups: list  # [(name, np.array(edge indices))]
    lnod: int
    n_eb: int
    nbr: np.ndarray  # [N,4] by element side (SENW); -1 on boundary
    nbr_side: np.ndarray  # [N,4] common side of the neighbour
    bidx: np.ndarray  # [N,4] boundary edge index or -1
    be_el: np.ndarray  # [N_eb]
    be_side: np.ndarray  # [N_eb]

    @property
    def n_el(self) -> int:
        return len(self.elem_nodes)


def read_msh(path: str, occ: int) -> Mesh:
    """Gmsh 4.1 ASCII reader with the semantics of Mesh::read_msh_file (src/Mesh.cpp:93-340)."""
    with open(path) as f:
        text = f.read().split("\n")
    pos = {}
    for n, ln in enumerate(text):
        if ln.strip().startswith("$") and ln.strip() not in pos:
            pos[ln.strip()] = n
    # physical names: only dimension-1 entries define boundaries
    p = pos["$PhysicalNames"] + 1
    nphys = int(text[p].split()[0])
    bnames, btags = [], []
    for k in range(nphys):
        tok = text[p + 1 + k].split()
        if int(tok[0]) != 1:
            continue
        btags.append(int(tok[1]))
        bnames.append(tok[2].strip('"'))
    # entities: curve tag -> physical tag (or 0 when the curve has none)
    p = pos["$Entities"] + 1
    npt, ncv, nsf, _ = (int(v) for v in text[p].split()[:4])
    curve_phys = {}
    for k in range(ncv):
        tok = text[p + 1 + npt + k].split()
        ntags = int(tok[7])
        curve_phys[int(tok[0])] = int(tok[8]) if ntags > 0 else 0
    # nodes
    p = pos["$Nodes"] + 1
    nblk, nnod, nmin, nmax = (int(v) for v in text[p].split()[:4])
    coords = {}
    p += 1
    for _ in range(nblk):
        tok = text[p].split()
        cnt = int(tok[3])
        tags = [int(text[p + 1 + k].split()[0]) for k in range(cnt)]
        for k in range(cnt):
            c = text[p + 1 + cnt + k].split()
            coords[tags[k]] = (float(c[0]), float(c[1]))
        p += 1 + 2 * cnt
    # elements
    p = pos["$Elements"] + 1
    nblk = int(text[p].split()[0])
    p += 1
    groups = [[] for _ in bnames]
    edges, quads = [], []
    last_edge_nodes = None
    for _ in range(nblk):
        tok = text[p].split()
        dim, etag, etype, cnt = (int(v) for v in tok[:4])
        rows = [[int(v) for v in text[p + 1 + k].split()] for k in range(cnt)]
        p += 1 + cnt
        if dim == 1:
            if etype not in EDGE_NODES:
                raise ValueError(f"unsupported line type {etype}")
            last_edge_nodes = EDGE_NODES[etype]
            ph = curve_phys[etag]
            if ph == 0:
                continue
            g = btags.index(ph)
            for r in rows:
                groups[g].append(len(edges))
                edges.append(r[1:1 + EDGE_NODES[etype]])
        elif dim == 2:
            if etype not in FACE_NODES:
                raise ValueError(f"unsupported face type {etype}")
            for r in rows:
                quads.append(r[1:1 + FACE_NODES[etype]])
    lnod = last_edge_nodes
    lin = lnod - 1
    if occ:
        for q in range(len(quads)):
            old = list(quads[q])
            new = list(old)
            for jo in range(lnod):
                for io in range(lnod):
                    new[tensor2fem(lin - jo, lin - io, lin)] = old[tensor2fem(io, jo, lin)]
            quads[q] = new
    # compact node numbering (only the coordinates matter for the solution)
    used = sorted({v for e in edges for v in e} | {v for q in quads for v in q})
    remap = {v: i for i, v in enumerate(used)}
    xy = np.array([coords[v] for v in used])
    edges = [[remap[v] for v in e] for e in edges]
    quads = [[remap[v] for v in q] for q in quads]
    n_eb = len(edges)
    n = len(quads)
    # process_mesh (src/Mesh.cpp:342-487): sides S,E,N,W run corner s -> corner s+1;
    # an edge is identified by its corner pair; boundary edges take the element's
    # counter-clockwise node order.
    key_to_edge = {}
    for e, nodes in enumerate(edges):
        key_to_edge.setdefault((min(nodes[0], nodes[1]), max(nodes[0], nodes[1])), e)
    elem_edges = np.zeros((n, 4), dtype=np.int64)
    for el, q in enumerate(quads):
        nen = len(q)
        ene = {4: 2, 9: 3, 8: 3, 16: 4, 25: 5}[nen]
        for s in range(4):
            en = [q[s], q[(s + 1) % 4]] + q[4 + s * (ene - 2): 4 + (s + 1) * (ene - 2)]
            key = (min(en[0], en[1]), max(en[0], en[1]))
            if key in key_to_edge:
                e = key_to_edge[key]
                edges[e] = en
            else:
                e = len(edges)
                key_to_edge[key] = e
                edges.append(en)
            elem_edges[el, s] = e
    owners = {}
    for el in range(n):
        for s in range(4):
            owners.setdefault(int(elem_edges[el, s]), []).append((el, s))
    nbr = np.full((n, 4), -1, dtype=np.int64)
    nbr_side = np.full((n, 4), -1, dtype=np.int64)
    bidx = np.full((n, 4), -1, dtype=np.int64)
    be_el = np.zeros(n_eb, dtype=np.int64)
    be_side = np.zeros(n_eb, dtype=np.int64)
    for el in range(n):
        for s in range(4):
            e = int(elem_edges[el, s])
            others = [(o, so) for (o, so) in owners[e] if o != el]
            if others:
                o, so = min(others)
                nbr[el, s], nbr_side[el, s] = o, so
            else:
                if e >= n_eb:
                    raise ValueError("a boundary side has no boundary edge in the mesh file")
                bidx[el, s] = e
                be_el[e], be_side[e] = el, s
    grp = [(bnames[g], np.array(groups[g], dtype=np.int64)) for g in range(len(bnames))]
    return Mesh(xy, quads, edges, grp, lnod, n_eb, nbr, nbr_side, bidx, be_el, be_side)


# ----------------------------------------------------------------------------- bases
def legendre(n: int, x):
    x = np.asarray(x, dtype=float)
    if n == 0:
        return np.ones_like(x)
    p0, p1 = np.ones_like(x), x
    for i in range(2, n + 1):
        p0, p1 = p1, ((2 * i - 1) * x * p1 - (i - 1) * p0) / i
    return p1


def lagrange(nodes: np.ndarray, x: np.ndarray):
    """Values V[k, m] = l_k(x_m) and derivatives Dv[k, m] = l_k'(x_m)."""
    nodes = np.asarray(nodes, float)
    x = np.atleast_1d(np.asarray(x, float))
    n = len(nodes)
    V = np.ones((n, len(x)))
    Dv = np.zeros((n, len(x)))
    for k in range(n):
        den = np.prod([nodes[k] - nodes[j] for j in range(n) if j != k])
        for j in range(n):
            if j == k:
                continue
            V[k] *= x - nodes[j]
            term = np.ones(len(x))
            for i in range(n):
                if i != k and i != j:
                    term *= x - nodes[i]
            Dv[k] += term
        V[k] /= den
        Dv[k] /= den
    return V, Dv


@dataclass
class Bases:
    K: int
    L: int
    xs: np.ndarray
    w: np.ndarray
    sbb: np.ndarray  # [K,2] l_k(-1), l_k(+1)
    sbgb: np.ndarray  # [K,2] l_k'(-1), l_k'(+1)
    D: np.ndarray  # [K,K] D[k,m] = l_k'(x_m)
    R: np.ndarray  # [K,2] Radau values (left, right)
    gR: np.ndarray  # [K,2] Radau derivatives
    gsb: np.ndarray  # [L,K] geometry basis at sps
    gsgb: np.ndarray  # [L,K]
    gbb: np.ndarray  # [L,2]
    gbgb: np.ndarray  # [L,2]
    gp: np.ndarray  # g'(-1), g'(+1)


def make_bases(K: int, L: int) -> Bases:
    """src/HO_2D.cpp:486-673 (Gauss-Legendre nodes from numpy's leggauss)."""
    xs, w = np.polynomial.legendre.leggauss(K)
    gx = np.linspace(-1.0, 1.0, L)
    sbb, sbgb = lagrange(xs, [-1.0, 1.0])
    _, D = lagrange(xs, xs)
    gsb, gsgb = lagrange(gx, xs)
    gbb, gbgb = lagrange(gx, [-1.0, 1.0])
    if K == 1:
        R = np.array([[0.5, 0.5]])
        gR = np.array([[-0.5, 0.5]])
    else:
        c = 0.5 * (-1.0) ** K
        cd = 0.5 * K * (-1.0) ** K
        R = np.stack([c * (legendre(K, xs) - legendre(K - 1, xs)), c * (legendre(K, -xs) - legendre(K - 1, -xs))], 1)
        gR = np.stack([cd * (legendre(K, xs) + legendre(K - 1, xs)) / (1.0 + xs),
                       -cd * (legendre(K, -xs) + legendre(K - 1, -xs)) / (1.0 - xs)], 1)
    gp = np.array([-0.5 * K * (K + 1.0), 0.5 * K * (K + 1.0)])
    return Bases(K, L, xs, w, sbb, sbgb, D, R, gR, gsb, gsgb, gbb, gbgb, gp)


# ----------------------------------------------------------------------------- metrics
def element_coords(mesh: Mesh) -> np.ndarray:
    L = mesh.lnod
    X = np.zeros((mesh.n_el, L, L, 2))
    for el, q in enumerate(mesh.elem_nodes):
        for j in range(L):
            for i in range(L):
                X[el, j, i] = mesh.xy[q[tensor2fem(i, j, L - 1)]]
    return X


def make_metrics(X: np.ndarray, B: Bases) -> dict:
    """Volume and face metrics (src/HO_2D.cpp:1240-1388)."""
    x, y = X[..., 0], X[..., 1]
    xxi = np.einsum("mi,nj,enm->eji", B.gsgb, B.gsb, x)
    yxi = np.einsum("mi,nj,enm->eji", B.gsgb, B.gsb, y)
    xeta = np.einsum("nj,mi,enm->eji", B.gsgb, B.gsb, x)
    yeta = np.einsum("nj,mi,enm->eji", B.gsgb, B.gsb, y)
    J = xxi * yeta - xeta * yxi
    dxdx = np.stack([np.stack([yeta / J, -xeta / J], -1), np.stack([-yxi / J, xxi / J], -1)], -2)
    g0 = np.stack([-xeta, yeta], -1)
    g1 = np.stack([xxi, -yxi], -1)
    g = [g0, g1]
    G = np.zeros(J.shape + (2, 2))
    for r in range(2):
        for s in range(2):
            G[..., r, s] = np.sum(g[r] * g[s], -1) / J
    N, K = J.shape[0], B.K
    fxx = np.zeros((N, 4, K))
    fxe = np.zeros((N, 4, K))
    fyx = np.zeros((N, 4, K))
    fye = np.zeros((N, 4, K))
    for t in range(2):  # west/east: xi = -1/+1
        fxx[:, t] = np.einsum("i,jk,eji->ek", B.gbgb[:, t], B.gsb, x)
        fyx[:, t] = np.einsum("i,jk,eji->ek", B.gbgb[:, t], B.gsb, y)
        fxe[:, t] = np.einsum("i,jk,eji->ek", B.gbb[:, t], B.gsgb, x)
        fye[:, t] = np.einsum("i,jk,eji->ek", B.gbb[:, t], B.gsgb, y)
    for t in range(2):  # south/north: eta = -1/+1
        fxx[:, 2 + t] = np.einsum("j,ik,eji->ek", B.gbb[:, t], B.gsgb, x)
        fyx[:, 2 + t] = np.einsum("j,ik,eji->ek", B.gbb[:, t], B.gsgb, y)
        fxe[:, 2 + t] = np.einsum("j,ik,eji->ek", B.gbgb[:, t], B.gsb, x)
        fye[:, 2 + t] = np.einsum("j,ik,eji->ek", B.gbgb[:, t], B.gsb, y)
    fJ = fxx * fye - fxe * fyx
    fA = np.concatenate([fxe[:, :2] ** 2 + fye[:, :2] ** 2, fxx[:, 2:] ** 2 + fyx[:, 2:] ** 2], 1)
    fB = fxx * fxe + fyx * fye
    fAn = np.sqrt(fA)
    GB = np.zeros((N, 2, 2, K, 2))
    gf0 = np.stack([-fxe, fye], -1)
    gf1 = np.stack([fxx, -fyx], -1)
    for d in range(2):
        for t in range(2):
            ijp = 2 * d + t
            gd = (gf0, gf1)[d][:, ijp]
            for r in range(2):
                gr = (gf0, gf1)[r][:, ijp]
                GB[:, d, t, :, r] = np.sum(gd * gr, -1) / fJ[:, ijp]
    return dict(xxi=xxi, xeta=xeta, yxi=yxi, yeta=yeta, J=J, dxdx=dxdx, G=G, GB=GB, fJ=fJ, fA=fA, fB=fB, fAn=fAn)


# ----------------------------------------------------------------------------- assembly
def _bf(side: int, k, K: int):
    """Boundary flux-point index of local face point k (src/HO_2D.cpp:1640)."""
    return (side // 2) * (K - 2 * np.asarray(k) - 1) + np.asarray(k)


def _rs(p, q, d: int, K: int):
    """Volume index of point p along direction d on the line q (src/HO_2D.cpp:1586-1588)."""
    return (p * d + q * (1 - d)) * K + (p * (1 - d) + q * d)


def _face_weight_tables(B: Bases):
    """Wc[d][t][ij, q, (b, a, r)]: the K^2 x K face coupling W = Wc . G[el][:, :, :, d],
    i.e. sum over (m, r) of (D[m][.] - tmp2) * G[el][b][a][r][d] * gR[.][t]
    (src/HO_2D.cpp:1614-1637, 1680-1700, 1729-1749)."""
    K = B.K
    Wc = np.zeros((2, 2, K * K, K, K, K, 2))
    for d in range(2):
        for t in range(2):
            for j in range(K):
                for i in range(K):
                    ij = j * K + i
                    for m in range(K):
                        for r in range(2):
                            a = m * (1 - r) + i * r
                            b = m * r + j * (1 - r)
                            q = a * d + b * (1 - d)
                            sn = B.D[m, i * (1 - r) + j * r]
                            ngr = B.gR[a * (1 - d) + b * d, t]
                            tmp2 = B.sbb[m, 0] * B.gR[j * r + i * (1 - r), 0] + B.sbb[m, 1] * B.gR[j * r + i * (1 - r), 1]
                            Wc[d, t, ij, q, b, a, r] += (sn - tmp2) * ngr
    return Wc.reshape(2, 2, K * K, K, K * K * 2)


def _volume_table(B: Bases):
    """C[ij*K^2+rs, (b, a, r, d)] for the element-interior term (src/HO_2D.cpp:1567-1596)."""
    K = B.K
    C = np.zeros((K * K, K * K, K, K, 2, 2))
    for j in range(K):
        for i in range(K):
            ij = j * K + i
            for m in range(K):
                for r in range(2):
                    a = m * (1 - r) + i * r
                    b = m * r + j * (1 - r)
                    tmp3 = B.sbb[m, 0] * B.gR[j * r + i * (1 - r), 0] + B.sbb[m, 1] * B.gR[j * r + i * (1 - r), 1]
                    sn = B.D[m, i * (1 - r) + j * r]
                    for d in range(2):
                        t1 = a * (1 - d) + b * d
                        for p in range(K):
                            rs = (p * d + b * (1 - d)) * K + (p * (1 - d) + a * d)
                            tmp2 = 0.5 * (B.sbb[p, 0] * B.gR[t1, 0] + B.sbb[p, 1] * B.gR[t1, 1])
                            C[ij, rs, b, a, r, d] += sn * (B.D[p, t1] - tmp2) + tmp3 * (-B.D[p, t1] + tmp2)
    return C.reshape(K ** 4, K * K * 4)


def assemble_laplacian(mesh: Mesh, B: Bases, M: dict, sw_p: np.ndarray):
    """Poisson operator and boundary-source tensor (src/HO_2D.cpp:1533-1804, 3011-3062).

    Returns (A as CSR with the reference's |a| > 1e-14 filter, boundary_source[N_eb][K^2][K]).
    """
    K, N = B.K, mesh.n_el
    K2 = K * K
    G = M["G"]
    Lc = (G.reshape(N, -1) @ _volume_table(B).T).reshape(N, K2, K2)
    Ln = np.zeros((N, 4, K2, K2))
    bsrc = np.zeros((mesh.n_eb, K2, K))
    Wc = _face_weight_tables(B)
    gp = B.gp
    jj, ii = np.divmod(np.arange(K2), K)
    for d in range(2):
        Gd = G[..., d].reshape(N, -1)  # [N, (b, a, r)]
        for t in range(2):
            ijp = 2 * d + t
            side = int(I2F[ijp])
            W = np.einsum("Qqg,eg->eQq", Wc[d, t], Gd)  # [N, K2, K]
            alpha = ii * d + jj * (1 - d)
            perp = jj * d + ii * (1 - d)
            ngr = B.gR[perp, t]  # [K2]
            pp = np.arange(K)
            for el in range(N):
                GBe = M["GB"][el, d, t]  # [K, 2]
                if mesh.bidx[el, side] >= 0:
                    e = int(mesh.bidx[el, side])
                    Wel = W[el]
                    # own extrapolation replaced by the boundary value: -0.5 W sbb[p][t]
                    for q in range(K):
                        Lc[el][:, _rs(pp, q, d, K)] -= 0.5 * np.outer(Wel[:, q], B.sbb[:, t])
                    if sw_p[e] == DIRICHLET:
                        for q in range(K):
                            bsrc[e][:, _bf(side, q, K)] += Wel[:, q]
                        A = GBe[alpha, d]
                        Bc = GBe[alpha, 1 - d]
                        for r_ in range(K2):
                            Lc[el][r_, _rs(pp, alpha[r_], d, K)] += A[r_] * (B.sbgb[:, t] - gp[t] * B.sbb[:, t]) * ngr[r_]
                            bsrc[e][r_, _bf(side, alpha[r_], K)] += A[r_] * gp[t] * ngr[r_]
                            bsrc[e][r_, _bf(side, pp, K)] += Bc[r_] * B.D[:, alpha[r_]] * ngr[r_]
                    else:
                        Nm = np.zeros((K, K))
                        for i_ in range(K):
                            Nm[i_, :] = -GBe[i_, 1 - d] * B.D[:, i_]
                            Nm[i_, i_] += -GBe[i_, d] * gp[t]
                        Ninv = np.linalg.inv(Nm)
                        sign = 1.0 if t else -1.0
                        s = np.sqrt(GBe[:, d] * M["fJ"][el, ijp])  # [K]
                        for r_ in range(K2):
                            bsrc[e][r_, _bf(side, alpha[r_], K)] += sign * ngr[r_] * s[alpha[r_]]
                        # W (tmp2 - sn) = -Wel
                        WN = Wel @ Ninv  # [K2, K] over p
                        bsrc[e][:, _bf(side, pp, K)] += -sign * WN * s[None, :]
                        tmp4 = B.sbgb[:, t] - gp[t] * B.sbb[:, t]  # [K] over p
                        WNc = Wel @ Ninv  # [K2, K] over c
                        for p in range(K):
                            cols = _rs(p, np.arange(K), d, K)  # rs(p, c)
                            Lc[el][:, cols] += WNc * tmp4[p] * GBe[None, :, d]
                else:
                    eln = int(mesh.nbr[el, side])
                    ijpm = int(F2I[mesh.nbr_side[el, side]])
                    dn, tn = ijpm // 2, ijpm % 2
                    rev = (d + t + dn + tn + 1) % 2
                    Wel = W[el]
                    Ln_el = Ln[el, side]
                    for q in range(K):
                        Mq = rev * (K - 2 * q - 1) + q
                        Ln_el[:, _rs(pp, Mq, dn, K)] += 0.5 * np.outer(Wel[:, q], B.sbb[:, tn])
                    GBn = M["GB"][eln, dn, tn]
                    sign = -1.0 if t == tn else 1.0
                    Malpha = rev * (K - 2 * alpha - 1) + alpha
                    A = GBe[alpha, d]
                    Bc = GBe[alpha, 1 - d]
                    An = GBn[Malpha, dn]
                    Bn = GBn[Malpha, 1 - dn]
                    Mm = rev * (K - 2 * pp - 1) + pp
                    for r_ in range(K2):
                        a_ = alpha[r_]
                        Lc[el][r_, _rs(pp, a_, d, K)] += (0.5 * A[r_] * B.sbgb[:, t] - 0.25 * gp[t] * A[r_] * B.sbb[:, t]
                                                          + 0.25 * sign * gp[tn] * An[r_] * B.sbb[:, t]) * ngr[r_]
                        Ln_el[r_, _rs(pp, Malpha[r_], dn, K)] += (0.5 * sign * An[r_] * B.sbgb[:, tn]
                                                                 - 0.25 * sign * gp[tn] * An[r_] * B.sbb[:, tn]
                                                                 + 0.25 * gp[t] * A[r_] * B.sbb[:, tn]) * ngr[r_]
                        coeff = 0.25 * (Bc[r_] * B.D[:, a_] + sign * Bn[r_] * B.D[Mm, Malpha[r_]]) * ngr[r_]  # over m
                        for m in range(K):
                            Lc[el][r_, _rs(pp, m, d, K)] += coeff[m] * B.sbb[:, t]
                            Ln_el[r_, _rs(pp, Mm[m], dn, K)] += coeff[m] * B.sbb[:, tn]
    # CSR with the reference's filter: centre block first, then S, E, N, W neighbours
    rows, cols, vals = [], [], []
    base = np.arange(N)[:, None, None] * K2
    r_idx = base + np.arange(K2)[None, :, None]
    c_idx = base + np.arange(K2)[None, None, :]
    rows.append(np.broadcast_to(r_idx, Lc.shape).ravel())
    cols.append(np.broadcast_to(c_idx, Lc.shape).ravel())
    vals.append(Lc.ravel())
    for s in range(4):
        has = mesh.nbr[:, s] >= 0
        eln = np.where(has, mesh.nbr[:, s], 0)
        cb = eln[:, None, None] * K2 + np.arange(K2)[None, None, :]
        rows.append(np.broadcast_to(r_idx, Lc.shape)[has].ravel())
        cols.append(np.broadcast_to(cb, Lc.shape)[has].ravel())
        vals.append(Ln[:, s][has].ravel())
    rows = np.concatenate(rows)
    cols = np.concatenate(cols)
    vals = np.concatenate(vals)
    keep = np.abs(vals) > 1e-14
    A = sp.csr_matrix((vals[keep], (rows[keep], cols[keep])), shape=(N * K2, N * K2))
    A.sort_indices()
    return A, bsrc


# ----------------------------------------------------------------------------- case
class Case:
    """One solver instance: setup sequence of src/main.cpp:44-77 plus the time loop."""

    def __init__(self, input_path: str, dt: float | None = None):
        cfg = read_input(input_path)
        self.cfg = cfg
        self.K = cfg["knod"]
        self.re_inv = cfg["reyn_inv"]
        self.dt = dt if dt is not None else cfg["dt"]
        self.ptype = cfg["ptype"]
        self.adv_type = cfg["adv"]
        self.ti_type = cfg["ti"]
        mesh_path = os.path.join(os.path.dirname(os.path.abspath(input_path)), cfg["mesh"])
        self.mesh = read_msh(mesh_path, cfg["occ"])
        self.L = self.mesh.lnod
        self.B = make_bases(self.K, self.L)
        self.X = element_coords(self.mesh)
        self.M = make_metrics(self.X, self.B)
        self.N = self.mesh.n_el
        self.neb = self.mesh.n_eb
        K = self.K
        # side tables in ijp terms
        m = self.mesh
        self.f_bidx = m.bidx[:, I2F]  # [N,4]
        self.f_nbr = m.nbr[:, I2F]
        self.f_nijp = np.where(self.f_nbr >= 0, F2I[np.maximum(m.nbr_side[:, I2F], 0)], -1)
        self.be_ijp = F2I[m.be_side]
        self.setup_bc()
        self.A, self.bsrc = assemble_laplacian(m, self.B, self.M, self.sw_p)
        self.lu = spla.splu(self.A.tocsc())
        self.omega = np.zeros((self.N, K, K))
        self.psi = np.zeros((self.N, K, K))
        self.vel = np.zeros((self.N, K, K, 2))
        self.t = 0.0

    # -- boundary conditions (src/HO_2D.cpp:675-1238, 1979-2217)
    def _group(self, name):
        for g, (nm, ed) in enumerate(self.mesh.groups):
            if nm == name:
                yield g, ed

    def _edge_y(self, e):
        """y at the K solution points of boundary edge e, in edge order (src/HO_2D.cpp:781)."""
        nodes = self.mesh.edge_nodes[e]
        ys = np.array([self.mesh.xy[nodes[tensor2fem_1d(j, self.L - 1)], 1] for j in range(self.L)])
        return self.B.gsb.T @ ys

    def _inlet_span(self):
        y_min = y_max = 0.0
        for _, ed in self._group("inlet"):
            n0 = self.mesh.edge_nodes[ed[0]][0]
            y_min = y_max = self.mesh.xy[n0, 1]
            for e in ed:
                for n in self.mesh.edge_nodes[e][:2]:
                    y_min = min(y_min, self.mesh.xy[n, 1])
                    y_max = max(y_max, self.mesh.xy[n, 1])
        return y_min, y_max

    def setup_bc(self):
        K, neb = self.K, self.neb
        ng = len(self.mesh.groups)
        self.noslip = np.zeros(ng, dtype=bool)
        self.sw_p = np.zeros(neb, dtype=np.int64)
        self.sw_d = np.zeros(neb, dtype=np.int64)
        self.bc_p = np.zeros((neb, K))
        self.bc_nv = np.zeros((neb, K))
        self.bc_pv = np.zeros((neb, K))
        self.bc_d = np.zeros((neb, K))
        self.bc_w = np.zeros((neb, K))
        self.vjump = np.zeros((neb, K))
        self.bc_adv = np.zeros((neb, K))
        pt = self.ptype
        if pt == 1:
            self.noslip[:] = True
            self.sw_p[:] = DIRICHLET
            self.sw_d[:] = NEUMANN
            for _, ed in self._group("top"):
                self.bc_pv[ed] = -1.0
        elif pt in (2, 3):
            y_min, y_max = self._inlet_span()
            for g, (nm, ed) in enumerate(self.mesh.groups):
                if nm == "inlet":
                    self.noslip[g] = False
                    for e in ed:
                        self.sw_d[e] = DIRICHLET
                        self.sw_p[e] = DIRICHLET
                        y = self._edge_y(e)
                        if pt == 2:
                            h2 = (y_max - y_min) ** 2
                            self.bc_p[e] = (y - y_min) ** 2 * (3 * y_max - y_min - 2 * y) / h2
                            self.bc_d[e] = 6 * (2 * y - y_min - y_max) / h2
                            self.bc_nv[e] = 6 * (y - y_min) * (y - y_max) / h2
                        else:
                            self.bc_p[e] = y - y_min
                            self.bc_d[e] = 0.0
                            self.bc_nv[e] = -1.0
                elif nm == "outlet":
                    self.noslip[g] = False
                    self.sw_d[ed] = NEUMANN
                    self.sw_p[ed] = NEUMANN
                    self.bc_d[ed] = 0.0
                    self.bc_p[ed] = 0.0
                elif nm in ("top", "bottom"):
                    self.noslip[g] = (pt == 2)
                    self.sw_p[ed] = DIRICHLET
                    self.sw_d[ed] = NEUMANN
                    if nm == "top":
                        self.bc_p[ed] = y_max - y_min
                    else:
                        self.bc_p[ed] = 0.0
                    self.bc_nv[ed] = 0.0
                    if pt == 2:
                        self.bc_pv[ed] = 0.0
                    else:
                        self.bc_pv[ed] = -1.0 if nm == "top" else 1.0
                elif nm == "object" and pt == 3:
                    self.noslip[g] = True
                    self.sw_p[ed] = DIRICHLET
                    self.sw_d[ed] = NEUMANN
                    self.bc_p[ed] = 0.5 * (y_max - y_min)
                    self.bc_nv[ed] = 0.0
                    self.bc_pv[ed] = 0.0
        else:
            raise NotImplementedError(f"problem_type {pt}")
        self._flip_to_h()

    def _flip_to_h(self):
        """Outward-normal values into the local h direction (src/HO_2D.cpp:1228-1237, 2203-2215)."""
        sign = 2.0 * (self.be_ijp % 2) - 1.0
        self.bc_nv *= sign[:, None]
        neu = self.sw_d == NEUMANN
        self.bc_d[neu] *= sign[neu, None]

    def update_bcs(self, time):
        pt = self.ptype
        if pt in (2, 3):
            y_min, y_max = self._inlet_span()
            tc = 2.0 * abs(math.sin(math.pi / 40.0 * time))
            for nm, ed in self.mesh.groups:
                if nm == "inlet":
                    for e in ed:
                        y = self._edge_y(e)
                        if pt == 2:
                            h2 = (y_max - y_min) ** 2
                            self.bc_p[e] = tc * (y - y_min) ** 2 * (3 * y_max - y_min - 2 * y) / h2
                            self.bc_d[e] = tc * 6 * (2 * y - y_min - y_max) / h2
                            self.bc_nv[e] = tc * 6 * (y - y_min) * (y - y_max) / h2
                        else:
                            self.bc_p[e] = tc * (y - y_min)
                            self.bc_nv[e] = -tc
                elif nm == "top":
                    self.bc_p[ed] = tc * (y_max - y_min)
                    if pt == 3:
                        self.bc_d[ed] = 0.0
                        self.bc_pv[ed] = -tc
                elif nm == "bottom" and pt == 3:
                    self.bc_pv[ed] = tc
                elif nm == "object" and pt == 3:
                    self.bc_p[ed] = tc * 0.5 * (y_max - y_min)
        self._flip_to_h()

    # -- face traces
    def _traces(self, f):
        """Values and xi/eta derivatives extrapolated to the 4 faces: [N,4,K] each."""
        B = self.B
        v = np.stack([f @ B.sbb[:, 0], f @ B.sbb[:, 1],
                      np.einsum("emi,m->ei", f, B.sbb[:, 0]), np.einsum("emi,m->ei", f, B.sbb[:, 1])], 1)
        g = np.stack([f @ B.sbgb[:, 0], f @ B.sbgb[:, 1],
                      np.einsum("emi,m->ei", f, B.sbgb[:, 0]), np.einsum("emi,m->ei", f, B.sbgb[:, 1])], 1)
        return v, g

    def _nbr_gather(self, arr):
        """arr[eln][ijpm][jn] aligned with the local face points, and the orientation sign."""
        K = self.K
        out = np.zeros_like(arr)
        sign = np.zeros(arr.shape[:2])
        k = np.arange(K)
        for ijp in range(4):
            nb = self.f_nbr[:, ijp]
            has = nb >= 0
            ijpm = self.f_nijp[has, ijp]
            rev = (ijp + ijpm - ijp // 2 - ijpm // 2 + 1) % 2
            jn = rev[:, None] * (K - 2 * k[None, :] - 1) + k[None, :]
            out[has, ijp] = arr[nb[has][:, None], ijpm[:, None], jn]
            sign[has, ijp] = 2.0 * ((ijp + ijpm) % 2) - 1.0
        return out, sign

    def _bfpi(self, ijp):
        return _bf(int(I2F[ijp]), np.arange(self.K), self.K)

    def _common(self, v, g, sw, vals, interior_only=False):
        """Method-2 common values and normal fluxes (src/HO_2D.cpp:2833-2927).

        Returns comm value [N,4,K], comm normal flux [N,4,K] (faces averaged), and the
        per-face arrays before averaging."""
        B, K = self.B, self.K
        fA, fB, fJ, fAn = self.M["fA"], self.M["fB"], self.M["fJ"], self.M["fAn"]
        vn, _ = self._nbr_gather(v)
        comm = np.zeros_like(v)
        flux = g.copy()
        cgrad = np.zeros_like(v)
        for ijp in range(4):
            ibnd = ijp % 2
            inter = self.f_nbr[:, ijp] >= 0
            comm[inter, ijp] = 0.5 * (v[inter, ijp] + vn[inter, ijp])
            bnd = ~inter
            e = self.f_bidx[bnd, ijp]
            bf = self._bfpi(ijp)
            dirich = sw[e] == DIRICHLET
            els = np.nonzero(bnd)[0]
            # Dirichlet: common value is the boundary value
            ed, eld = e[dirich], els[dirich]
            comm[eld, ijp] = vals[ed][:, bf]
            # Neumann: solve the K x K system for the common value
            en, eln = e[~dirich], els[~dirich]
            if len(en):
                cg = vals[en][:, bf] * fAn[eln, ijp]
                cgrad[eln, ijp] = cg
                rhs = fJ[eln, ijp] * cg - fA[eln, ijp] * (g[eln, ijp] - v[eln, ijp] * B.gp[ibnd])
                Mt = -fB[eln, ijp][:, :, None] * B.D.T[None, :, :]
                Mt[:, np.arange(K), np.arange(K)] += fA[eln, ijp] * B.gp[ibnd]
                comm[eln, ijp] = np.linalg.solve(Mt, rhs[..., None])[..., 0]
            # corrected derivative and normal flux (interior and Dirichlet faces)
            flx = inter.copy()
            flx[eld] = True
            c = comm[flx, ijp]
            dv = g[flx, ijp] + (c - v[flx, ijp]) * B.gp[ibnd]
            cross = c @ B.D
            flux[flx, ijp] = (dv * fA[flx, ijp] - cross * fB[flx, ijp]) / fJ[flx, ijp]
            cgrad[eld, ijp] = flux[eld, ijp]
        fn, sgn = self._nbr_gather(flux)
        inter = self.f_nbr >= 0
        cgrad[inter] = 0.5 * (flux[inter] + sgn[inter][:, None] * fn[inter])
        return comm, cgrad

    def _fr_grad_fluxes(self, f, comm, cgrad, v):
        """f~, g~ at the solution points and their face corrections (src/HO_2D.cpp:2773-2803)."""
        B, Mt = self.B, self.M
        gR = B.gR
        dx = f @ B.D + (comm[:, 0] - v[:, 0])[:, :, None] * gR[:, 0][None, None, :] \
            + (comm[:, 1] - v[:, 1])[:, :, None] * gR[:, 1][None, None, :]
        de = np.einsum("edk,dj->ejk", f, B.D) + (comm[:, 2] - v[:, 2])[:, None, :] * gR[:, 0][None, :, None] \
            + (comm[:, 3] - v[:, 3])[:, None, :] * gR[:, 1][None, :, None]
        xxi, xeta, yxi, yeta, J = Mt["xxi"], Mt["xeta"], Mt["yxi"], Mt["yeta"], Mt["J"]
        ft = (dx * (xeta * xeta + yeta * yeta) - de * (xxi * xeta + yxi * yeta)) / J
        gt = (de * (xxi * xxi + yxi * yxi) - dx * (xxi * xeta + yxi * yeta)) / J
        fB = np.stack([cgrad[:, 0] - ft @ B.sbb[:, 0], cgrad[:, 1] - ft @ B.sbb[:, 1]], 1)
        gB = np.stack([cgrad[:, 2] - np.einsum("edk,d->ek", gt, B.sbb[:, 0]),
                       cgrad[:, 3] - np.einsum("edk,d->ek", gt, B.sbb[:, 1])], 1)
        return ft, gt, fB, gB

    # -- the hot path
    def poisson_rhs(self, vort):
        K2 = self.K * self.K
        rhs = (-vort * self.M["J"]).reshape(self.N, K2)
        contrib = np.einsum("eqa,ea->eq", self.bsrc, self.bc_p)
        np.add.at(rhs, self.mesh.be_el, -contrib)
        return rhs.ravel()

    def solve_poisson(self, vort):
        rhs = self.poisson_rhs(vort)
        if np.iscomplexobj(rhs):  # complex-step derivatives (ho2d_cs): the LU is real
            psi = self.lu.solve(np.ascontiguousarray(rhs.real)) + 1j * self.lu.solve(np.ascontiguousarray(rhs.imag))
        else:
            psi = self.lu.solve(rhs)
        self.psi = psi.reshape(self.N, self.K, self.K)

    def velocity(self):
        """u = dpsi/dy, v = -dpsi/dx with side outputs (src/HO_2D.cpp:3174-3366)."""
        B, K, Mt = self.B, self.K, self.M
        v, g = self._traces(self.psi)
        # Neumann psi values are given as d(psi)/dn; the solver uses the h-direction sign
        vals = self.bc_p.copy()
        psign = 2.0 * (self.be_ijp % 2) - 1.0
        neu = self.sw_p == NEUMANN
        vals[neu] = psign[neu, None] * self.bc_p[neu]
        comm, cgrad = self._common(v, g, self.sw_p, vals)
        for ijp in range(4):
            bnd = self.f_bidx[:, ijp] >= 0
            els = np.nonzero(bnd)[0]
            e = self.f_bidx[bnd, ijp]
            bf = self._bfpi(ijp)
            d_ = self.sw_p[e] == DIRICHLET
            self.vjump[e[d_][:, None], bf[None, :]] = cgrad[els[d_], ijp] / Mt["fAn"][els[d_], ijp]
            n_ = ~d_
            if n_.any():
                vsign = 1.0 - 2.0 * (ijp // 2)
                nv = (vsign * comm[els[n_], ijp]) @ B.D / Mt["fAn"][els[n_], ijp]
                self.bc_nv[e[n_][:, None], bf[None, :]] = nv
        ft, gt, fB, gB = self._fr_grad_fluxes(self.psi, comm, cgrad, v)
        R = B.R
        tx = ft + fB[:, 0][:, :, None] * R[:, 0][None, None, :] + fB[:, 1][:, :, None] * R[:, 1][None, None, :]
        ty = gt + gB[:, 0][:, None, :] * R[:, 0][None, :, None] + gB[:, 1][:, None, :] * R[:, 1][None, :, None]
        J = Mt["J"]
        dpdx = (tx * Mt["xxi"] + ty * Mt["xeta"]) / J
        dpdy = (tx * Mt["yxi"] + ty * Mt["yeta"]) / J
        self.vel = np.stack([dpdy, -dpdx], -1)

    def update_diffusion_bc(self):
        for g, (nm, ed) in enumerate(self.mesh.groups):
            if not self.noslip[g]:
                continue
            sign = (self.be_ijp[ed] % 2) * 2.0 - 1.0
            self.vjump[ed] += sign[:, None] * self.bc_pv[ed]
            self.bc_d[ed] = self.vjump[ed] / (self.dt * self.re_inv)

    def rhs_diffusion(self, vort):
        """Re^-1 Laplacian(omega), Huynh method 2 with g_DG (src/HO_2D.cpp:2666-2831)."""
        B = self.B
        v, g = self._traces(vort)
        comm, cgrad = self._common(v, g, self.sw_d, self.bc_d)
        for ijp in range(4):
            bnd = self.f_bidx[:, ijp] >= 0
            e = self.f_bidx[bnd, ijp]
            self.bc_w[e[:, None], self._bfpi(ijp)[None, :]] = comm[bnd, ijp]
        ft, gt, fB, gB = self._fr_grad_fluxes(vort, comm, cgrad, v)
        gR = B.gR
        lap = ft @ B.D + fB[:, 0][:, :, None] * gR[:, 0][None, None, :] + fB[:, 1][:, :, None] * gR[:, 1][None, None, :]
        lap += np.einsum("edk,dj->ejk", gt, B.D) + gB[:, 0][:, None, :] * gR[:, 0][None, :, None] \
            + gB[:, 1][:, None, :] * gR[:, 1][None, :, None]
        return lap * self.re_inv / self.M["J"]

    def update_advection_bc(self):
        el = self.mesh.be_el
        ijp = self.be_ijp
        for e in range(self.neb):
            bf = self._bfpi(int(ijp[e]))
            self.bc_adv[e, bf] = self.bc_w[e, bf] * self.bc_nv[e, bf] * self.M["fAn"][el[e], ijp[e]]

    def _contravariant(self):
        Mt = self.M
        u, v = self.vel[..., 0], self.vel[..., 1]
        J = Mt["J"]
        ux = u * Mt["dxdx"][..., 0, 0] * J + v * Mt["dxdx"][..., 0, 1] * J
        uy = u * Mt["dxdx"][..., 1, 0] * J + v * Mt["dxdx"][..., 1, 1] * J
        return ux, uy

    def _lift_divergence(self, fx, fy, up):
        """-(d/dxi fx + d/deta fy + Radau lift of (common - extrapolated)) / J."""
        B = self.B
        bx = np.stack([up[:, 0] - fx @ B.sbb[:, 0], up[:, 1] - fx @ B.sbb[:, 1]], 1)
        by = np.stack([up[:, 2] - np.einsum("emi,m->ei", fy, B.sbb[:, 0]),
                       up[:, 3] - np.einsum("emi,m->ei", fy, B.sbb[:, 1])], 1)
        gR = B.gR
        r = fx @ B.D + np.einsum("edk,dj->ejk", fy, B.D)
        r += bx[:, 0][:, :, None] * gR[:, 0][None, None, :] + bx[:, 1][:, :, None] * gR[:, 1][None, None, :]
        r += by[:, 0][:, None, :] * gR[:, 0][None, :, None] + by[:, 1][:, None, :] * gR[:, 1][None, :, None]
        return -r / self.M["J"]

    def _boundary_face_values(self, arr_eb):
        """Boundary-edge array [N_eb][K] mapped onto faces [N,4,K] (zero elsewhere)."""
        out = np.zeros((self.N, 4, self.K), dtype=np.result_type(arr_eb, float))
        for ijp in range(4):
            bnd = self.f_bidx[:, ijp] >= 0
            e = self.f_bidx[bnd, ijp]
            out[bnd, ijp] = arr_eb[e[:, None], self._bfpi(ijp)[None, :]]
        return out

    def rhs_advection(self, vort):
        """-div(u omega), discontinuous mass flux with the |d omega| > 1e-4 switch (src/HO_2D.cpp:2245-2437)."""
        ux, uy = self._contravariant()
        fx, fy = ux * vort, uy * vort
        wv, _ = self._traces(vort)
        uv, _ = self._traces_flux(ux, uy)
        flx = uv * wv
        bvals = self._boundary_face_values(self.bc_adv)
        inter = self.f_nbr >= 0
        flx = np.where(inter[..., None], flx, bvals)
        fn, sgn = self._nbr_gather(flx)
        wn, _ = self._nbr_gather(wv)
        up = flx.copy()
        s = sgn[..., None]
        avg = 0.5 * (flx + s * fn)
        dw = wv - wn
        big = np.abs(np.real(dw)) > 1e-4
        a = np.where(big, (flx - s * fn) / np.where(big, dw, 1.0), 0.0)
        # |a| written as a sgn(Re a): the same value, and complex-step differentiable
        upw = avg + np.where(big, 0.5 * SGN[None, :, None] * (a * np.sign(np.real(a))) * dw, 0.0)
        up[inter] = upw[inter]
        return self._lift_divergence(fx, fy, up)

    def _traces_flux(self, ux, uy):
        B = self.B
        v = np.stack([ux @ B.sbb[:, 0], ux @ B.sbb[:, 1],
                      np.einsum("emi,m->ei", uy, B.sbb[:, 0]), np.einsum("emi,m->ei", uy, B.sbb[:, 1])], 1)
        return v, None

    def rhs_advection_continuous(self, vort):
        """-div(u omega) with a continuous volumetric flux and pure upwinding (src/HO_2D.cpp:2439-2645)."""
        B, Mt = self.B, self.M
        u, v = self.vel[..., 0], self.vel[..., 1]
        dx = u * Mt["yeta"] - v * Mt["xeta"]
        dy = -u * Mt["yxi"] + v * Mt["xxi"]
        bvf, _ = self._traces_flux(dx, dy)
        bnv = self._boundary_face_values(self.bc_nv) * Mt["fAn"]
        bvn, sgn = self._nbr_gather(bvf)
        inter = self.f_nbr >= 0
        cvf = np.where(inter[..., None], 0.5 * (bvf + sgn[..., None] * bvn), bnv)
        R = B.R
        cx = dx + (cvf[:, 0] - bvf[:, 0])[:, :, None] * R[:, 0][None, None, :] \
            + (cvf[:, 1] - bvf[:, 1])[:, :, None] * R[:, 1][None, None, :]
        cy = dy + (cvf[:, 2] - bvf[:, 2])[:, None, :] * R[:, 0][None, :, None] \
            + (cvf[:, 3] - bvf[:, 3])[:, None, :] * R[:, 1][None, :, None]
        fx, fy = cx * vort, cy * vort
        wv, _ = self._traces(vort)
        wn, _ = self._nbr_gather(wv)
        t = (np.arange(4) % 2)[None, :, None].astype(float)
        pos = np.real(cvf) > 0.0
        upw = np.where(pos, cvf * (t * wv + (1 - t) * wn), cvf * ((1 - t) * wv + t * wn))
        up = np.where(inter[..., None], upw, self._boundary_face_values(self.bc_adv))
        return self._lift_divergence(fx, fy, up)

    def stage(self, vort_in, coeff):
        """One explicit stage: k = dt * (advection + diffusion) (src/HO_2D.cpp:1806-1839)."""
        self.update_bcs(self.t + coeff * self.dt)
        self.solve_poisson(vort_in)
        self.velocity()
        self.update_diffusion_bc()
        self.rhs_diff = self.rhs_diffusion(vort_in)
        self.update_advection_bc()
        if self.adv_type == 1:
            self.rhs_adv = self.rhs_advection(vort_in)
        else:
            self.rhs_adv = self.rhs_advection_continuous(vort_in)
        return self.dt * (self.rhs_adv + self.rhs_diff)

    def step(self):
        """One time step (src/HO_2D.cpp:1465-1531)."""
        w = self.omega
        if self.ti_type == 1:
            self.omega = w + self.stage(w, 0.0)
        elif self.ti_type == 2:
            k1 = self.stage(w, 0.0)
            k2 = self.stage(w + k1, 1.0)
            self.omega = w + 0.5 * (k1 + k2)
        else:
            k1 = self.stage(w, 0.0)
            k2 = self.stage(w + 0.5 * k1, 0.5)
            k3 = self.stage(w + 0.5 * k2, 0.5)
            k4 = self.stage(w + k3, 1.0)
            self.omega = w + (k1 + 2.0 * k2 + 2.0 * k3 + k4) / 6.0
        self.t += self.dt

    def run(self, nsteps):
        for _ in range(nsteps):
            self.step()
