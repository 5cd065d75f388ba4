"""The library's host setup against the reference's own setup arrays, on the CPU.

tests/host_harness.cpp compiles the library's host code (ho-cxx_b200/csrc/host_io.cpp,
host_setup.cpp, host_hybrid.cpp, host_amg.cpp, host_kron.cpp) with g++ and sets up
  * each golden case from its input.dat and Gmsh mesh: the mesh tables, bases, metrics,
    boundary conditions and the Poisson operator's blocks are compared with the arrays the
    reference dumped after its setup (ref.npz: setup_mesh .. form_Laplace_operator_matrix);
  * each hybrid case from the driver's arrays (load_mesh_arrays_d, load_inout_arrays_d,
    process_mesh_input): mesh tables, Jacobians, the boundary conditions of problem type 11
    (wall / open / inlet / outlet switches and the inlet streamfunction chain), the
    boundary source, solution-point areas, open-boundary points and the normal / parallel
    split of the driver's open-boundary velocities against the reference's
    (hybrid_setup_ref.npz, hybrid_ref.npz).
Integer tables must be equal; FP64 values agree to round-off (1e-11 of the array's scale,
1e-13 for the bases).
"""

import ctypes
import json
import os
import shutil
import subprocess

import numpy as np
import pytest
import scipy.sparse as sp

from conftest import GOLDEN, GOLDEN_CASES, REPO, reference_root

CSRC = os.path.join(REPO, "ho-cxx_b200", "csrc")
HYB = os.path.join(GOLDEN, "hybrid")
HYB_CASES = sorted(d for d in os.listdir(HYB) if os.path.isfile(os.path.join(HYB, d, "hybrid_setup_ref.npz")))
TOL = 1e-11


@pytest.fixture(scope="module")
def lib(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    out = str(tmp_path_factory.mktemp("host_harness") / "libhost_harness.so")
    srcs = [os.path.join(REPO, "tests", "host_harness.cpp")] + [os.path.join(CSRC, f) for f in
                                                                 ("host_io.cpp", "host_setup.cpp", "host_hybrid.cpp",
                                                                  "host_amg.cpp", "host_kron.cpp")]
    subprocess.run(["g++", "-O1", "-std=c++17", "-shared", "-fPIC", "-I", CSRC, *srcs, "-o", out], check=True,
                   capture_output=True, text=True)
    L = ctypes.CDLL(out)
    L.case_from_input.restype = ctypes.c_void_p
    L.case_from_input.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.c_int)]
    L.case_from_arrays.restype = ctypes.c_void_p
    L.case_free.argtypes = [ctypes.c_void_p]
    L.case_dims.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_long)]
    L.case_group_name.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_char_p, ctypes.c_int]
    L.case_get.restype = ctypes.c_long
    L.case_get.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_void_p]
    L.case_split_open.argtypes = [ctypes.c_void_p] * 4
    L.case_check_block_reductions.restype = ctypes.c_long
    L.case_check_block_reductions.argtypes = [ctypes.c_void_p]
    L.case_build_hierarchy.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
    L.case_level_csr.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_char_p] + [ctypes.c_void_p] * 4
    L.case_level_ell.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_char_p] + [ctypes.c_void_p] * 3
    L.case_level_vec.restype = ctypes.c_long
    L.case_level_vec.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
    L.kron_eigs.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    L.kron_vecs.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    L.case_kron.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    L.case_kron_smoother.restype = ctypes.c_long
    L.case_kron_smoother.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
    L.bases_get.restype = ctypes.c_long
    L.bases_get.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_char_p, ctypes.c_void_p]
    return L


class HostCase:
    def __init__(self, lib, handle):
        self.lib, self.h = lib, handle
        d = (ctypes.c_long * 6)()
        lib.case_dims(handle, d)
        self.N, self.K, self.L, self.neb, self.ngroups, self.nnz = list(d)
        buf = ctypes.create_string_buffer(256)
        self.groups = []
        for g in range(self.ngroups):
            assert lib.case_group_name(handle, g, buf, 256) == 0
            self.groups.append(buf.value.decode())

    def __getitem__(self, name):
        n = self.lib.case_get(self.h, name.encode(), None)
        assert n >= 0, name
        out = np.zeros(n)
        self.lib.case_get(self.h, name.encode(), out.ctypes.data_as(ctypes.c_void_p))
        return out

    def ints(self, name):
        return self[name].astype(np.int64)

    def close(self):
        self.lib.case_free(self.h)


def rel(a, b):
    return float(np.abs(np.ravel(a) - np.ravel(b)).max() / max(np.abs(b).max(), 1e-300))


def close_abs(mine, ref, tol=TOL):
    """|mine - ref| <= tol * max(1, |ref|) elementwise scale of the whole array."""
    ref = np.asarray(ref, dtype=float)
    return float(np.abs(np.ravel(mine) - ref.ravel()).max(initial=0.0)) <= tol * max(1.0, np.abs(ref).max(initial=0.0))


def blocks_to_csr(c: HostCase):
    """The assembled operator from the block form: block (el, slot)[rs][ij] is
    A[el K^2 + ij, col K^2 + rs]; entries at or below 1e-14 in magnitude dropped as the
    reference's assembly does."""
    K2 = c.K * c.K
    blocks = c["blocks"].reshape(c.N, 5, K2, K2)
    col = c.ints("block_col").reshape(c.N, 5)
    rows, cols, vals = [], [], []
    ij = np.arange(K2)
    for el in range(c.N):
        for s in range(5):
            if col[el, s] < 0:
                continue
            b = blocks[el, s]  # [rs][ij]
            r = el * K2 + ij[None, :] + 0 * ij[:, None]
            cc = col[el, s] * K2 + ij[:, None] + 0 * ij[None, :]
            keep = np.abs(b) > 1e-14
            rows.append(r[keep])
            cols.append(cc[keep])
            vals.append(b[keep])
    n = c.N * K2
    return sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(n, n))


@pytest.fixture(scope="module", params=GOLDEN_CASES)
def golden(request, lib):
    d = os.path.join(GOLDEN, request.param)
    code = ctypes.c_int(0)
    h = lib.case_from_input(os.path.join(d, "input.dat").encode(), ctypes.byref(code))
    assert h, f"setup failed with code {code.value}"
    c = HostCase(lib, h)
    yield c, dict(np.load(os.path.join(d, "ref.npz"))), json.load(open(os.path.join(d, "meta.json")))
    c.close()


def test_mesh_tables(golden):
    c, ref, meta = golden
    assert (c.N, c.K, c.neb) == (meta["N_el"], meta["Knod"], meta["N_edges_boundary"])
    assert c.groups == meta["boundaries"]
    # elem_neighbor etc. are [el][side] with -1 where the side is on the boundary
    np.testing.assert_array_equal(c.ints("nbr"), ref["elem_neighbor"].ravel())
    np.testing.assert_array_equal(c.ints("nbr_side"), ref["elem_neighbor_side"].ravel())
    np.testing.assert_array_equal(c.ints("bidx"), ref["elem_boundary_index"].ravel())
    np.testing.assert_array_equal(c.ints("be_el"), ref["bedge_element"])
    np.testing.assert_array_equal(c.ints("be_side"), ref["bedge_side"])


def test_bases(golden):
    c, ref, _ = golden
    for mine, nm in [("xs", "sps_local_coor"), ("w", "sps_weight"), ("D", "sps_sps_grad_basis"),
                     ("R", "sps_radau"), ("gR", "sps_grad_radau"), ("sbb", "sps_boundary_basis"),
                     ("sbgb", "sps_boundary_grad_basis")]:
        assert rel(c[mine], ref[nm]) < 1e-13, nm


def test_metrics(golden):
    c, ref, _ = golden
    for mine, nm in [("J", "vol_jac"), ("G", "G"), ("GB", "GB"), ("fJ", "face_jac"), ("fA", "face_Acoef"),
                     ("fAn", "face_Anorm")]:
        assert rel(c[mine], ref[nm]) < TOL, nm
    # face_Bcoef vanishes on affine meshes: compare absolutely against the face scale
    assert np.abs(c["fB"] - ref["face_Bcoef"].ravel()).max() <= TOL * np.abs(ref["face_Acoef"]).max()


def test_boundary_conditions(golden):
    c, ref, _ = golden
    np.testing.assert_array_equal(c.ints("sw_p"), ref["BC_switch_Poisson"])
    np.testing.assert_array_equal(c.ints("sw_d"), ref["BC_switch_diffusion"])
    for mine, nm in [("bc_p", "BC_Poisson"), ("bc_nv", "BC_normal_vel"), ("bc_pv", "BC_parl_vel"),
                     ("bc_d", "BC_diffusion")]:
        assert close_abs(c[mine], ref[nm]), nm


def test_poisson_operator(golden):
    c, ref, _ = golden
    n = c.N * c.K ** 2
    A = sp.csr_matrix((ref["A_val"], ref["A_col"], ref["A_ptr"][: n + 1]), shape=(n, n))
    mine = blocks_to_csr(c)
    assert c.nnz == A.nnz == mine.nnz
    assert abs(mine - A).max() <= 1e-13 * abs(A).max()
    assert rel(c["bsrc"], ref["boundary_source"]) < 1e-13


def test_block_jacobi_inverse(golden):
    """The inverse diagonal blocks of the block-Jacobi smoother."""
    c, _, _ = golden
    K2 = c.K * c.K
    blocks = c["blocks"].reshape(c.N, 5, K2, K2)
    col = c.ints("block_col").reshape(c.N, 5)
    dinv = c["dinv"].reshape(c.N, K2, K2)
    for el in range(c.N):
        assert col[el, 0] == el
        Dm = blocks[el, 0].T  # [ij][rs]
        assert np.abs(dinv[el].T @ Dm - np.eye(K2)).max() <= 1e-12 * np.linalg.cond(Dm)


def _two_matrix_gauss_jordan(D):
    """Gauss-Jordan with partial pivoting (first row of largest magnitude) on [A | I] for a
    stack of matrices, each step rounding a product and then a difference, as the host code
    does without FMA."""
    a = D.copy()
    N, n, _ = a.shape
    inv = np.broadcast_to(np.eye(n), a.shape).copy()
    ar = np.arange(N)
    for k in range(n):
        p = k + np.argmax(np.abs(a[:, k:, k]), axis=1)
        assert (a[ar, p, k] != 0.0).all()
        for m in (a, inv):
            rk = m[ar, k].copy()
            m[ar, k] = m[ar, p]
            m[ar, p] = rk
        d = 1.0 / a[:, k, k]
        a[:, k, :] *= d[:, None]
        inv[:, k, :] *= d[:, None]
        for i in range(n):
            if i != k:
                l = a[:, i, k].copy()
                a[:, i, :] -= l[:, None] * a[:, k, :]
                inv[:, i, :] -= l[:, None] * inv[:, k, :]
    return inv


def test_block_inverse_bits(golden):
    """The in-place inverse (one matrix, column swaps undone at the end; the AVX2 or the
    baseline clone, whichever this CPU selects) gives the same bits as the two-matrix
    elimination on every diagonal block."""
    c, _, _ = golden
    K2 = c.K * c.K
    Dm = c["blocks"].reshape(c.N, 5, K2, K2)[:, 0].transpose(0, 2, 1)  # [ij][rs]
    dinv = c["dinv"][: c.N * K2 * K2].reshape(c.N, K2, K2).transpose(0, 2, 1)
    assert np.array_equal(dinv, _two_matrix_gauss_jordan(Dm))


def test_streamed_block_reductions(golden):
    """assemble_poisson keeps the blocks only on request. The row, column and block sums it
    streams instead must be the sums of the kept blocks, bit for bit, in the summation order
    the preconditioner setups used. An assembly without the blocks must give the same
    outputs."""
    c, _, _ = golden
    assert c.lib.case_check_block_reductions(c.h) == 0


def _roundtrip_meshes():
    from ho2d import meshgen

    from test_vtk import q2_cavity

    return {"cavity_jittered": meshgen.cavity(6, jitter=0.2, seed=3),
            "bfs": meshgen.backward_facing_step(h=1.0 / 3.0, jitter=0.15, seed=2),
            "cylinder": meshgen.cylinder_ogrid(n_r=4, n_theta=12, r0=0.5, r1=3.0),
            "q2_cavity": q2_cavity(n=3)}


@pytest.mark.parametrize("name", ["cavity_jittered", "bfs", "cylinder", "q2_cavity"])
def test_msh_writer_reader_round_trip(lib, tmp_path, name):
    """meshgen.write_msh then the library's reader (read_msh, process_mesh): every element's
    nodes in Gmsh slot order, every boundary group with its edges, coordinates exact
    (written with 17 significant digits)."""
    from ho2d import meshgen

    mesh = _roundtrip_meshes()[name]
    meshgen.write_msh(mesh, str(tmp_path / "mesh.msh"))
    quadratic = mesh.quads.shape[1] == 9
    meshgen.write_input_dat(str(tmp_path / "input.dat"), "mesh.msh", knod=3, reyn=100.0, dt=1e-3, num_steps=1,
                            problem_type=1, lnod_in=2 if quadratic else 1)
    code = ctypes.c_int(0)
    h = lib.case_from_input(str(tmp_path / "input.dat").encode(), ctypes.byref(code))
    # problem type 1 only sets up the cavity's walls; any group names are accepted
    assert h, f"setup failed with code {code.value}"
    c = HostCase(lib, h)
    try:
        L2 = mesh.quads.shape[1]
        assert (c.N, c.L * c.L) == (mesh.n_el, L2)
        xy = c["node_xy"].reshape(-1, 2)
        el = c.ints("elem_nodes").reshape(c.N, L2)
        np.testing.assert_array_equal(xy[el], mesh.xy[mesh.quads])
        assert c.groups == list(mesh.boundaries)
        be = c.ints("bedge_nodes").reshape(c.neb, c.L)
        grp = c.ints("be_group")
        for g, nm in enumerate(c.groups):
            ref = mesh.boundaries[nm]
            mine = be[grp == g]
            assert len(mine) == len(ref), nm
            # ends as an unordered pair (the reader orients edges by their element), then the
            # midpoint of a quadratic edge; both hold the ends first
            def key(p):
                return tuple(sorted(map(tuple, p[:2]))) + tuple(map(tuple, p[2:]))

            assert sorted(key(xy[e]) for e in mine) == sorted(key(mesh.xy[e]) for e in ref), nm
    finally:
        c.close()


def _hybrid_arrays(name):
    d = os.path.join(HYB, name)
    spec = {}
    for line in open(os.path.join(d, "spec.txt")):
        k, v = line.split()
        spec[k] = float(v)
    arrays = {f[:-4]: np.load(os.path.join(d, f)) for f in os.listdir(d) if f.endswith(".npy")}
    return (spec, arrays, dict(np.load(os.path.join(d, "hybrid_setup_ref.npz"))),
            dict(np.load(os.path.join(d, "hybrid_ref.npz"))))


def _hybrid_case(lib, spec, a):
    h, code = _from_arrays(lib, spec, a)
    assert h, f"hybrid setup failed with code {code}"
    return HostCase(lib, h)


def _from_arrays(lib, spec, a):
    """case_from_arrays on a driver's arrays: (handle or None, status code)."""
    i32, f64 = np.int32, np.float64

    def arr(key, dt):
        v = np.ascontiguousarray(a.get(key, np.zeros(0, dt)), dtype=dt)
        return len(v), v

    keep = []

    def ptr(v):
        keep.append(v)
        return v.ctypes.data_as(ctypes.c_void_p)

    nxy, xy = arr("nodes", f64)
    nidx, el = arr("elems", i32)
    nw, wall = arr("wall", i32)
    no, opn = arr("open", i32)
    niv, inv = arr("inletvel", f64)
    ni, inl = arr("inlet", i32)
    nov, outv = arr("outletvel", f64)
    nout, outl = arr("outlet", i32)
    code = ctypes.c_int(0)
    ci = ctypes.c_int
    h = lib.case_from_arrays(ci(int(spec["knod"])), ci(int(spec["iorder"])), ci(nxy), ptr(xy), ci(nidx), ptr(el),
                             ci(nw), ptr(wall), ci(no), ptr(opn), ci(niv), ptr(inv), ci(ni), ptr(inl), ci(nov),
                             ptr(outv), ci(nout), ptr(outl), ctypes.byref(code))
    return h, code.value


@pytest.fixture(scope="module", params=HYB_CASES)
def hybrid(request, lib):
    spec, a, sref, rref = _hybrid_arrays(request.param)
    c = _hybrid_case(lib, spec, a)
    yield c, a, sref, rref
    c.close()


def test_hybrid_mesh_tables(hybrid):
    c, _, s, _ = hybrid
    np.testing.assert_array_equal(c.ints("nbr"), s["setup_elem_neighbor"].ravel())
    np.testing.assert_array_equal(c.ints("nbr_side"), s["setup_elem_neighbor_side"].ravel())
    np.testing.assert_array_equal(c.ints("be_el"), s["setup_bedge_element"])
    np.testing.assert_array_equal(c.ints("be_side"), s["setup_bedge_side"])
    np.testing.assert_array_equal(c.ints("be_group"), s["setup_bedge_group"])
    assert rel(c["J"], s["setup_vol_jac"]) < TOL
    assert rel(c["fAn"], s["setup_face_Anorm"]) < TOL


def test_hybrid_boundary_conditions(hybrid):
    c, _, s, _ = hybrid
    np.testing.assert_array_equal(c.ints("sw_p"), s["setup_BC_switch_Poisson"])
    np.testing.assert_array_equal(c.ints("sw_d"), s["setup_BC_switch_diffusion"])
    np.testing.assert_array_equal(c.ints("noslip"), s["setup_BC_no_slip"])
    for mine, nm in [("bc_p", "setup_BC_Poisson"), ("bc_nv", "setup_BC_normal_vel"),
                     ("bc_pv", "setup_BC_parl_vel"), ("bc_d", "setup_BC_diffusion")]:
        assert close_abs(c[mine], s[nm]), nm
    assert rel(c["bsrc"], s["setup_boundary_source"]) < 1e-13 if np.abs(s["setup_boundary_source"]).max() > 0 \
        else np.abs(c["bsrc"]).max() == 0


def test_hybrid_inlet_chain_carries_the_inflow(hybrid):
    """Independent of the reference: with inlets, the streamfunction on the walls differs
    by the flow that enters between them (psi changes by -len * v_n along an inlet)."""
    c, a, _, _ = hybrid
    if "inlet" not in a:
        pytest.skip("no inlets")
    K = c.K
    bc_p = c["bc_p"].reshape(c.neb, K)
    grp = c.ints("be_group")
    walls = bc_p[grp == c.groups.index("wall")]
    levels = np.unique(np.round(walls[:, 0], 12))
    nodes = a["nodes"].reshape(-1, 2)
    inl = a["inlet"].reshape(-1, 2)
    inflow = float(np.sum(-a["inletvel"] * np.linalg.norm(nodes[inl[:, 1]] - nodes[inl[:, 0]], axis=1)))
    assert len(levels) == 2
    assert abs(abs(levels[1] - levels[0]) - abs(inflow)) < 1e-12


def test_hybrid_areas_and_open_points(hybrid):
    c, _, _, r = hybrid
    assert rel(c["areas"], r["areas"]) < 1e-13
    if "openpts" in r:
        assert rel(c["openpts"], r["openpts"]) < 1e-13
    else:
        assert len(c["openpts"]) == 0


def test_hybrid_open_velocity_split(hybrid):
    c, a, s, _ = hybrid
    steps = sorted(int(k.rsplit("_", 1)[1]) for k in s if k.startswith("open_velnorm_end_"))
    if not steps:
        pytest.skip("no open boundary")
    K = c.K
    open_rows = np.flatnonzero(c.ints("be_group") == c.groups.index("open"))
    nrm = c["open_normals"].reshape(c.neb, K, 2)
    np.testing.assert_allclose(np.linalg.norm(nrm[open_rows], axis=-1), 1.0, rtol=1e-13)
    for st in steps:
        xyvel = np.ascontiguousarray(a[f"openvel_{st}"], dtype=np.float64)
        vn, vp = np.zeros(c.neb * K), np.zeros(c.neb * K)
        c.lib.case_split_open(c.h, xyvel.ctypes.data_as(ctypes.c_void_p), vn.ctypes.data_as(ctypes.c_void_p),
                              vp.ctypes.data_as(ctypes.c_void_p))
        vn, vp = vn.reshape(c.neb, K)[open_rows], vp.reshape(c.neb, K)[open_rows]
        assert close_abs(vn, s[f"open_velnorm_end_{st}"], 1e-13), st
        assert close_abs(vp, s[f"open_velparl_end_{st}"], 1e-13), st


# ---- coarse hierarchy of the Poisson preconditioner (host_amg.cpp) ----------------------


def _level(c, level, which):
    dims = (ctypes.c_long * 3)()
    if c.lib.case_level_csr(c.h, level, which.encode(), dims, None, None, None) != 0:
        return None
    n, m, nnz = list(dims)
    ptr, col, val = np.zeros(n + 1, np.int32), np.zeros(nnz, np.int32), np.zeros(nnz)
    c.lib.case_level_csr(c.h, level, which.encode(), dims, ptr.ctypes.data_as(ctypes.c_void_p),
                         col.ctypes.data_as(ctypes.c_void_p), val.ctypes.data_as(ctypes.c_void_p))
    return sp.csr_matrix((val, col, ptr), shape=(n, m))


def _vec(c, level):
    n = c.lib.case_level_vec(c.h, level, None)
    out = np.zeros(n)
    c.lib.case_level_vec(c.h, level, out.ctypes.data_as(ctypes.c_void_p))
    return out


@pytest.fixture(scope="module", params=["bfs2_rk4", "cyl4x8_rk4", "cavity24j"])
def hierarchy(request, lib, tmp_path_factory):
    """A coarse hierarchy forced to coarsen (dense-solve size 8, or 64 on the 24 x 24
    jittered cavity) and the assembled operator it starts from."""
    if request.param.startswith("cavity"):
        from ho2d import meshgen

        inp = meshgen.make_case("cavityj24", str(tmp_path_factory.mktemp("amg")), knod=3, jitter=0.2, seed=7)
        dense = 64
    else:
        inp = os.path.join(GOLDEN, request.param, "input.dat")
        dense = 8
    code = ctypes.c_int(0)
    h = lib.case_from_input(inp.encode(), ctypes.byref(code))
    assert h, code.value
    c = HostCase(lib, h)
    L = lib.case_build_hierarchy(h, dense, dense)
    assert L >= 2, L
    yield c, L, blocks_to_csr(c)
    c.close()


def _dense_close(a, b, tol=1e-12):
    a, b = np.asarray(a.todense() if sp.issparse(a) else a), np.asarray(b.todense() if sp.issparse(b) else b)
    return np.abs(a - b).max() <= tol * max(np.abs(b).max(), 1e-300)


def test_p0_level_is_the_galerkin_operator(hierarchy):
    """Level 0 = P^T A P for P the element indicator, A the assembled FR operator (which the
    Poisson test above pins to the reference's matrix)."""
    c, _, A = hierarchy
    K2 = c.K * c.K
    P = sp.csr_matrix((np.ones(c.N * K2), (np.arange(c.N * K2), np.repeat(np.arange(c.N), K2))),
                      shape=(c.N * K2, c.N))
    assert _dense_close(_level(c, 0, "A"), P.T @ A @ P)


def test_coarse_levels_are_galerkin_products(hierarchy):
    c, L, _ = hierarchy
    for l in range(L - 1):
        A, P, R = _level(c, l, "A"), _level(c, l, "P"), _level(c, l, "R")
        assert P.shape == (A.shape[0], _level(c, l + 1, "A").shape[0])
        assert P.shape[1] < P.shape[0]  # it coarsens
        assert _dense_close(R, P.T, 0.0)
        assert _dense_close(_level(c, l + 1, "A"), R @ A @ P)
        assert (np.asarray(abs(P).sum(axis=0)).ravel() > 0).all()  # no empty aggregate


def test_spai0_weights(hierarchy):
    c, L, _ = hierarchy
    for l in range(L):
        A = _level(c, l, "A")
        m = _vec(c, l)
        d = A.diagonal()
        s = np.asarray(A.multiply(A).sum(axis=1)).ravel()
        np.testing.assert_allclose(m, d / s, rtol=1e-14)


def test_cycle_operators(hierarchy):
    """M = R (I - A diag(m)), S = 2 diag(m) - diag(m) A diag(m), Q = (I - diag(m) A) P, and
    together they are the V(1,1) two-level cycle with SPAI-0 smoothing from zero and an
    exact coarse solve."""
    c, L, _ = hierarchy
    rng = np.random.Generator(np.random.PCG64(9))
    for l in range(L - 1):
        A, P, R = _level(c, l, "A"), _level(c, l, "P"), _level(c, l, "R")
        m = _vec(c, l)
        Dm = sp.diags(m)
        I = sp.identity(A.shape[0])
        M, S, Q = _level(c, l, "M"), _level(c, l, "S"), _level(c, l, "Q")
        assert _dense_close(M, R @ (I - A @ Dm))
        assert _dense_close(S, 2 * Dm - Dm @ A @ Dm)
        assert _dense_close(Q, (I - Dm @ A) @ P)
        f = rng.standard_normal(A.shape[0])
        Ac = (R @ A @ P).toarray()
        u1 = m * f
        uc = np.linalg.solve(Ac, R @ (f - A @ u1))
        u2 = u1 + P @ uc
        u = u2 + m * (f - A @ u2)
        np.testing.assert_allclose(S @ f + Q @ np.linalg.solve(Ac, M @ f), u, rtol=1e-10,
                                   atol=1e-12 * np.abs(u).max())


def test_coarsest_dense_inverse(hierarchy):
    c, L, _ = hierarchy
    A = _level(c, L - 1, "A").toarray()
    inv = _vec(c, -1).reshape(A.shape)
    assert np.abs(inv @ A - np.eye(A.shape[0])).max() < 1e-10 * np.linalg.cond(A)


def test_ell_copies(hierarchy):
    c, L, _ = hierarchy
    for l in range(L):
        for which in ("A", "M", "S", "Q") if l < L - 1 else ("A",):
            A = _level(c, l, which)
            dims = (ctypes.c_long * 3)()
            assert c.lib.case_level_ell(c.h, l, which.encode(), dims, None, None) == 0
            n, m, w = list(dims)
            assert w % 4 == 0 and w >= np.diff(A.indptr).max()
            col, val = np.zeros(n * w, np.int32), np.zeros(n * w)
            c.lib.case_level_ell(c.h, l, which.encode(), dims, col.ctypes.data_as(ctypes.c_void_p),
                                 val.ctypes.data_as(ctypes.c_void_p))
            E = sp.csr_matrix((val, (np.repeat(np.arange(n), w), col)), shape=(n, m))  # padding adds zeros
            assert _dense_close(E, A, 0.0)


# ---- known answer: the reference's manufactured Poisson solution -----------------------


def _bilinear_points(c, xi, eta):
    """Physical coordinates of (xi, eta) in every bilinear element [N][..., 2]."""
    xy = c["node_xy"].reshape(-1, 2)
    en = c.ints("elem_nodes").reshape(c.N, 4)  # Gmsh slots SW, SE, NE, NW
    N = [(1 - xi) * (1 - eta) / 4, (1 + xi) * (1 - eta) / 4, (1 + xi) * (1 + eta) / 4, (1 - xi) * (1 + eta) / 4]
    return sum(N[a][None, ..., None] * xy[en[:, a]][(slice(None),) + (None,) * np.ndim(xi) + (slice(None),)]
               for a in range(4))


@pytest.mark.parametrize("jitter", [0.0, 0.2])
def test_manufactured_poisson_solution_converges_spectrally(lib, tmp_path, jitter):
    """The reference's Poisson test (src/HO_2D.cpp:1440, 1852-1879): omega =
    -4 (r^2 + 1) exp(r^2), so that Lap psi = -omega has psi = exp(r^2); Dirichlet psi =
    exp(r^2) on the walls of a 4 x 4 cavity. The library's assembled operator and boundary
    source (the Poisson right-hand side -omega J - boundary_source . BC_Poisson) solved
    exactly must approach exp(r^2) at the solution points spectrally in K."""
    from ho2d import meshgen

    errs = []
    for K in (3, 4, 5, 6, 7):
        d = tmp_path / f"k{K}_{jitter}"
        inp = meshgen.make_case("cavityj4" if jitter else "cavity4", str(d), knod=K, jitter=jitter, seed=3)
        code = ctypes.c_int(0)
        h = lib.case_from_input(inp.encode(), ctypes.byref(code))
        assert h, code.value
        c = HostCase(lib, h)
        try:
            xs = c["xs"]
            XI, ETA = np.meshgrid(xs, xs)  # [j][i]
            sp_xy = _bilinear_points(c, XI, ETA)  # [N][j][i][2]
            r2 = (sp_xy ** 2).sum(-1)
            omega = -4.0 * (r2 + 1.0) * np.exp(r2)
            # boundary flux points in boundary-array order: face point k of the element's
            # side, stored at (side / 2)(K - 2k - 1) + k
            bc_p = np.zeros((c.neb, K))
            be_el, be_side = c.ints("be_el"), c.ints("be_side")
            for e in range(c.neb):
                side = be_side[e]
                for k in range(K):
                    t = xs[k]
                    xi, eta = {0: (t, -1.0), 1: (1.0, t), 2: (t, 1.0), 3: (-1.0, t)}[side]
                    p = _bilinear_points(c, np.array(xi), np.array(eta))[be_el[e]]
                    bc_p[e, (side // 2) * (K - 2 * k - 1) + k] = np.exp((p ** 2).sum())
            K2 = K * K
            b = -(omega.reshape(c.N, K2) * c["J"].reshape(c.N, K2))
            bsrc = c["bsrc"].reshape(c.neb, K2, K)
            for e in range(c.neb):
                b[be_el[e]] -= bsrc[e] @ bc_p[e]
            from scipy.sparse.linalg import spsolve

            psi = spsolve(blocks_to_csr(c).tocsc(), b.ravel())
            errs.append(np.abs(psi - np.exp(r2).ravel()).max())
        finally:
            c.close()
    errs = np.array(errs)
    assert errs[-1] < 1e-6, errs
    assert (errs[1:] < errs[:-1] / 3).all(), errs


# ---- Kronecker-sum approximation of the diagonal blocks (host_kron.cpp) -----------------


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


@pytest.mark.parametrize("n", [2, 3, 5, 8])
def test_real_eigenvalues_and_vectors(lib, n):
    rng = np.random.Generator(np.random.PCG64(n))
    for trial in range(20):
        lam = np.sort(rng.uniform(-5, 5, n)) + np.arange(n) * 0.3  # distinct, real
        S = rng.standard_normal((n, n)) + 3 * np.eye(n)
        A = np.ascontiguousarray(S @ np.diag(lam) @ np.linalg.inv(S))
        got = np.zeros(n)
        assert lib.kron_eigs(n, _p(A), _p(got)) == 1, trial
        np.testing.assert_allclose(np.sort(got), np.sort(lam), rtol=1e-9, atol=1e-9 * np.abs(lam).max())
        V = np.zeros((n, n))
        assert lib.kron_vecs(n, _p(A), _p(got), _p(V)) == 1
        np.testing.assert_allclose(A @ V, V * got[None, :], atol=1e-7 * np.abs(A).max())
    # a rotation block has a complex pair: rejected
    R = np.eye(n)
    R[:2, :2] = [[0.0, -1.0], [1.0, 0.0]]
    Q = np.linalg.qr(rng.standard_normal((n, n)))[0]
    A = np.ascontiguousarray(Q @ R @ Q.T)
    assert lib.kron_eigs(n, _p(A), _p(np.zeros(n))) == 0


@pytest.mark.parametrize("name", ["bfs2_rk4", "cavj6_adv2", "cyl4x8_rk4"])
def test_kronecker_sum_fit_matches_its_definition(lib, name):
    """For every element: the fitted inverse applied by fast diagonalisation equals the
    inverse of I (x) Ax + Ay (x) I built densely from the least-squares fit of the block,
    and the defect ||I - M D||_2 equals its dense value."""
    code = ctypes.c_int(0)
    h = lib.case_from_input(os.path.join(GOLDEN, name, "input.dat").encode(), ctypes.byref(code))
    c = HostCase(lib, h)
    try:
        K, K2 = c.K, c.K * c.K
        blocks = c["blocks"].reshape(c.N, 5, K2, K2)
        rng = np.random.Generator(np.random.PCG64(5))
        ok = 0
        for el in range(c.N):
            D = blocks[el, 0].T.copy()  # [ij][rs]
            Dr = D.reshape(K, K, K, K)  # [j][i][l][k]
            Ax = np.einsum("jijk->ik", Dr) / K
            Ay = np.einsum("jili->jl", Dr) / K
            dg = np.einsum("jiji->ji", Dr)
            np.fill_diagonal(Ax, dg.mean(axis=0))
            np.fill_diagonal(Ay, dg.mean(axis=1) - dg.mean())
            Mfit = np.kron(np.eye(K), Ax) + np.kron(Ay, np.eye(K))
            r = rng.standard_normal(K2)
            z = np.zeros(K2)
            dfx = ctypes.c_double(0.0)
            if lib.case_kron(h, el, _p(r), _p(z), ctypes.byref(dfx)) != 1:
                assert np.iscomplexobj(np.linalg.eigvals(Ax)) or np.iscomplexobj(np.linalg.eigvals(Ay))
                continue
            ok += 1
            Minv = np.linalg.inv(Mfit)
            np.testing.assert_allclose(z, Minv @ r, rtol=1e-7, atol=1e-9 * np.abs(Minv @ r).max())
            exact = np.linalg.norm(np.eye(K2) - Minv @ D, 2)
            assert exact * (1 - 1e-3) <= dfx.value <= exact * (1 + 1e-9), (el, dfx.value, exact)
        assert ok >= 0.9 * c.N
    finally:
        c.close()


@pytest.mark.parametrize("case,knod,expect", [("bfs", 5, 41), ("cavityj64", 7, 348)])
def test_kronecker_smoother_fallback_counts(lib, tmp_path, case, knod, expect):
    """The elements that keep the exact inverse block (defect ||I - M D||_2 > 0.5): as many
    as the numpy study of this smoother found on the same meshes (bench step, K = 5: 41 of
    14,625; jittered 64^2 cavity, K = 7: 348 of 4,096), within the power iteration's
    underestimate of the defect."""
    from ho2d import meshgen

    inp = meshgen.make_case(case, str(tmp_path), knod=knod, steps=1)
    code = ctypes.c_int(0)
    h = lib.case_from_input(inp.encode(), ctypes.byref(code))
    assert h, code.value
    c = HostCase(lib, h)
    try:
        defect = np.zeros(c.N)
        n = lib.case_kron_smoother(h, _p(defect))
        assert abs(n - expect) <= max(2, expect // 50), (n, expect)
        assert n == int((~(defect <= 0.5)).sum())
        assert np.median(defect[np.isfinite(defect)]) < 0.3
    finally:
        c.close()


# ---- bases for every supported order (the reference stops at K = 5) ---------------------


def _bases(lib, K, L, name):
    n = lib.bases_get(K, L, name.encode(), None)
    assert n > 0, (K, L, name, n)
    out = np.zeros(n)
    lib.bases_get(K, L, name.encode(), _p(out))
    return out


@pytest.mark.parametrize("K", range(1, 9))
def test_solution_bases_against_legendre(lib, K):
    """Gauss-Legendre points and weights (numpy's leggauss); Lagrange basis at the ends
    (partition of unity, exact for degree < K); D exact on polynomials of degree < K;
    the Radau corrections g_L = (-1)^K/2 (P_K - P_{K-1}) and g_R(x) = g_L(-x) with their
    derivatives at the points; and the constants g'(-1), g'(+1) = -K(K+1)/2, +K(K+1)/2 of
    the method-2 diffusion flux (src/HO_2D.cpp:548-549; not g_L's own end slope, which is
    -K^2/2)."""
    from numpy.polynomial import legendre as Lg

    xs, w = _bases(lib, K, 2, "xs"), _bases(lib, K, 2, "w")
    gx, gw = Lg.leggauss(K)
    np.testing.assert_allclose(xs, gx, atol=1e-15 * K)
    np.testing.assert_allclose(w, gw, atol=1e-14)
    assert abs(w.sum() - 2.0) < 1e-14
    sbb, sbgb = _bases(lib, K, 2, "sbb").reshape(K, 2), _bases(lib, K, 2, "sbgb").reshape(K, 2)
    D = _bases(lib, K, 2, "D").reshape(K, K)  # D[k][m] = l_k'(x_m)
    np.testing.assert_allclose(sbb.sum(axis=0), 1.0, atol=1e-13)
    for deg in range(K):
        p = np.polynomial.Polynomial.basis(deg)
        vals = p(xs)
        np.testing.assert_allclose(vals @ sbb, p(np.array([-1.0, 1.0])), atol=1e-12 * 4 ** K)
        np.testing.assert_allclose(vals @ sbgb, p.deriv()(np.array([-1.0, 1.0])), atol=1e-11 * 4 ** K)
        np.testing.assert_allclose(vals @ D, p.deriv()(xs), atol=1e-11 * 4 ** K)
    R, gR = _bases(lib, K, 2, "R").reshape(K, 2), _bases(lib, K, 2, "gR").reshape(K, 2)
    cK = np.zeros(K + 1)
    cK[K] = 1.0
    cK1 = np.zeros(K + 1)
    cK1[K - 1] = 1.0
    gL = 0.5 * (-1) ** K * (cK - cK1)
    gLd = Lg.legder(gL)
    assert abs(Lg.legval(-1.0, gL) - 1.0) < 1e-14 and abs(Lg.legval(1.0, gL)) < 1e-14
    np.testing.assert_allclose(R[:, 0], Lg.legval(xs, gL), atol=1e-13)
    np.testing.assert_allclose(R[:, 1], Lg.legval(-xs, gL), atol=1e-13)
    np.testing.assert_allclose(gR[:, 0], Lg.legval(xs, gLd), atol=1e-11 * K * K)
    np.testing.assert_allclose(gR[:, 1], -Lg.legval(-xs, gLd), atol=1e-11 * K * K)
    gp = _bases(lib, K, 2, "gp")
    np.testing.assert_allclose(gp, [-K * (K + 1) / 2, K * (K + 1) / 2], rtol=1e-15)
    np.testing.assert_allclose(Lg.legval(-1.0, gLd), -K * K / 2, rtol=1e-12)


@pytest.mark.parametrize("L", [2, 3, 4])
def test_geometry_bases(lib, L):
    """Equispaced Lagrange basis of the L geometry nodes at the solution points and at the
    ends: partition of unity, exact for degree < L, derivatives likewise."""
    K = 5
    xs = _bases(lib, K, L, "xs")
    gsb, gsgb = _bases(lib, K, L, "gsb").reshape(L, K), _bases(lib, K, L, "gsgb").reshape(L, K)
    gbb, gbgb = _bases(lib, K, L, "gbb").reshape(L, 2), _bases(lib, K, L, "gbgb").reshape(L, 2)
    nodes = np.linspace(-1.0, 1.0, L)
    ends = np.array([-1.0, 1.0])
    for deg in range(L):
        p = np.polynomial.Polynomial.basis(deg)
        np.testing.assert_allclose(p(nodes) @ gsb, p(xs), atol=1e-13)
        np.testing.assert_allclose(p(nodes) @ gsgb, p.deriv()(xs), atol=1e-12)
        np.testing.assert_allclose(p(nodes) @ gbb, p(ends), atol=1e-13)
        np.testing.assert_allclose(p(nodes) @ gbgb, p.deriv()(ends), atol=1e-12)


def test_bases_reject_unsupported_orders(lib):
    assert lib.bases_get(0, 2, b"xs", None) < 0
    assert lib.bases_get(9, 2, b"xs", None) < 0


def test_affine_metrics_are_constant(lib, tmp_path):
    """A mesh of equal parallelograms (the unit cavity sheared by x += 0.3 y, 3 x 3 cells):
    x_xi = h/2, y_xi = 0, x_eta = 0.3 h/2, y_eta = h/2, J = h^2/4 at every solution point,
    and every face Jacobian |g| is the half-length of its edge."""
    from ho2d import meshgen

    n, h = 3, 1.0 / 3
    m = meshgen.cavity(n)
    m.xy = m.xy.copy()
    m.xy[:, 0] += 0.3 * m.xy[:, 1]
    meshgen.write_msh(m, str(tmp_path / "mesh.msh"))
    meshgen.write_input_dat(str(tmp_path / "input.dat"), "mesh.msh", knod=4, reyn=100.0, dt=1e-3, num_steps=1,
                            problem_type=1)
    code = ctypes.c_int(0)
    hd = lib.case_from_input(str(tmp_path / "input.dat").encode(), ctypes.byref(code))
    assert hd, code.value
    c = HostCase(lib, hd)
    try:
        np.testing.assert_allclose(c["J"], h * h / 4, rtol=1e-13)
        for name, val in (("xxi", h / 2), ("yxi", 0.0), ("xeta", 0.3 * h / 2), ("yeta", h / 2)):
            np.testing.assert_allclose(c[name], val, atol=1e-14, err_msg=name)
        fAn = c["fAn"].reshape(c.N, 4, c.K)  # ijp 0, 1: W/E faces (along eta); 2, 3: S/N (along xi)
        np.testing.assert_allclose(fAn[:, :2], np.hypot(0.3, 1.0) * h / 2, rtol=1e-13)
        np.testing.assert_allclose(fAn[:, 2:], h / 2, rtol=1e-13)
        G = c["G"].reshape(c.N, c.K, c.K, 2, 2)  # (g_r . g_s) / J, constant
        np.testing.assert_allclose(G - G[:1, :1, :1], 0.0, atol=1e-12)
    finally:
        c.close()


# ---- host-side fault injection: malformed meshes from a driver's arrays ------------------

_XY = [[0, 0], [1, 0], [2, 0], [0, 1], [1, 1], [2, 1]]
_QUADS = [[0, 1, 4, 3], [1, 2, 5, 4]]
_WALL = [[0, 1], [1, 2], [2, 5], [5, 4], [4, 3], [3, 0]]


def _arrays_case(lib, xy, quads, wall):
    spec = {"knod": 3, "iorder": 1}
    a = {"nodes": np.asarray(xy, float).ravel(), "elems": np.asarray(quads, np.int32).ravel(),
         "wall": np.asarray(wall, np.int32).ravel()}
    h, code = _from_arrays(lib, spec, a)
    return (HostCase(lib, h) if h else None), code


@pytest.mark.parametrize("what,xy,quads,wall", [
    ("an element side no boundary edge covers", _XY, _QUADS, _WALL[:-1]),
    ("a boundary edge inside the mesh", _XY, _QUADS, _WALL + [[1, 4]]),
    ("a boundary edge on no element", _XY, _QUADS, _WALL + [[0, 5]]),
    ("an edge shared by three elements", _XY + [[1, 2]], _QUADS + [[4, 1, 6, 6]], _WALL),
    ("a quad with a repeated node", _XY, [[0, 1, 4, 4], [1, 2, 5, 4]], _WALL),
    ("a boundary edge given twice", _XY, _QUADS, _WALL + [[0, 1]]),
])
def test_malformed_mesh_arrays_are_rejected(lib, what, xy, quads, wall):
    """process_mesh returns the malformed-mesh code (3) instead of building tables whose
    indices the kernels would follow."""
    c, code = _arrays_case(lib, xy, quads, wall)
    assert c is None and code == 3, what


def test_clockwise_quad_has_negative_jacobian(lib):
    """A clockwise quad passes the mesh processing; its Jacobian is negative, which the
    library's setup rejects (non-positive element Jacobian, code 3)."""
    c, code = _arrays_case(lib, _XY, [[0, 3, 4, 1], [1, 2, 5, 4]], _WALL)
    assert code == 0
    try:
        J = c["J"].reshape(2, -1)
        assert (J[0] < 0).all() and (J[1] > 0).all()
    finally:
        c.close()


# ---- the reference's own shipped meshes (read where they lie; skipped without them) -----

REFERENCE_INPUT = os.path.join(reference_root(), "input")
REF_BIN = os.path.join(REPO, "oracle", "_ref", "ho2d_ref")


@pytest.mark.parametrize("dat", ["input_cavity.dat", "input_bfs.dat", "input_cylinder.dat"])
def test_host_setup_on_shipped_meshes(lib, tmp_path, dat):
    """The reference's shipped inputs (quadratic cavity and step meshes, the OCC-oriented
    cylinder at K = 3): the library's host setup against the reference's own setup dump
    (oracle/_ref/ho2d_ref --setup) of the same files."""
    if not (os.path.isdir(REFERENCE_INPUT) and os.path.exists(REF_BIN)):
        pytest.skip("the reference's input/ directory or oracle/_ref/ho2d_ref is not available")
    lines = open(os.path.join(REFERENCE_INPUT, dat)).read().split("\n")
    shutil.copy(os.path.join(REFERENCE_INPUT, lines[7].strip()), tmp_path)
    lines[27] = "1"  # one time step: only the setup is compared
    inp = tmp_path / "input.dat"
    inp.write_text("\n".join(lines))
    env = dict(os.environ, HO_SHIM_SOLVER="direct")
    subprocess.run([REF_BIN, str(inp), str(tmp_path / "ref"), "--setup"], check=True, env=env,
                   stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL, timeout=600)
    ref = {f[:-4]: np.load(tmp_path / "ref" / f) for f in os.listdir(tmp_path / "ref") if f.endswith(".npy")}
    meta = json.load(open(tmp_path / "ref" / "meta.json"))
    code = ctypes.c_int(0)
    h = lib.case_from_input(str(inp).encode(), ctypes.byref(code))
    assert h, code.value
    c = HostCase(lib, h)
    try:
        assert (c.N, c.K, c.L, c.neb) == (meta["N_el"], meta["Knod"], meta["Lnod"], meta["N_edges_boundary"])
        assert c.groups == meta["boundaries"]
        for mine, nm in [("nbr", "elem_neighbor"), ("nbr_side", "elem_neighbor_side"),
                         ("bidx", "elem_boundary_index"), ("be_el", "bedge_element"), ("be_side", "bedge_side"),
                         ("sw_p", "BC_switch_Poisson"), ("sw_d", "BC_switch_diffusion")]:
            np.testing.assert_array_equal(c.ints(mine), ref[nm].ravel(), err_msg=nm)
        for mine, nm in [("J", "vol_jac"), ("G", "G"), ("GB", "GB"), ("fJ", "face_jac"), ("fA", "face_Acoef"),
                         ("fAn", "face_Anorm")]:
            assert rel(c[mine], ref[nm]) < TOL, nm
        assert np.abs(c["fB"] - ref["face_Bcoef"].ravel()).max() <= TOL * np.abs(ref["face_Acoef"]).max()
        for mine, nm in [("bc_p", "BC_Poisson"), ("bc_nv", "BC_normal_vel"), ("bc_pv", "BC_parl_vel"),
                         ("bc_d", "BC_diffusion")]:
            assert close_abs(c[mine], ref[nm]), nm
        n = c.N * c.K ** 2
        A = sp.csr_matrix((ref["A_val"], ref["A_col"], ref["A_ptr"][: n + 1]), shape=(n, n))
        mine = blocks_to_csr(c)
        assert c.nnz == A.nnz == mine.nnz
        assert abs(mine - A).max() <= 1e-12 * abs(A).max()
        assert rel(c["bsrc"], ref["boundary_source"]) < 1e-12
    finally:
        c.close()


def test_host_code_under_sanitizers(tmp_path):
    """tests/sanitizer_driver.cpp runs the host code end to end under AddressSanitizer and
    UndefinedBehaviorSanitizer (leak checks on). It covers the mesh reader, the setup, the
    streamed and Kronecker-sum assembly, the coarse hierarchy, sample points, the VTK queue
    and the hybrid geometry, on bilinear and curved golden meshes with sample points inside
    and outside the domain. Any report fails the run."""
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    exe = str(tmp_path / "drv")
    srcs = [os.path.join(REPO, "tests", "sanitizer_driver.cpp")] + [os.path.join(CSRC, f) for f in (
        "host_io.cpp", "host_setup.cpp", "host_amg.cpp", "host_kron.cpp", "host_samples.cpp", "host_hybrid.cpp",
        "output_host.cpp")]
    r = subprocess.run(["g++", "-std=c++17", "-O1", "-g", "-fsanitize=address,undefined", "-fno-omit-frame-pointer",
                        "-I", CSRC, *srcs, "-o", exe, "-lpthread"], capture_output=True, text=True)
    if r.returncode != 0 and "sanitize" in r.stderr:
        pytest.skip("sanitizer runtimes not available")
    assert r.returncode == 0, r.stderr[-2000:]
    samples = tmp_path / "samples.dat"
    samples.write_text("0.2 0.3\n0.7 0.8\n-0.1 0.5\n0.5 1.2\n")
    args = []
    for case in ("bfs2_rk4", "cavq3_rk4", "cyl4x8_rk4", "cavj6_adv2"):
        args += [os.path.join(GOLDEN, case, "input.dat"), str(samples)]
    out = tmp_path / "vtk"
    out.mkdir()
    env = dict(os.environ, ASAN_OPTIONS="detect_leaks=1:halt_on_error=1",
               UBSAN_OPTIONS="print_stacktrace=1:halt_on_error=1")
    r = subprocess.run([exe, *args, str(out)], capture_output=True, text=True, env=env, timeout=600)
    assert r.returncode == 0 and "runtime error" not in r.stderr and "Sanitizer" not in r.stderr, r.stderr[-3000:]
    assert r.stdout.count("vtk 0") == 4, r.stdout


def test_bf16_rounding_matches_torch(lib):
    """The rounding of the optional BF16 smoother blocks: round to nearest, ties to even,
    bit for bit against torch's float32 -> bfloat16 conversion, on random values over the
    whole finite range, exact ties, values one ulp either side of them, and subnormals."""
    torch = pytest.importorskip("torch")
    rng = np.random.Generator(np.random.PCG64(12))
    bits = rng.integers(0, 0x7F7FFFFF, 200000, dtype=np.uint32) | (rng.integers(0, 2, 200000, dtype=np.uint32) << 31)
    ties = (rng.integers(0, 0x7F7F, 5000, dtype=np.uint32) << 16) | 0x8000
    x = np.concatenate([bits, ties, ties + 1, ties - 1, np.arange(1, 5000, dtype=np.uint32)]).view(np.float32)
    x = np.ascontiguousarray(x)
    out = np.zeros(x.size, np.uint16)
    lib.bf16_array.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
    lib.bf16_array(x.ctypes.data, out.ctypes.data, x.size)
    ref = torch.from_numpy(x).to(torch.bfloat16).view(torch.int16).numpy().view(np.uint16)
    np.testing.assert_array_equal(out, ref)


@pytest.mark.parametrize("name", ["bfs2_rk4", "cavq3_rk4", "cyl4x8_rk4"])
def test_kronecker_element_body_matches_host_apply(lib, name):
    """The element body the device smoother will run (kron_apply.cuh, host build with one
    thread) against kron_apply on every element's fitted factors."""
    lib.case_kron_body.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    code = ctypes.c_int(0)
    h = lib.case_from_input(os.path.join(GOLDEN, name, "input.dat").encode(), ctypes.byref(code))
    c = HostCase(lib, h)
    try:
        K2 = c.K * c.K
        rng = np.random.Generator(np.random.PCG64(8))
        for el in range(c.N):
            r = rng.standard_normal(K2)
            z_body, z_host = np.zeros(K2), np.zeros(K2)
            dfx = ctypes.c_double(0.0)
            ok_host = lib.case_kron(h, el, _p(r), _p(z_host), ctypes.byref(dfx))
            ok_body = lib.case_kron_body(h, el, _p(r.copy()), _p(z_body))
            assert ok_host == ok_body
            if ok_body:
                np.testing.assert_allclose(z_body, z_host, rtol=1e-12, atol=1e-14 * np.abs(z_host).max())
    finally:
        c.close()


@pytest.mark.parametrize("name", ["bfs2_rk4", "cavq3_rk4", "cav4_euler_k3"])
def test_kronecker_device_arrays(lib, name):
    """The packed arrays the device smoother reads (kron_device_arrays) applied element by
    element as the kernel will (the element body on the factors, or the exact block where
    the fit falls back) equal the fitted inverse (kron_apply) and the exact inverse."""
    lib.case_kron_device.restype = ctypes.c_long
    lib.case_kron_device.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    code = ctypes.c_int(0)
    h = lib.case_from_input(os.path.join(GOLDEN, name, "input.dat").encode(), ctypes.byref(code))
    c = HostCase(lib, h)
    try:
        K2 = c.K * c.K
        r = np.random.Generator(np.random.PCG64(9)).standard_normal(c.N * K2)
        z = np.zeros_like(r)
        n_exact = lib.case_kron_device(h, _p(r), _p(z))
        assert n_exact >= 0
        dinv = c["dinv"][: c.N * K2 * K2].reshape(c.N, K2, K2)  # [rs][ij]
        exact = 0
        for el in range(c.N):
            re = r[el * K2:(el + 1) * K2].copy()
            zk = np.zeros(K2)
            dfx = ctypes.c_double(0.0)
            if lib.case_kron(h, el, _p(re), _p(zk), ctypes.byref(dfx)) and dfx.value <= 0.5:
                np.testing.assert_allclose(z[el * K2:(el + 1) * K2], zk, rtol=1e-12, atol=1e-14 * np.abs(zk).max())
            else:
                exact += 1
                np.testing.assert_allclose(z[el * K2:(el + 1) * K2], dinv[el].T @ re, rtol=1e-12)
        assert exact == n_exact
    finally:
        c.close()
