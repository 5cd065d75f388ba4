"""B200-native HO-CXX vorticity-streamfunction flux-reconstruction solver.

``HO_2D`` mirrors the member functions of the reference's ``HO_2D`` class
(src/HO_2D.hpp:219-290) on top of the C ABI in ``include/ho2d.h``; the whole time step
runs in the CUDA library ``ho2d/_lib/libho2d.so``.
"""

from __future__ import annotations

import ctypes

import numpy as np

from . import capi
from .capi import FP64, MIXED, MIXED_KRYLOV, HO2DError  # noqa: F401


class HO_2D:
    """One solver instance (one mesh), like the reference's ``HO_2D``.

    Errors raise :class:`HO2DError` with the C ABI's status code where the reference
    calls ``exit()`` or returns a non-zero char.
    """

    def __init__(self):
        self._lib = capi.load()
        h = ctypes.c_void_p()
        self._check(self._lib.ho2d_create(ctypes.byref(h)), handle=None)
        self._h = h
        self._setup = False

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            self._lib.ho2d_destroy(h)
            self._h = None

    close = __del__

    def _check(self, code: int, handle="self"):
        if code != capi.HO2D_OK:
            msg = self._lib.ho2d_last_error(self._h if handle == "self" else None) or b""
            raise HO2DError(code, msg.decode(errors="replace"))

    # -- setup sequence of src/main.cpp:44-75
    def read_input_file(self, path: str) -> int:
        self._check(self._lib.ho2d_read_input(self._h, str(path).encode()))
        return 0

    def setup(self) -> None:
        if not self._setup:
            self._check(self._lib.ho2d_setup(self._h))
            self._setup = True
            n, k, neb, lnod = (ctypes.c_int32() for _ in range(4))
            self._check(self._lib.ho2d_get_sizes(self._h, ctypes.byref(n), ctypes.byref(k), ctypes.byref(neb),
                                                 ctypes.byref(lnod)))
            self.N_el, self.Knod, self.N_edges_boundary, self.Lnod = n.value, k.value, neb.value, lnod.value

    # the reference's individual setup calls all map onto the one device setup
    def setup_mesh(self) -> int:
        self.setup()
        return 0

    allocate_arrays = setup_mesh
    setup_sps_gps = setup_mesh

    def read_process_sample_points(self) -> None:
        """Nothing to do: the setup reads the input's sample-points file."""

    form_bases = setup_mesh
    form_metrics = setup_mesh
    setup_IC_BC_SRC = setup_mesh
    form_Laplace_operator_matrix = setup_mesh

    # -- time stepping
    def solve_vorticity_streamfunction(self) -> int:
        self._check(self._lib.ho2d_solve(self._h))
        return 0

    def solve_advection_diffusion(self, nsteps: int = 1) -> int:
        self._check(self._lib.ho2d_step(self._h, int(nsteps)))
        return 0

    def Euler_time_integrate(self, coeff: float) -> np.ndarray:
        """One stage on the current vorticity; returns k = dt (advective + diffusive)."""
        self._check(self._lib.ho2d_stage(self._h, float(coeff)))
        return self.get_field(capi.FIELD_STAGE_K)

    def solveto_d(self, outerdt: float, numstep: int, integtype: int, reyn: float, region: int = 0) -> None:
        self._check(self._lib.ho2d_solveto(self._h, float(outerdt), int(numstep), int(integtype), float(reyn),
                                           int(region)))

    # -- data exchange
    def _vol(self, comps=1):
        return np.zeros((self.N_el, self.Knod, self.Knod) + ((comps,) if comps > 1 else ()), dtype=np.float64)

    def getallvorts_d(self) -> np.ndarray:
        out = self._vol()
        self._check(self._lib.ho2d_get_vort(self._h, out.size, capi.dptr(out)))
        return out

    get_vorticity = getallvorts_d

    def setsolnvort_d(self, vort) -> None:
        a = np.ascontiguousarray(vort, dtype=np.float64)
        self._check(self._lib.ho2d_set_vort(self._h, a.size, capi.dptr(a)))

    set_vorticity = setsolnvort_d

    def get_streamfunction(self) -> np.ndarray:
        out = self._vol()
        self._check(self._lib.ho2d_get_psi(self._h, out.size, capi.dptr(out)))
        return out

    def get_velocity(self) -> np.ndarray:
        out = self._vol(2)
        self._check(self._lib.ho2d_get_vel(self._h, out.size, capi.dptr(out)))
        return out

    def get_field(self, which: int) -> np.ndarray:
        out = self._vol()
        self._check(self._lib.ho2d_get_field(self._h, int(which), out.size, capi.dptr(out)))
        return out

    def get_boundary(self, which: int) -> np.ndarray:
        out = np.zeros((self.N_edges_boundary, self.Knod))
        self._check(self._lib.ho2d_get_boundary(self._h, int(which), out.size, capi.dptr(out)))
        return out

    def set_boundary(self, which: int, values) -> None:
        a = np.ascontiguousarray(values, dtype=np.float64)
        self._check(self._lib.ho2d_set_boundary(self._h, int(which), a.size, capi.dptr(a)))

    def getsolnpts_d(self) -> np.ndarray:
        out = self._vol(2)
        self._check(self._lib.ho2d_get_solution_points(self._h, out.size, capi.dptr(out)))
        return out

    def getsolnptlen(self) -> int:
        """Length of the getsolnpts_d array: x, y per solution point (src/HO_2D.cpp:3942-3944)."""
        return 2 * self.N_el * self.Knod * self.Knod

    # -- hybrid operation (src/HO_2D.hpp:251-290): an external Lagrangian driver
    def set_defaults(self) -> None:
        self._check(self._lib.ho2d_set_defaults(self._h))
        self._setup = False

    def enable_hybrid(self) -> None:
        self._check(self._lib.ho2d_enable_hybrid(self._h))

    def set_elemorder(self, knod: int) -> None:
        self._check(self._lib.ho2d_set_elemorder(self._h, int(knod)))

    def load_mesh_arrays_d(self, iorder: int, xy, elems, wall=(), open_=()) -> None:
        """Nodes (x, y pairs), elements (Lnod^2 Gmsh-ordered node indices each), and the
        "wall" and "open" boundary edges (Lnod node indices each, counter-clockwise)."""
        xy = np.ascontiguousarray(xy, dtype=np.float64).ravel()
        el = np.ascontiguousarray(elems, dtype=np.int32).ravel()
        w = np.ascontiguousarray(wall, dtype=np.int32).ravel()
        o = np.ascontiguousarray(open_, dtype=np.int32).ravel()
        self._check(self._lib.ho2d_load_mesh_arrays(self._h, int(iorder), xy.size, capi.dptr(xy), el.size,
                                                    capi.iptr(el), w.size, capi.iptr(w), o.size, capi.iptr(o)))

    def load_inout_arrays_d(self, velin=(), idxin=(), velout=(), idxout=()) -> None:
        vi = np.ascontiguousarray(velin, dtype=np.float64).ravel()
        ii = np.ascontiguousarray(idxin, dtype=np.int32).ravel()
        vo = np.ascontiguousarray(velout, dtype=np.float64).ravel()
        io = np.ascontiguousarray(idxout, dtype=np.int32).ravel()
        self._check(self._lib.ho2d_load_inout_arrays(self._h, vi.size, capi.dptr(vi), ii.size, capi.iptr(ii),
                                                     vo.size, capi.dptr(vo), io.size, capi.iptr(io)))

    def process_mesh_input(self) -> None:
        self._check(self._lib.ho2d_process_mesh_input(self._h))
        self._setup = True
        n, k, neb, lnod = (ctypes.c_int32() for _ in range(4))
        self._check(self._lib.ho2d_get_sizes(self._h, ctypes.byref(n), ctypes.byref(k), ctypes.byref(neb),
                                             ctypes.byref(lnod)))
        self.N_el, self.Knod, self.N_edges_boundary, self.Lnod = n.value, k.value, neb.value, lnod.value

    def getsolnareas_d(self) -> np.ndarray:
        out = self._vol()
        self._check(self._lib.ho2d_get_solution_areas(self._h, out.size, capi.dptr(out)))
        return out

    def getopenptlen(self) -> int:
        n = ctypes.c_int32()
        self._check(self._lib.ho2d_get_open_point_count(self._h, ctypes.byref(n)))
        return n.value

    def getopenpts_d(self) -> np.ndarray:
        out = np.zeros(self.getopenptlen())
        self._check(self._lib.ho2d_get_open_points(self._h, out.size, capi.dptr(out)))
        return out.reshape(-1, self.Knod, 2)

    def setopenvels_d(self, xyvel) -> None:
        a = np.ascontiguousarray(xyvel, dtype=np.float64).ravel()
        self._check(self._lib.ho2d_set_open_velocities(self._h, a.size, capi.dptr(a)))

    def setopenvort_d(self, vort) -> None:
        a = np.ascontiguousarray(vort, dtype=np.float64).ravel()
        self._check(self._lib.ho2d_set_open_vorticity(self._h, a.size, capi.dptr(a)))

    def setptogweights_d(self, wgt) -> None:
        a = np.ascontiguousarray(wgt, dtype=np.float64).ravel()
        self._check(self._lib.ho2d_set_ptog_weights(self._h, a.size, capi.dptr(a)))

    def get_hoquad_weights_d(self) -> np.ndarray:
        out = np.zeros((self.Knod, self.Knod))
        self._check(self._lib.ho2d_get_hoquad_weights(self._h, out.size, capi.dptr(out)))
        return out

    def set_output_dir(self, path) -> None:
        """Where solve_vorticity_streamfunction writes its VTK files (None: nowhere)."""
        self._check(self._lib.ho2d_set_output_dir(self._h, None if path is None else str(path).encode()))

    def trigger_write(self, indx: int, subidx: int = -1, path=None) -> None:
        """The reference's two VTK files of the current fields (save_vorticity_vtk,
        save_smooth_vtk) into path (None: the working directory)."""
        self._check(self._lib.ho2d_write_vtk(self._h, int(indx), int(subidx),
                                             None if path is None else str(path).encode()))

    def clean_up(self) -> None:
        self._check(self._lib.ho2d_clean_up(self._h))
        self._setup = False

    # -- controls and statistics
    def get_boundary_points(self) -> np.ndarray:
        """[N_eb][K][x, y] of the boundary flux points, in the boundary arrays' order."""
        out = np.zeros((self.N_edges_boundary, self.Knod, 2))
        self._check(self._lib.ho2d_get_boundary_points(self._h, out.size, capi.dptr(out)))
        return out

    def set_precision(self, mode: int) -> None:
        self._check(self._lib.ho2d_set_precision(self._h, int(mode)))

    def set_smoother(self, kind: int) -> None:
        """Smoother of the FP32 preconditioner for the next setup (capi.SMOOTHER_*; -1: default)."""
        self._check(self._lib.ho2d_set_smoother(self._h, int(kind)))

    def smoother(self):
        """(kind in use, elements that keep their exact inverse block under SMOOTHER_KRON)."""
        k, n = ctypes.c_int32(), ctypes.c_int32()
        self._check(self._lib.ho2d_get_smoother(self._h, ctypes.byref(k), ctypes.byref(n)))
        return k.value, n.value

    def set_device_setup(self, on: bool) -> None:
        """Assemble the Poisson operator on the device (True, the default) or the host, at the
        next setup."""
        self._check(self._lib.ho2d_set_device_setup(self._h, 1 if on else 0))

    def get_poisson_setup(self, which: int) -> np.ndarray:
        """One assembled Poisson array (capi.SETUP_*), shaped as ho2d.h describes it."""
        N, K, neb = self.N_el, self.Knod, self.N_edges_boundary
        K2 = K * K
        shape = {capi.SETUP_DINV: (N, K2, K2), capi.SETUP_ROWSUM: (N, 5, K2), capi.SETUP_COLSUM: (N, 5, K2),
                 capi.SETUP_BSUM: (N, 5), capi.SETUP_BSRC: (neb, K2, K), capi.SETUP_BCOL: (N, 5)}[which]
        out = np.zeros(shape)
        self._check(self._lib.ho2d_get_poisson_setup(self._h, int(which), out.size, capi.dptr(out)))
        return out

    def set_poisson_tolerance(self, rel_tol: float, max_iter: int) -> None:
        self._check(self._lib.ho2d_set_poisson_tolerance(self._h, float(rel_tol), int(max_iter)))

    def poisson_stats(self):
        it, res = ctypes.c_int32(), ctypes.c_double()
        self._check(self._lib.ho2d_poisson_stats(self._h, ctypes.byref(it), ctypes.byref(res)))
        return it.value, res.value

    def fp64_finishes(self) -> int:
        """Mixed solves since setup that the FP64 solve finished (stalled refinement)."""
        n = ctypes.c_int64()
        self._check(self._lib.ho2d_fp64_finishes(self._h, ctypes.byref(n)))
        return n.value

    def solve_counters(self):
        """(Poisson solves, Krylov iterations, refinement sweeps) since setup."""
        a, b, c = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        self._check(self._lib.ho2d_solve_counters(self._h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)))
        return a.value, b.value, c.value

    def time(self):
        t, dt = ctypes.c_double(), ctypes.c_double()
        self._check(self._lib.ho2d_get_time(self._h, ctypes.byref(t), ctypes.byref(dt)))
        return t.value, dt.value

    def set_time(self, t: float) -> None:
        self._check(self._lib.ho2d_set_time(self._h, float(t)))

    def time_steps(self, nsteps: int):
        """Advance nsteps and return (total device ms, Poisson device ms) from CUDA events."""
        tot, pois = ctypes.c_double(), ctypes.c_double()
        self._check(self._lib.ho2d_time_steps(self._h, int(nsteps), ctypes.byref(tot), ctypes.byref(pois)))
        return tot.value, pois.value

    def profile_spmv(self, reps: int = 20):
        """(average ms per launch, algorithmic bytes per launch) of the Poisson SpMV kernel."""
        ms, by = ctypes.c_double(), ctypes.c_double()
        self._check(self._lib.ho2d_profile_spmv(self._h, int(reps), ctypes.byref(ms), ctypes.byref(by)))
        return ms.value, by.value

    def profile_krylov(self, iterations: int = 20):
        """Per-launch device ms and algorithmic bytes of the Krylov kernels inside BiCGSTAB
        iterations on the current state: dict kernel -> (ms, bytes) for "smoother" (the fine
        part of the smoothing step), "operator", "xr_update", "coarse_cycle" and
        "smoother_combine" (the coarse correction and the face traces)."""
        ms = (ctypes.c_double * 5)()
        by = (ctypes.c_double * 5)()
        self._check(self._lib.ho2d_profile_krylov(self._h, int(iterations), ms, by))
        names = ("smoother", "operator", "xr_update", "coarse_cycle", "smoother_combine")
        return {n: (ms[i], by[i]) for i, n in enumerate(names)}

    def apply_poisson(self, x) -> np.ndarray:
        """y = A x with the device's (matrix-free) Poisson operator, FP64."""
        a = np.ascontiguousarray(x, dtype=np.float64)
        out = np.zeros_like(a)
        self._check(self._lib.ho2d_apply_poisson(self._h, a.size, capi.dptr(a), capi.dptr(out)))
        return out

    def forces(self):
        """FP64 force (fx = drag, fy = lift; density 1) on the boundary group "object"."""
        fx, fy = ctypes.c_double(), ctypes.c_double()
        self._check(self._lib.ho2d_get_forces(self._h, ctypes.byref(fx), ctypes.byref(fy)))
        return fx.value, fy.value

    # -- discrete adjoint (no counterpart in the reference; ho2d.adjoint wraps it for torch)
    def set_adjoint_storage(self, fp32: bool) -> None:
        """FP32 (True) or FP64 storage of the adjoint's checkpoints and stage states."""
        self._check(self._lib.ho2d_set_adjoint_storage(self._h, 1 if fp32 else 0))

    def adjoint_forward(self, nsteps: int, ckpt_every: int = 25) -> None:
        """nsteps time steps from the current state, keeping the vorticity every ckpt_every steps."""
        self._check(self._lib.ho2d_adjoint_forward(self._h, int(nsteps), int(ckpt_every)))

    def adjoint_backward(self, dJ_domegaT):
        """(dJ/d omega0 [N_el][K][K], dJ/d BC_parl_vel [N_eb][K]) from dJ/d omega(T)."""
        g = np.ascontiguousarray(dJ_domegaT, dtype=np.float64).ravel()
        gw = np.zeros_like(g)
        gpv = np.zeros(self.N_edges_boundary * self.Knod)
        self._check(self._lib.ho2d_adjoint_backward(self._h, g.size, capi.dptr(g), capi.dptr(gw), gpv.size,
                                                    capi.dptr(gpv)))
        return gw.reshape(self.N_el, self.Knod, self.Knod), gpv.reshape(self.N_edges_boundary, self.Knod)

    def stage_adjoint(self, coeff: float, lam_k):
        """Adjoint of Euler_time_integrate(coeff) at the current state: (lam of the stage
        input [N_el][K][K], lam of BC_parl_vel [N_eb][K]) from lam of k."""
        lk = np.ascontiguousarray(lam_k, dtype=np.float64).ravel()
        lw = np.zeros_like(lk)
        lpv = np.zeros(self.N_edges_boundary * self.Knod)
        self._check(self._lib.ho2d_stage_adjoint(self._h, float(coeff), lk.size, capi.dptr(lk), capi.dptr(lw),
                                                 lpv.size, capi.dptr(lpv)))
        return lw.reshape(self.N_el, self.Knod, self.Knod), lpv.reshape(self.N_edges_boundary, self.Knod)

    def apply_poisson_transpose(self, x) -> np.ndarray:
        """y = A^T x with the transposed matrix-free Poisson operator, FP64."""
        a = np.ascontiguousarray(x, dtype=np.float64)
        out = np.zeros_like(a)
        self._check(self._lib.ho2d_apply_poisson_transpose(self._h, a.size, capi.dptr(a), capi.dptr(out)))
        return out

    def adjoint_stats(self):
        """(iterations, relative residual) of the last transposed Poisson solve."""
        it, res = ctypes.c_int32(), ctypes.c_double()
        self._check(self._lib.ho2d_adjoint_stats(self._h, ctypes.byref(it), ctypes.byref(res)))
        return it.value, res.value

    def launch_count(self) -> int:
        n = ctypes.c_int64()
        self._check(self._lib.ho2d_last_launch_count(self._h, ctypes.byref(n)))
        return n.value
