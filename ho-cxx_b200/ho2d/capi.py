"""ctypes binding of the C ABI in include/ho2d.h (libho2d.so, built in-tree).

Loading fails loudly when the library is missing: there is no CPU fallback.
"""

from __future__ import annotations

import ctypes
import os

import numpy as np

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_lib", "libho2d.so")

HO2D_OK = 0
STATUS = {0: "HO2D_OK", 1: "HO2D_ERR_ARG", 2: "HO2D_ERR_IO", 3: "HO2D_ERR_MESH", 4: "HO2D_ERR_UNSUPPORTED",
          5: "HO2D_ERR_CUDA", 6: "HO2D_ERR_NOT_CONVERGED", 7: "HO2D_ERR_NONFINITE"}
FP64, MIXED, MIXED_KRYLOV = 0, 1, 2
BC_POISSON, BC_NORMAL_VEL, BC_PARL_VEL, BC_DIFFUSION, BC_VORTICITY, BC_VELOCITY_JUMP, BC_ADVECTION = range(7)
SMOOTHER_BLOCKS, SMOOTHER_BF16, SMOOTHER_KRON = range(3)
SETUP_DINV, SETUP_ROWSUM, SETUP_COLSUM, SETUP_BSUM, SETUP_BSRC, SETUP_BCOL = range(6)
FIELD_VORTICITY, FIELD_STREAMFUNCTION, FIELD_RHS_DIFFUSIVE, FIELD_RHS_ADVECTIVE, FIELD_STAGE_K, FIELD_JACOBIAN = range(6)

# exported symbol -> (restype, argtypes); every name declared in include/ho2d.h
_P = ctypes.c_void_p
_I = ctypes.c_int32
_D = ctypes.c_double
_DP = ctypes.POINTER(ctypes.c_double)
_IP = ctypes.POINTER(ctypes.c_int32)
SIGNATURES = {
    "ho2d_create": (ctypes.c_int, [ctypes.POINTER(_P)]),
    "ho2d_destroy": (ctypes.c_int, [_P]),
    "ho2d_read_input": (ctypes.c_int, [_P, ctypes.c_char_p]),
    "ho2d_setup": (ctypes.c_int, [_P]),
    "ho2d_solve": (ctypes.c_int, [_P]),
    "ho2d_step": (ctypes.c_int, [_P, _I]),
    "ho2d_stage": (ctypes.c_int, [_P, _D]),
    "ho2d_solveto": (ctypes.c_int, [_P, _D, _I, _I, _D, _I]),
    "ho2d_get_sizes": (ctypes.c_int, [_P, _IP, _IP, _IP, _IP]),
    "ho2d_get_vort": (ctypes.c_int, [_P, _I, _DP]),
    "ho2d_set_vort": (ctypes.c_int, [_P, _I, _DP]),
    "ho2d_get_psi": (ctypes.c_int, [_P, _I, _DP]),
    "ho2d_get_vel": (ctypes.c_int, [_P, _I, _DP]),
    "ho2d_get_field": (ctypes.c_int, [_P, _I, _I, _DP]),
    "ho2d_get_boundary": (ctypes.c_int, [_P, _I, _I, _DP]),
    "ho2d_set_boundary": (ctypes.c_int, [_P, _I, _I, _DP]),
    "ho2d_get_solution_points": (ctypes.c_int, [_P, _I, _DP]),
    "ho2d_set_precision": (ctypes.c_int, [_P, _I]),
    "ho2d_set_smoother": (ctypes.c_int, [_P, _I]),
    "ho2d_get_smoother": (ctypes.c_int, [_P, _IP, _IP]),
    "ho2d_set_device_setup": (ctypes.c_int, [_P, _I]),
    "ho2d_get_poisson_setup": (ctypes.c_int, [_P, _I, ctypes.c_int64, _DP]),
    "ho2d_set_poisson_tolerance": (ctypes.c_int, [_P, _D, _I]),
    "ho2d_poisson_stats": (ctypes.c_int, [_P, _IP, _DP]),
    "ho2d_get_time": (ctypes.c_int, [_P, _DP, _DP]),
    "ho2d_solve_counters": (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int64),
                                           ctypes.POINTER(ctypes.c_int64)]),
    "ho2d_fp64_finishes": (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_int64)]),
    "ho2d_set_time": (ctypes.c_int, [_P, _D]),
    "ho2d_time_steps": (ctypes.c_int, [_P, _I, _DP, _DP]),
    "ho2d_profile_spmv": (ctypes.c_int, [_P, _I, _DP, _DP]),
    "ho2d_profile_krylov": (ctypes.c_int, [_P, _I, _DP, _DP]),
    "ho2d_apply_poisson": (ctypes.c_int, [_P, _I, _DP, _DP]),
    "ho2d_apply_poisson_noalloc": (ctypes.c_int, [_P, _I, ctypes.c_void_p, ctypes.c_void_p]),
    "ho2d_get_forces": (ctypes.c_int, [_P, _DP, _DP]),
    "ho2d_get_boundary_points": (ctypes.c_int, [_P, _I, _DP]),
    "ho2d_set_output_dir": (ctypes.c_int, [_P, ctypes.c_char_p]),
    "ho2d_write_vtk": (ctypes.c_int, [_P, _I, _I, ctypes.c_char_p]),
    "ho2d_set_defaults": (ctypes.c_int, [_P]),
    "ho2d_enable_hybrid": (ctypes.c_int, [_P]),
    "ho2d_set_elemorder": (ctypes.c_int, [_P, _I]),
    "ho2d_load_mesh_arrays": (ctypes.c_int, [_P, _I, _I, _DP, _I, _IP, _I, _IP, _I, _IP]),
    "ho2d_load_inout_arrays": (ctypes.c_int, [_P, _I, _DP, _I, _IP, _I, _DP, _I, _IP]),
    "ho2d_process_mesh_input": (ctypes.c_int, [_P]),
    "ho2d_get_solution_areas": (ctypes.c_int, [_P, _I, _DP]),
    "ho2d_get_open_point_count": (ctypes.c_int, [_P, _IP]),
    "ho2d_get_open_points": (ctypes.c_int, [_P, _I, _DP]),
    "ho2d_set_open_velocities": (ctypes.c_int, [_P, _I, _DP]),
    "ho2d_set_open_vorticity": (ctypes.c_int, [_P, _I, _DP]),
    "ho2d_set_ptog_weights": (ctypes.c_int, [_P, _I, _DP]),
    "ho2d_get_hoquad_weights": (ctypes.c_int, [_P, _I, _DP]),
    "ho2d_clean_up": (ctypes.c_int, [_P]),
    "ho2d_set_adjoint_storage": (ctypes.c_int, [_P, _I]),
    "ho2d_adjoint_forward": (ctypes.c_int, [_P, _I, _I]),
    "ho2d_adjoint_backward": (ctypes.c_int, [_P, _I, _DP, _DP, _I, _DP]),
    "ho2d_stage_adjoint": (ctypes.c_int, [_P, _D, _I, _DP, _DP, _I, _DP]),
    "ho2d_apply_poisson_transpose": (ctypes.c_int, [_P, _I, _DP, _DP]),
    "ho2d_adjoint_stats": (ctypes.c_int, [_P, _IP, _DP]),
    "ho2d_last_launch_count": (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_int64)]),
    "ho2d_last_error": (ctypes.c_char_p, [_P]),
}

_lib = None


def load() -> ctypes.CDLL:
    """Load libho2d.so (raises if it was not built) and declare every signature."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m ho2d.build` (needs nvcc)")
        lib = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


class HO2DError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{STATUS.get(code, code)}: {msg}")
        self.code = code


def dptr(a: np.ndarray):
    return a.ctypes.data_as(_DP)


def iptr(a: np.ndarray):
    return a.ctypes.data_as(_IP)
