"""The allocation-free operator entry point against the allocating one.

ho2d_apply_poisson_noalloc serves callers that cannot let a library call cudaMalloc
(codes that own all device memory through their own pool or a fixed budget): it works on
caller-owned device buffers and keeps its only working memory in a fixed array compiled
into the library. Here the caller's device buffers are allocated by the test itself.
"""

import ctypes
import os

import numpy as np
import pytest

from conftest import GOLDEN

from ho2d import HO_2D, capi, meshgen

pytestmark = pytest.mark.gpu

TOL = 1e-12  # same kernels, same operand: only the trace buffer's location differs


def _cudart():
    capi.load()  # libho2d.so pulls in the CUDA runtime it was linked against
    rt = ctypes.CDLL("libcudart.so.12")
    rt.cudaMalloc.argtypes = [ctypes.POINTER(ctypes.c_void_p), ctypes.c_size_t]
    rt.cudaFree.argtypes = [ctypes.c_void_p]
    rt.cudaMemcpy.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int]
    rt.cudaMemGetInfo.argtypes = [ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(ctypes.c_size_t)]
    return rt


def _free_bytes(rt):
    free, total = ctypes.c_size_t(), ctypes.c_size_t()
    assert rt.cudaMemGetInfo(ctypes.byref(free), ctypes.byref(total)) == 0
    return free.value


class DeviceArray:
    H2D, D2H = 1, 2

    def __init__(self, rt, n):
        self.rt, self.n, self.p = rt, n, ctypes.c_void_p()
        assert rt.cudaMalloc(ctypes.byref(self.p), n * 8) == 0

    def upload(self, a):
        a = np.ascontiguousarray(a, dtype=np.float64).ravel()
        assert self.rt.cudaMemcpy(self.p, a.ctypes.data, self.n * 8, self.H2D) == 0

    def download(self):
        out = np.empty(self.n)
        assert self.rt.cudaMemcpy(out.ctypes.data, self.p, self.n * 8, self.D2H) == 0
        return out

    def free(self):
        self.rt.cudaFree(self.p)


def _solver(inp):
    s = HO_2D()
    s.read_input_file(inp)
    s.setup()
    return s


@pytest.mark.parametrize("case", ["cav4_rk4", "cyl4x8_rk4", "bfs2_rk4"])
def test_noalloc_matches_allocating_entry_point_twice(case):
    rt = _cudart()
    s = _solver(os.path.join(GOLDEN, case, "input.dat"))
    n = s.N_el * s.Knod * s.Knod
    dx, dy = DeviceArray(rt, n), DeviceArray(rt, n)
    rng = np.random.Generator(np.random.PCG64(17))
    try:
        for _ in range(2):  # the second call sees the first call's leftovers in the shared array
            x = rng.standard_normal((s.N_el, s.Knod, s.Knod))
            y_ref = s.apply_poisson(x).ravel()
            dx.upload(x)
            # device memory is handed out in pages of at least 2 MiB: any allocation inside
            # the call would show as a drop of the free bytes
            free0 = _free_bytes(rt)
            code = s._lib.ho2d_apply_poisson_noalloc(s._h, n, dx.p, dy.p)
            assert code == 0, s._lib.ho2d_last_error(s._h)
            assert _free_bytes(rt) == free0
            y = dy.download()
            assert np.abs(y - y_ref).max() <= TOL * np.abs(y_ref).max()
    finally:
        dx.free()
        dy.free()


def test_noalloc_rejects_meshes_beyond_its_fixed_scratch(tmp_path):
    # 148 x 148 quads at Knod = 6: N_el * Knod = 131,424 > 131,072
    inp = meshgen.make_case("cavity148", str(tmp_path), knod=6, steps=1)
    rt = _cudart()
    s = _solver(inp)
    n = s.N_el * s.Knod * s.Knod
    dx, dy = DeviceArray(rt, n), DeviceArray(rt, n)
    try:
        code = s._lib.ho2d_apply_poisson_noalloc(s._h, n, dx.p, dy.p)
        assert code == 1  # HO2D_ERR_ARG
        assert b"fixed scratch" in s._lib.ho2d_last_error(s._h)
    finally:
        dx.free()
        dy.free()
