"""Poisson setup on the device against the host setup, through the C ABI.

The device assembles the block operator with the host's own element routine
(assemble_element.hpp) compiled without fused multiply-adds, so every assembled array -- the
inverse diagonal blocks, the row and column sums of every block, the block sums, the
boundary source and the block columns -- must equal the host's bit for bit. The coarsest
level's dense inverse is computed differently (device Gauss-Jordan against host LU), so
the time steps of the two setups agree to round-off of the converged solve, not bitwise.

Cases: the golden meshes (bilinear, curved, cylinder O-grids with Neumann outflow, the
backward-facing step), jittered cavities at K = 2..8, and a cavity large enough for the
smoothed-aggregation levels and the BF16 coarsest inverse.
"""

import os

import numpy as np
import pytest

from conftest import GOLDEN, GOLDEN_CASES

from ho2d import FP64, MIXED_KRYLOV, HO_2D, capi, meshgen

pytestmark = pytest.mark.gpu

ARRAYS = (capi.SETUP_DINV, capi.SETUP_ROWSUM, capi.SETUP_COLSUM, capi.SETUP_BSUM, capi.SETUP_BSRC, capi.SETUP_BCOL)


def _solver(inp, device, precision=FP64, smoother=-1):
    s = HO_2D()
    s.read_input_file(inp)
    s.set_precision(precision)
    s.set_smoother(smoother)
    s.set_device_setup(device)
    s.set_poisson_tolerance(1e-12, 2000)
    s.setup()
    return s


def _cases(tmp_path):
    out = [os.path.join(GOLDEN, c, "input.dat") for c in GOLDEN_CASES]
    for k in range(2, 9):
        out.append(meshgen.make_case("cavityj6", str(tmp_path / f"j6_{k}"), knod=k, steps=2))
    return out


def test_device_assembly_is_bitwise_the_host_assembly(tmp_path):
    for inp in _cases(tmp_path):
        dev, host = _solver(inp, True), _solver(inp, False)
        for which in ARRAYS:
            a, b = dev.get_poisson_setup(which), host.get_poisson_setup(which)
            assert a.shape == b.shape
            assert np.array_equal(a, b), (inp, which, float(np.max(np.abs(a - b))))
        dinv = dev.get_poisson_setup(capi.SETUP_DINV)
        assert np.all(np.isfinite(dinv)) and np.any(dinv != 0.0)
        dev.close()
        host.close()


def _steps(s, w0, n):
    s.set_vorticity(w0)
    s.solve_advection_diffusion(n)
    return s.get_vorticity(), s.get_streamfunction()


@pytest.mark.parametrize("precision", [FP64, MIXED_KRYLOV])
def test_device_setup_steps_match_host_setup(tmp_path, precision):
    # a 48 x 48 cavity coarsens below the dense size through smoothed aggregation, so the
    # device's dense inverse (and, for the FP32 preconditioner, its BF16 copy) is in use
    cases = [os.path.join(GOLDEN, "cyl4x8_rk4", "input.dat"),
             os.path.join(GOLDEN, "bfs2_rk4", "input.dat"),
             meshgen.make_case("cavityj48", str(tmp_path / "j48"), knod=4, steps=3)]
    for inp in cases:
        dev, host = _solver(inp, True, precision), _solver(inp, False, precision)
        rng = np.random.Generator(np.random.PCG64(3))
        w0 = rng.standard_normal((dev.N_el, dev.Knod, dev.Knod))
        wd, pd = _steps(dev, w0, 3)
        wh, ph = _steps(host, w0, 3)
        assert np.max(np.abs(pd - ph)) <= 1e-9 * np.max(np.abs(ph)), inp
        assert np.max(np.abs(wd - wh)) <= 1e-9 * np.max(np.abs(wh)), inp
        dev.close()
        host.close()


def test_device_setup_kron_fit_matches_host(tmp_path):
    """The Kronecker-sum fit runs on the downloaded device blocks: the same elements keep
    their exact block as under the host assembly, and the mixed-precision steps agree."""
    inp = meshgen.make_case("cavityj16", str(tmp_path / "j16"), knod=7, steps=2)
    dev = _solver(inp, True, MIXED_KRYLOV, capi.SMOOTHER_KRON)
    host = _solver(inp, False, MIXED_KRYLOV, capi.SMOOTHER_KRON)
    assert dev.smoother() == host.smoother()
    rng = np.random.Generator(np.random.PCG64(5))
    w0 = rng.standard_normal((dev.N_el, dev.Knod, dev.Knod))
    wd, pd = _steps(dev, w0, 2)
    wh, ph = _steps(host, w0, 2)
    assert np.max(np.abs(pd - ph)) <= 1e-9 * np.max(np.abs(ph))
    dev.close()
    host.close()
