"""The FP32 preconditioner's smoother variants on the GPU, through the C ABI.

HO2D_SMOOTHER_BF16 stores the exact inverse blocks in BF16; HO2D_SMOOTHER_KRON replaces
them by Kronecker-sum factors (fast diagonalisation) and keeps the exact block only where
the fit is poor. Neither changes the converged answer: the FP32 solve sits inside FP64
refinement on the FP64 operator, so the mixed-precision run with either smoother agrees
with the FP64 run as closely as with the exact FP32 blocks. A layout or ordering mistake
in a smoother would only slow the inner solve, so the tests also bound the inner
iteration counts against the exact blocks'.
"""

import os

import numpy as np
import pytest

from conftest import GOLDEN

from ho2d import FP64, MIXED_KRYLOV, HO_2D, capi, meshgen

pytestmark = pytest.mark.gpu

TOL = 1e-9  # mixed Krylov vs FP64: Poisson round-off below its 1e-12 tolerance


def _solver(inp, precision, smoother=-1):
    s = HO_2D()
    s.read_input_file(inp)
    s.set_precision(precision)
    s.set_smoother(smoother)
    s.set_poisson_tolerance(1e-12, 2000)
    s.setup()
    return s


def _run(s, w0, steps):
    s.set_vorticity(w0)
    iters = []
    for _ in range(steps):
        s.solve_advection_diffusion(1)
        iters.append(s.poisson_stats()[0])
    return s.get_vorticity(), s.get_streamfunction(), iters


def _cases(tmp_path):
    # two golden meshes and a jittered K = 7 cavity on which the Kronecker fit falls back
    # to the exact block for some elements but not others in the same CTA (5 elements)
    return [
        (os.path.join(GOLDEN, "cav4_rk4", "input.dat"), 3),
        (os.path.join(GOLDEN, "cyl4x8_rk4", "input.dat"), 3),
        (meshgen.make_case("cavityj16", str(tmp_path / "j16"), knod=7, steps=3), 3),
    ]


@pytest.mark.parametrize("kind", [capi.SMOOTHER_BF16, capi.SMOOTHER_KRON])
def test_smoother_variant_matches_fp64(tmp_path, kind):
    for inp, steps in _cases(tmp_path):
        ref = _solver(inp, FP64)
        rng = np.random.Generator(np.random.PCG64(17))
        w0 = rng.standard_normal((ref.N_el, ref.Knod, ref.Knod))
        w64, p64, _ = _run(ref, w0, steps)
        base = _solver(inp, MIXED_KRYLOV, capi.SMOOTHER_BLOCKS)
        assert base.smoother() == (capi.SMOOTHER_BLOCKS, 0)
        _, _, it_base = _run(base, w0, steps)
        var = _solver(inp, MIXED_KRYLOV, kind)
        k, n_exact = var.smoother()
        assert k == kind
        if kind == capi.SMOOTHER_KRON and "j16" in inp:
            assert 0 < n_exact < var.N_el, n_exact  # both paths of the kernel run
        w, p, it_var = _run(var, w0, steps)
        assert np.linalg.norm(w - w64) <= TOL * np.linalg.norm(w64), inp
        assert np.linalg.norm(p - p64) <= TOL * np.linalg.norm(p64), inp
        assert var.poisson_stats()[1] < 1e-11
        assert sum(it_var) <= 1.5 * sum(it_base) + 6, (inp, it_var, it_base)


def test_smoother_choice_validated():
    s = HO_2D()
    with pytest.raises(capi.HO2DError):
        s.set_smoother(3)


@pytest.mark.parametrize("graphs", ["1", "0"])
def test_stalled_refinement_is_finished_in_fp64(tmp_path, monkeypatch, graphs):
    """A mixed solve whose refinement stops short of the tolerance (stalled, or at the sweep
    cap) is finished by the FP64 solve: with the cap at one sweep the first solves end short,
    the FP64 solve finishes them, and the steps still agree with the FP64 path at the
    Poisson tolerance."""
    monkeypatch.setenv("HO2D_MAX_SWEEPS", "1")
    monkeypatch.setenv("HO2D_GRAPHS", graphs)
    inp = os.path.join(GOLDEN, "cyl4x8_rk4", "input.dat")
    ref = _solver(inp, FP64)
    s = _solver(inp, MIXED_KRYLOV)
    rng = np.random.Generator(np.random.PCG64(23))
    w0 = rng.standard_normal((ref.N_el, ref.Knod, ref.Knod))
    w_ref, p_ref, _ = _run(ref, w0, 2)
    w, p, _ = _run(s, w0, 2)
    assert s.fp64_finishes() > 0
    assert np.max(np.abs(p - p_ref)) <= TOL * np.max(np.abs(p_ref))
    assert np.max(np.abs(w - w_ref)) <= TOL * np.max(np.abs(w_ref))


@pytest.mark.parametrize("knod", [3, 4, 5, 6, 7, 8])
def test_staged_operator_is_the_prefetch_operator(tmp_path, monkeypatch, knod):
    """The FP32 operator with its inputs staged by bulk copies (HO2D_OP_STAGE=1) computes
    what the default kernel computes from global memory (HO2D_OP_STAGE=0), bit for bit: the same
    arithmetic on the same values, in the same CTA order. A jittered 13 x 13 cavity gives a
    ragged last tile at every K, and odd K exercise the unaligned span starts."""
    inp = meshgen.make_case("cavityj13", str(tmp_path / "j13"), knod=knod, steps=2)
    rng = np.random.Generator(np.random.PCG64(29))
    out = {}
    for staged in ("1", "0"):
        monkeypatch.setenv("HO2D_OP_STAGE", staged)
        s = _solver(inp, MIXED_KRYLOV)
        w0 = rng.standard_normal((s.N_el, s.Knod, s.Knod)) if not out else out["w0"]
        out.setdefault("w0", w0)
        out[staged] = _run(s, w0, 2)
        s.close()
    (w1, p1, it1), (w0_, p0, it0) = out["1"], out["0"]
    assert it1 == it0
    assert np.array_equal(p1, p0)
    assert np.array_equal(w1, w0_)
