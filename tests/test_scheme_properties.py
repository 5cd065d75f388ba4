"""Properties of the FR discretisation that hold exactly, whatever the reference values.

Conservation of the advective term: the FR divergence integrates (weights w_i w_j, times
J) to the common normal fluxes on the element's faces; the common flux of an interior face
is the same from both sides (both advection schemes), so over the mesh
    sum_points w_i w_j J RHS_adv = - sum_boundary_edges s sum_m w_m BC_advection,
s = +1 on E/N faces and -1 on W/S faces (BC_advection is the flux in the element's local
coordinate direction). CPU: the oracle (pinned to the reference's golden vectors). GPU: the
library's stage through the C ABI (solution-point areas from getsolnareas_d).
"""

import os

import numpy as np
import pytest

from conftest import GOLDEN, GOLDEN_CASES

import ho2d_oracle as O


def boundary_sign(case):
    ijp = np.array([O.F2I[s] for s in case.mesh.be_side])
    return np.where(ijp % 2 == 1, 1.0, -1.0)


def conservation_defect(rhs_adv, areas, bc_adv, sign, w):
    total = float((rhs_adv * areas).sum())
    bflux = -float((sign[:, None] * bc_adv * w[None, :]).sum())
    scale = float(np.abs(rhs_adv * areas).sum()) + 1e-300
    return abs(total - bflux) / scale


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_advection_is_conservative_oracle(name):
    c = O.Case(os.path.join(GOLDEN, name, "input.dat"))
    c.omega = np.random.default_rng(3).standard_normal((c.N, c.K, c.K))
    c.t = 0.0
    c.stage(c.omega, 0.0)
    areas = np.outer(c.B.w, c.B.w)[None] * c.M["J"]
    assert conservation_defect(c.rhs_adv, areas, c.bc_adv, boundary_sign(c), c.B.w) < 1e-13


@pytest.mark.gpu
@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_advection_is_conservative_device(name):
    from ho2d import HO_2D, capi

    inp = os.path.join(GOLDEN, name, "input.dat")
    c = O.Case(inp)
    s = HO_2D()
    s.read_input_file(inp)
    s.set_poisson_tolerance(1e-14, 2000)
    s.setup()
    s.set_vorticity(np.random.default_rng(3).standard_normal((s.N_el, s.Knod, s.Knod)))
    s.Euler_time_integrate(0.0)
    rhs_adv = s.get_field(capi.FIELD_RHS_ADVECTIVE)
    bc_adv = s.get_boundary(capi.BC_ADVECTION)
    areas = s.getsolnareas_d().reshape(rhs_adv.shape)
    assert conservation_defect(rhs_adv, areas, bc_adv, boundary_sign(c), c.B.w) < 1e-10
