"""The synthetic workloads (ho2d.meshgen) against their stated recipes, on the CPU.

The benchmark and test meshes stand in for the reference's inputs: seeded synthetic
meshes of the stated shapes. These tests pin the shapes: element and boundary-edge counts,
counter-clockwise quads (the reader takes them without OCC reorientation), jitter on
interior nodes only and within its bound, seed determinism, the O-grid's radial growth,
and the differentiation case's initial vorticity (zero on the walls) and lid profile.
"""

import numpy as np
import pytest

from ho2d import meshgen


def signed_areas(m):
    p = m.xy[m.quads[:, :4]]
    x, y = p[..., 0], p[..., 1]
    return 0.5 * (x * np.roll(y, -1, axis=1) - np.roll(x, -1, axis=1) * y).sum(axis=1)


def boundary_nodes(m):
    return np.unique(np.concatenate([e.ravel() for e in m.boundaries.values()]))


def test_backward_facing_step_recipe():
    h = 1.0 / 15.0
    m = meshgen.backward_facing_step()
    assert m.n_el == 75 * 15 + 450 * 30 == 14625
    assert (signed_areas(m) > 0).all()
    assert {k: len(v) for k, v in m.boundaries.items()} == {"inlet": 15, "outlet": 30, "top": 75 + 450,
                                                             "bottom": 75 + 15 + 450}
    ref = meshgen.backward_facing_step(jitter=0.0)
    d = np.abs(m.xy - ref.xy)
    bn = boundary_nodes(m)
    assert d[bn].max() == 0.0  # boundary nodes stay on the walls
    assert 0.1 * h < d.max() <= 0.15 * h + 1e-15
    np.testing.assert_array_equal(m.xy, meshgen.backward_facing_step().xy)  # seed 2 is reproducible
    assert not np.array_equal(m.xy, meshgen.backward_facing_step(seed=3).xy)
    x, y = ref.xy[:, 0], ref.xy[:, 1]
    assert (x.min(), x.max(), y.min(), y.max()) == (-5.0, 30.0, -1.0, 1.0)
    assert not ((x < 0) & (y < 0)).any()  # no cells below the step upstream


def test_cylinder_ogrid_recipe():
    m = meshgen.cylinder_ogrid()
    assert m.n_el == 256 * 512
    assert (signed_areas(m) > 0).all()
    assert len(m.boundaries["object"]) == 512
    assert len(m.boundaries["inlet"]) + len(m.boundaries["outlet"]) == 512
    r = np.hypot(m.xy[:, 0], m.xy[:, 1])
    radii = np.unique(np.round(r, 9))
    assert len(radii) == 257
    np.testing.assert_allclose([radii[0], radii[-1]], [0.5, 20.0], rtol=1e-12)
    dr = np.diff(radii)
    np.testing.assert_allclose(dr[1:] / dr[:-1], 1.02, rtol=1e-6)
    np.testing.assert_allclose(dr[0], 19.5 * 0.02 / (1.02 ** 256 - 1), rtol=1e-6)
    mid = m.xy[m.boundaries["inlet"]].mean(axis=1)
    assert (mid[:, 0] < 0).all()
    assert (m.xy[m.boundaries["outlet"]].mean(axis=1)[:, 0] >= 0).all()


@pytest.mark.parametrize("n,jitter", [(16, 0.0), (64, 0.0), (24, 0.1)])
def test_cavity_recipe(n, jitter):
    m = meshgen.cavity(n, jitter=jitter, seed=5)
    assert m.n_el == n * n
    assert (signed_areas(m) > 0).all()
    assert list(m.boundaries) == ["bottom_wall", "right_wall", "top", "left_wall"]
    assert all(len(e) == n for e in m.boundaries.values())
    ref = meshgen.cavity(n)
    d = np.abs(m.xy - ref.xy).max(axis=1)
    assert d[boundary_nodes(m)].max() == 0.0
    assert d.max() <= jitter / n + 1e-15


def test_differentiation_case_fields():
    """Config 4: omega0 = sum c_mn sin(m pi x) sin(n pi y), c_mn ~ N(0,1)/(m^2+n^2), zero on
    the walls; lid u(x) = 1 + sum a_m sin(m pi x), a_m ~ N(0, 0.05); both seeded."""
    t = np.linspace(0.0, 1.0, 101)
    walls = np.concatenate([np.stack([t, 0 * t], -1), np.stack([t, 0 * t + 1], -1), np.stack([0 * t, t], -1),
                            np.stack([0 * t + 1, t], -1)])
    w = meshgen.sine_spectrum(walls, seed=4)
    assert np.abs(w).max() < 1e-12
    g = np.stack(np.meshgrid(t, t), -1)
    inside = meshgen.sine_spectrum(g, seed=4)
    assert np.abs(inside).max() > 0.1
    np.testing.assert_array_equal(inside, meshgen.sine_spectrum(g, seed=4))
    assert not np.array_equal(inside, meshgen.sine_spectrum(g, seed=42))
    a = meshgen.lid_coefficients(seed=41)
    assert a.shape == (4,) and np.abs(a).max() < 0.25
    u = meshgen.lid_velocity(t, a)
    np.testing.assert_allclose(u[[0, -1]], 1.0, atol=1e-12)  # corners keep u = 1


@pytest.mark.parametrize("name", ["cfg1_cavity16", "cfg2_bfs"])
def test_config_goldens_match_generated_inputs(tmp_path, name):
    """The benchmark configurations' golden vectors were made by the reference from the
    input.dat and mesh.msh that meshgen writes now, byte for byte (the GPU parity tests
    regenerate them instead of storing the meshes)."""
    import json
    import os
    import sys

    from conftest import GOLDEN

    meta_path = os.path.join(GOLDEN, name, "meta.json")
    if not os.path.exists(meta_path):
        pytest.skip(f"{name} golden not generated")
    sys.path.insert(0, GOLDEN)
    import make_config_golden as CG

    meta = json.load(open(meta_path))
    inp = CG.write_case(name, str(tmp_path))
    assert CG.sha256(inp) == meta["input_sha256"]
    assert CG.sha256(os.path.join(os.path.dirname(inp), "mesh.msh")) == meta["mesh_sha256"]


def test_cylinder_channel_mesh():
    """The channel O-grid of the shedding case: counter-clockwise cells, every outer edge on
    one side of the channel (corners on nodes), the cylinder resolved as in the O-grid."""
    m = meshgen.cylinder_channel(48, 96, r0=0.5, x_in=-15.0, x_out=45.0, half_h=15.0, stretch=1.04)
    xy = m.xy[m.quads]
    area = 0.5 * sum(xy[:, k, 0] * xy[:, (k + 1) % 4, 1] - xy[:, (k + 1) % 4, 0] * xy[:, k, 1] for k in range(4))
    assert area.min() > 0.0
    outer = sum(len(m.boundaries[k]) for k in ("inlet", "outlet", "top", "bottom"))
    assert outer == 96 and len(m.boundaries["object"]) == 96
    x_out = m.xy[m.boundaries["outlet"].ravel(), 0]
    assert np.allclose(m.xy[m.boundaries["inlet"].ravel(), 0], -15.0) and np.allclose(x_out, x_out[0])
    assert 40.0 < x_out[0] < 50.0
    assert np.allclose(m.xy[m.boundaries["top"].ravel(), 1], 15.0)
    assert np.allclose(m.xy[m.boundaries["bottom"].ravel(), 1], -15.0)
    r = np.hypot(m.xy[m.boundaries["object"].ravel(), 0], m.xy[m.boundaries["object"].ravel(), 1])
    assert np.allclose(r, 0.5)
