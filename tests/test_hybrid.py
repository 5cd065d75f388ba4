"""Hybrid operation (problem type 11): the entry points an external Lagrangian driver
calls (src/HO_2D.hpp:251-290), against the reference's own hybrid run.

tests/golden/make_hybrid_golden.py drove the reference (oracle/_ref/ho2d_ref --hybrid)
with the arrays in tests/golden/hybrid/<case>/ and kept its results in hybrid_ref.npz.
The GPU tests drive the library through the same sequence and compare: vorticity after
each outer solveto step (1e-9 relative; the Poisson solves at 1e-14), solution-point
areas and open-boundary points (1e-13). The CPU tests cover argument checking of the
host-side loaders.
"""

import os

import numpy as np
import pytest

from conftest import GOLDEN

from ho2d import HO_2D, HO2DError

HYB = os.path.join(GOLDEN, "hybrid")
CASES = sorted(d for d in os.listdir(HYB) if os.path.isfile(os.path.join(HYB, d, "hybrid_ref.npz")))


def load_case(name):
    d = os.path.join(HYB, name)
    spec = {}
    for line in open(os.path.join(d, "spec.txt")):
        k, v = line.split()
        spec[k] = float(v)
    arrays = {f[:-4]: np.load(os.path.join(d, f)) for f in os.listdir(d) if f.endswith(".npy")}
    return spec, arrays, dict(np.load(os.path.join(d, "hybrid_ref.npz")))


def run_hybrid(spec, a):
    """The driver sequence of oracle/ref_harness.cpp run_hybrid, through the C ABI."""
    empty_i, empty_d = np.zeros(0, np.int32), np.zeros(0)
    s = HO_2D()
    s.set_defaults()
    s.enable_hybrid()
    s.set_elemorder(int(spec["knod"]))
    s.set_poisson_tolerance(1e-14, 2000)
    s.load_mesh_arrays_d(int(spec["iorder"]), a["nodes"], a["elems"], a.get("wall", empty_i), a.get("open", empty_i))
    s.load_inout_arrays_d(a.get("inletvel", empty_d), a.get("inlet", empty_i), a.get("outletvel", empty_d),
                          a.get("outlet", empty_i))
    s.process_mesh_input()
    if "ptog" in a:
        s.setptogweights_d(a["ptog"])
    out = {}
    for st in range(-1, int(spec["nouter"])):
        if f"vort_{st}" in a:
            s.setsolnvort_d(a[f"vort_{st}"])
        if f"openvel_{st}" in a:
            s.setopenvels_d(a[f"openvel_{st}"])
        if f"openvort_{st}" in a:
            s.setopenvort_d(a[f"openvort_{st}"])
        if st < 0:
            continue
        s.solveto_d(spec["outerdt"], int(spec["numstep"]), int(spec["integ"]), spec["reyn"])
        out[f"vort_out_{st}"] = s.getallvorts_d().ravel()
    out["areas"] = s.getsolnareas_d().ravel()
    if s.getopenptlen():
        out["openpts"] = s.getopenpts_d().ravel()
    return s, out


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
def test_hybrid_run_matches_reference(name):
    spec, a, ref = load_case(name)
    s, out = run_hybrid(spec, a)
    assert set(out) == set(ref)
    for k, r in ref.items():
        tol = 1e-9 if k.startswith("vort_out") else 1e-13
        err = np.abs(out[k] - r).max() / max(np.abs(r).max(), 1e-300)
        assert err <= tol, (k, err)
    w = s.get_hoquad_weights_d()
    np.testing.assert_allclose(w.sum(), 1.0, rtol=1e-14)
    s.clean_up()
    with pytest.raises(HO2DError):
        s.getallvorts_d()


def test_hybrid_loaders_check_their_arguments():
    s = HO_2D()
    s.set_defaults()
    s.enable_hybrid()
    with pytest.raises(HO2DError) as e:
        s.set_elemorder(9)
    assert e.value.code == 4
    s.set_elemorder(3)
    xy = np.array([0, 0, 1, 0, 1, 1, 0, 1], float)
    with pytest.raises(HO2DError) as e:  # 3 indices: not a multiple of Lnod^2 = 4
        s.load_mesh_arrays_d(1, xy, [0, 1, 2])
    assert e.value.code == 1
    with pytest.raises(HO2DError) as e:  # node 7 does not exist
        s.load_mesh_arrays_d(1, xy, [0, 1, 2, 7])
    assert e.value.code == 3
    with pytest.raises(HO2DError) as e:  # geometry order 4 (Lnod 5) is not supported
        s.load_mesh_arrays_d(4, xy, [0, 1, 2, 3])
    assert e.value.code == 4
    s.load_mesh_arrays_d(1, xy, [0, 1, 2, 3], wall=[0, 1, 1, 2, 2, 3, 3, 0])
    with pytest.raises(HO2DError) as e:  # 3 values over 1 inlet edge
        s.load_inout_arrays_d([1.0, 2.0, 3.0], [0, 1])
    assert e.value.code == 1
