"""The Strouhal estimator of ho2d.shedding on synthetic lift series (CPU).

A lift history of a cylinder wake starts with a transient and settles into a periodic
oscillation. The series here are seeded stand-ins: a growing then saturating sinusoid
of known frequency with a mean offset, a second harmonic and noise. Both estimates (zero
crossings and the spectral peak) must recover the frequency to 1e-3 relative, and the
initial vortex of the shedding case must be small on the cylinder.
"""

import numpy as np
import pytest

from ho2d.shedding import SheddingCase, strouhal, upward_crossings


def series(f, t_end=80.0, dt=0.02, noise=1e-3, seed=0, phase=0.3):
    rng = np.random.Generator(np.random.PCG64(seed))
    t = np.arange(1, int(t_end / dt) + 1) * dt
    env = 0.35 / (1.0 + np.exp(-(t - 25.0) / 3.0))  # growth, then saturation
    y = 0.01 + env * np.sin(2 * np.pi * f * t + phase) + 0.1 * env * np.sin(4 * np.pi * f * t)
    return t, y + noise * rng.standard_normal(t.shape)


def test_upward_crossings_of_a_sine():
    t = np.linspace(0.0, 3.0, 3001)
    c = upward_crossings(t, np.sin(2 * np.pi * t - 0.1))
    np.testing.assert_allclose(c, 0.1 / (2 * np.pi) + np.arange(3), atol=1e-6)
    # noise about zero: no extra crossings with hysteresis
    rng = np.random.Generator(np.random.PCG64(1))
    y = np.sin(2 * np.pi * t - 0.1) + 0.05 * rng.standard_normal(t.shape)
    assert len(upward_crossings(t, y)) > 3
    assert len(upward_crossings(t, y, h=0.25)) == 3


@pytest.mark.parametrize("f", [0.125, 0.1655, 0.21])
def test_strouhal_recovers_the_frequency(f):
    t, y = series(f, seed=int(f * 1e4))
    st = strouhal(t, y, periods=4)
    assert abs(st["St"] - f) <= 1e-3 * f, st
    assert abs(st["St_fft"] - f) <= 1e-3 * f, st
    assert st["period_spread"] < 0.01
    assert abs(st["amplitude"] - 0.35) < 0.05


def test_strouhal_scales_with_diameter_and_speed():
    t, y = series(0.2)
    a = strouhal(t, y)
    b = strouhal(t, y, D=2.0, U=4.0)
    assert abs(b["St"] - a["St"] * 0.5) < 1e-12


def test_too_few_periods_gives_nan():
    t = np.arange(0.0, 12.0, 0.02)
    st = strouhal(t, 0.3 * np.sin(2 * np.pi * 0.2 * t), periods=4)  # 2.4 periods
    assert np.isnan(st["St"]) and st["crossings"] < 5


def test_noise_is_flagged_by_the_period_spread():
    """Before shedding the lift is noise: the estimate must not look like a clean period."""
    rng = np.random.Generator(np.random.PCG64(3))
    t = np.arange(0.0, 80.0, 0.02)
    st = strouhal(t, 1e-6 * rng.standard_normal(t.shape))
    assert np.isnan(st["St"]) or st["period_spread"] > 0.2


def test_initial_vortex_is_small_on_the_cylinder():
    th = np.linspace(0, 2 * np.pi, 721)
    xy = 0.5 * np.stack([np.cos(th), np.sin(th)], -1)
    w = SheddingCase.initial_vorticity(xy, 0.5)
    assert w.max() < 1e-4
    # its circulation is gamma (integral over the plane)
    g = np.linspace(-4, 6, 801)
    X, Y = np.meshgrid(g, g)
    W = SheddingCase.initial_vorticity(np.stack([X, Y], -1), 0.5)
    assert abs(W.sum() * (g[1] - g[0]) ** 2 - 0.5) < 1e-6
