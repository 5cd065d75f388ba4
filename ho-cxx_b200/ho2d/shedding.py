"""Vortex shedding behind the cylinder (problem type 3): the lift time series and its
Strouhal number.

Problem type 3 (src/HO_2D.cpp:819-906) is a cylinder of diameter D = 1 (the "object"
boundary at r = 0.5) in a channel: the stream enters through the straight inlet (psi =
U (y - y_min), normal velocity U), the top and bottom move with it, and the outlet is a
Neumann boundary. The reference's inflow is pulsatile, U(t) = 2 |sin(pi t / 40)|
(update_BCs, src/HO_2D.cpp:1979-2217; ``inflow_speed``), so it peaks at U = 2 (Re = 200 on
the peak speed) at t = 20. The force on the cylinder comes from ``HO_2D.forces()`` (FP64,
density 1; no counterpart in the reference); the drag and lift coefficients use the
instantaneous inflow speed, C = 2 F / (U(t)^2 D), and the Strouhal number St = f D / U uses
the lift frequency f and the mean inflow speed over the analysed window. The default run
ends at t = 30, so its last three shedding periods lie around and after the inflow peak.

The case: an O-grid of ``n_r`` x ``n_theta`` cells from the cylinder at r = 0.5 out to the
channel [-r1, 3 r1] x [-r1, r1] (radial spacing growing by ``stretch``, the rings blending
from circles into the channel's rectangle), K = ``knod``, Re = 100 (on U = 1). The step is
the smaller of the CFL-0.5 step for |u| <= 2 and the viscous bound of explicit RK4
(meshgen.cfl_dt, meshgen.viscous_dt). A symmetric start sheds only after round-off grows,
so the initial vorticity is a Gaussian vortex of circulation ``gamma`` centred off the axis
behind the cylinder (below 1e-4 on the cylinder). All fields are synthetic: no dataset is
involved.

St from a lift series: the upward zero crossings of lift - mean (the mean over the analysed
window) located by linear interpolation, with a hysteresis of a quarter of the half
peak-to-peak so that noise adds none; f = periods / (time between the first and the last
of the last ``periods`` + 1 crossings). Cross-check: the peak of the Hann-windowed spectrum
of the same window, refined by a parabola through the log magnitudes at the peak bin and
its two neighbours.
"""

from __future__ import annotations

import os
import time

import numpy as np

from . import FP64, MIXED, HO_2D, meshgen


def inflow_speed(t):
    """Problem type 3's inflow speed at time t: 2 |sin(pi t / 40)| (the reference's
    time-dependent inlet and channel walls, src/HO_2D.cpp:1979-2217)."""
    return 2.0 * np.abs(np.sin(np.pi / 40.0 * np.asarray(t, dtype=float)))


def upward_crossings(t: np.ndarray, y: np.ndarray, h: float = 0.0) -> np.ndarray:
    """Times where y goes from < 0 to >= 0, by linear interpolation between samples. With
    h > 0 a crossing counts only if y has been below -h since the last counted one, so
    that noise around zero adds no crossings."""
    t = np.asarray(t, dtype=float)
    y = np.asarray(y, dtype=float)
    i = np.flatnonzero((y[:-1] < 0.0) & (y[1:] >= 0.0))
    if h > 0.0 and len(i):
        below = np.flatnonzero(y < -h)
        keep, last = [], -1
        for k in i:  # armed when some sample after the last counted crossing is below -h
            j = np.searchsorted(below, last + 1)
            if j < len(below) and below[j] <= k:
                keep.append(k)
                last = k
        i = np.array(keep, dtype=int)
    return t[i] - y[i] * (t[i + 1] - t[i]) / (y[i + 1] - y[i])


def strouhal(t, lift, D: float = 1.0, U: float = 1.0, periods: int = 4) -> dict:
    """Strouhal number f D / U of the lift series (t ascending, uniform or not) from its
    last ``periods`` periods. Returns St (zero crossings), St_fft (spectral peak, uniform
    sampling assumed), the spread (max - min) / mean of the individual periods, the lift
    amplitude (half the peak-to-peak over the window) and the window [t0, t1]. St is NaN
    when fewer than periods + 1 upward crossings exist."""
    t = np.asarray(t, dtype=float)
    y = np.asarray(lift, dtype=float)
    out = {"St": float("nan"), "St_fft": float("nan"), "period_spread": float("nan"), "amplitude": float("nan"),
           "window": [float("nan"), float("nan")], "crossings": 0}
    # two passes: crossings of the signal about the mean of the second half, then about the
    # mean over the whole periods found; hysteresis a quarter of the half peak-to-peak
    half = y[len(y) // 2:]
    h = 0.125 * (half.max() - half.min()) if len(half) else 0.0
    c = upward_crossings(t, y - half.mean(), h)
    if len(c) < periods + 1:
        out["crossings"] = int(len(c))
        return out
    w = (t >= c[-periods - 1]) & (t <= c[-1])
    c = upward_crossings(t, y - y[w].mean(), h)
    out["crossings"] = int(len(c))
    if len(c) < periods + 1:
        return out
    c = c[-periods - 1:]
    per = np.diff(c)
    f = periods / (c[-1] - c[0])
    w = (t >= c[0]) & (t <= c[-1])
    out.update(St=float(f * D / U), period_spread=float((per.max() - per.min()) / per.mean()),
               amplitude=float(0.5 * (y[w].max() - y[w].min())), window=[float(c[0]), float(c[-1])])
    ts, ys = t[w], y[w] - y[w].mean()
    if len(ts) >= 16:
        dt = (ts[-1] - ts[0]) / (len(ts) - 1)
        n = 1 << int(np.ceil(np.log2(len(ts)))) + 3  # zero padding: finer bins
        spec = np.abs(np.fft.rfft(ys * np.hanning(len(ys)), n))
        k = int(np.argmax(spec[1:])) + 1
        if 1 <= k < len(spec) - 1:
            a, b, g = np.log(spec[k - 1:k + 2] + 1e-300)
            k = k + 0.5 * (a - g) / (a - 2 * b + g)
        out["St_fft"] = float(k / (n * dt) * D / U)
    return out


class SheddingCase:
    def __init__(self, workdir: str, n_r: int = 48, n_theta: int = 96, r1: float = 15.0, stretch: float = 1.04,
                 knod: int = 4, reyn: float = 100.0, gamma: float = 1.5, precision: int = FP64, tol: float = 1e-10,
                 max_iter: int = 500):
        os.makedirs(workdir, exist_ok=True)
        # the channel [-r1, 3 r1] x [-r1, r1] around the cylinder: problem type 3's straight
        # inlet (uniform inflow normal to it), top and bottom moving with the free stream, and
        # the outlet 3 r1 downstream, where the shed vortices have spread
        mesh = meshgen.cylinder_channel(n_r, n_theta, r0=0.5, x_in=-r1, x_out=3.0 * r1, half_h=r1, stretch=stretch)
        self.dt = min(meshgen.cfl_dt(mesh, knod, 2.0), meshgen.viscous_dt(mesh, knod, reyn))
        meshgen.write_msh(mesh, os.path.join(workdir, "mesh.msh"))
        self.inp = os.path.join(workdir, "input.dat")
        meshgen.write_input_dat(self.inp, "mesh.msh", knod, reyn, self.dt, 1, 3)
        self.n_el, self.knod, self.reyn, self.gamma = mesh.n_el, knod, reyn, gamma
        self.s = HO_2D()
        self.s.read_input_file(self.inp)
        self.s.set_precision(precision)
        self.s.set_poisson_tolerance(tol, max_iter)
        self.s.setup()
        self.w0 = self.initial_vorticity(self.s.getsolnpts_d(), gamma)

    @staticmethod
    def initial_vorticity(xy: np.ndarray, gamma: float, center=(1.5, 0.35), radius: float = 0.3) -> np.ndarray:
        """A Gaussian vortex of circulation gamma at ``center`` (behind the cylinder, off the
        axis): omega = gamma / (pi r^2) exp(-|x - c|^2 / r^2)."""
        d2 = (xy[..., 0] - center[0]) ** 2 + (xy[..., 1] - center[1]) ** 2
        return gamma / (np.pi * radius ** 2) * np.exp(-d2 / radius ** 2)

    def run(self, t_end: float, sample_dt: float = 0.02) -> dict:
        """Advance from the initial vorticity to t_end, sampling (drag, lift) every
        ~sample_dt; returns the series, St and wall time."""
        s = self.s
        s.set_time(0.0)
        s.setsolnvort_d(self.w0)
        every = max(1, int(round(sample_dt / self.dt)))
        nsamp = int(np.ceil(t_end / (every * self.dt)))
        t = np.zeros(nsamp)
        fx = np.zeros(nsamp)
        fy = np.zeros(nsamp)
        t0 = time.perf_counter()
        for i in range(nsamp):
            s.solve_advection_diffusion(every)
            t[i] = s.time()[0]
            fx[i], fy[i] = s.forces()
        wall = time.perf_counter() - t0
        # coefficients on the instantaneous inflow speed (D = 1, density 1)
        u2 = np.maximum(inflow_speed(t), 0.05) ** 2
        cd, cl = 2.0 * fx / u2, 2.0 * fy / u2
        # crossings of the lift force itself (the frequency needs no scale); three periods, as
        # the pulsatile inflow leaves about that many near its peak
        st = strouhal(t, fy, periods=3)
        w = (t >= st["window"][0]) & (t <= st["window"][1]) if np.isfinite(st["St"]) else t >= 0.5 * t[-1]
        u_mean = float(inflow_speed(t[w]).mean())
        for key in ("St", "St_fft"):
            st[key] = st[key] / u_mean if np.isfinite(st[key]) else st[key]
        return {"t": t, "cd": cd, "cl": cl, "St": st, "u_mean": u_mean, "cd_mean": float(cd[w].mean()),
                "cl_amplitude": float(0.5 * (cl[w].max() - cl[w].min())), "steps": int(nsamp * every),
                "wall_s": wall}


def run(workdir: str, t_end: float = 30.0, **kw) -> dict:
    """St, mean drag and lift amplitude in FP64 and with the FP32 Krylov
    (HO2D_MIXED: FP32 stage kernels and FP32 BiCGSTAB inside FP64 refinement) on the same
    case, and their differences."""
    out = {}
    for name, prec in (("fp64", FP64), ("mixed", MIXED)):
        c = SheddingCase(os.path.join(workdir, name), precision=prec, **kw)
        r = run_case(c, t_end)
        out[name] = r
        out.setdefault("case", {"n_el": c.n_el, "knod": c.knod, "dof": c.n_el * c.knod ** 2, "reyn": c.reyn,
                                "dt": c.dt, "t_end": t_end, "gamma": c.gamma})
    a, b = out["fp64"], out["mixed"]
    out["difference"] = {"St": abs(b["St"] - a["St"]), "cd_mean": abs(b["cd_mean"] - a["cd_mean"]),
                         "cl_amplitude": abs(b["cl_amplitude"] - a["cl_amplitude"])}
    return out


def run_case(c: SheddingCase, t_end: float) -> dict:
    r = c.run(t_end)
    st = r["St"]
    k = max(1, len(r["t"]) // 240)  # about 240 samples of the series
    return {"St": st["St"], "St_fft": st["St_fft"], "period_spread": st["period_spread"], "window": st["window"],
            "u_mean": r["u_mean"], "cd_mean": r["cd_mean"], "cl_amplitude": r["cl_amplitude"], "steps": r["steps"],
            "wall_s": r["wall_s"],
            "ms_per_step": 1e3 * r["wall_s"] / max(1, r["steps"]),
            "series": {"t": [round(float(x), 4) for x in r["t"][::k]], "cd": [float(x) for x in r["cd"][::k]],
                       "cl": [float(x) for x in r["cl"][::k]]}}
