"""The differentiation case: gradient of a final-time vorticity misfit by the discrete
adjoint, checked against central finite differences on the device.

Lid-driven cavity, n x n uniform quads (default 64 x 64), K = 5, Re = 1000, RK4. The
initial vorticity is the seeded sine spectrum of ``meshgen.sine_spectrum`` (seed 4); the
lid is u(x) = 1 + sum_{m=1..4} a_m sin(m pi x) with a_m ~ N(0, 0.05) (seed 41);
J = 0.5 ||omega(T) - omega_target||^2 with omega_target = omega(T) of a run from the
seed-42 spectrum under the same lid. The gradient with respect to (omega0, a) comes from
the adjoint (checkpoints every ``ckpt`` steps); it is checked along ``ndir`` seeded
directions (seed 43) against (J(x + h d) - J(x - h d)) / 2h of the FP64 forward. All
fields are synthetic: no dataset is involved.
"""

from __future__ import annotations

import time

import numpy as np

from . import FP64, MIXED_KRYLOV, HO_2D, capi, meshgen


def cavity_dt(n: int, knod: int, u_max: float = 1.2, cfl: float = 0.5, reyn: float = 1000.0,
              jitter: float = 0.0) -> float:
    """The smaller of the CFL-0.5 step cfl h / (u_max K^2), h = 1/n, and the viscous bound
    of explicit RK4 on the FR Laplacian 1.5 h_min^2 Re / K^4 (meshgen.viscous_dt), with
    h_min = (1 - 2 jitter) / n the smallest edge a +/-jitter*h perturbation can leave."""
    h_min = (1.0 - 2.0 * jitter) / n
    return min(cfl * (1.0 / n) / (u_max * knod * knod), 1.5 * h_min * h_min * reyn / knod ** 4)


class DifferentiationCase:
    def __init__(self, workdir: str, n: int = 64, knod: int = 5, reyn: float = 1000.0, steps: int = 500,
                 tol: float = 1e-13, max_iter: int = 2000, jitter: float = 0.0, w0_seed: int = 4,
                 precision: int = FP64):
        self.n, self.knod, self.reyn, self.steps = n, knod, reyn, steps
        self.dt = cavity_dt(n, knod, reyn=reyn, jitter=jitter)
        name = f"cavityj{n}" if jitter > 0 else f"cavity{n}"
        self.inp = meshgen.make_case(name, workdir, knod=knod, steps=steps, dt=self.dt, reyn=reyn, jitter=jitter,
                                     seed=5)
        self.tol, self.max_iter = tol, max_iter
        self.s = self.solver(precision)
        s = self.s
        xy = s.getsolnpts_d()
        bp = s.get_boundary_points()
        self.top = s.get_boundary(capi.BC_PARL_VEL) == -1.0  # BC_parl_vel = -1 on the lid (problem type 1)
        self.bx = bp[..., 0]
        self.w0 = meshgen.sine_spectrum(xy, seed=w0_seed)
        self.a = meshgen.lid_coefficients(seed=41)
        m = np.arange(1, len(self.a) + 1)
        # d BC_parl_vel / d a_m on the lid (BC_parl_vel = -u there)
        self.dpv_da = np.where(self.top[..., None], -np.sin(np.pi * self.bx[..., None] * m), 0.0)
        self.target = self.run(s, meshgen.sine_spectrum(xy, seed=42), self.a)

    def solver(self, precision: int) -> HO_2D:
        s = HO_2D()
        s.read_input_file(self.inp)
        s.set_precision(precision)
        s.set_poisson_tolerance(self.tol, self.max_iter)
        s.setup()
        return s

    def pv(self, a) -> np.ndarray:
        return np.where(self.top, -meshgen.lid_velocity(self.bx, a), 0.0)

    def _start(self, s: HO_2D, w0, a) -> None:
        s.set_time(0.0)
        s.set_boundary(capi.BC_PARL_VEL, self.pv(a))
        s.setsolnvort_d(w0)

    def run(self, s: HO_2D, w0, a) -> np.ndarray:
        self._start(s, w0, a)
        s.solve_advection_diffusion(self.steps)
        return s.getallvorts_d()

    def J(self, w0, a) -> float:
        return 0.5 * float(np.sum((self.run(self.s, w0, a) - self.target) ** 2))

    def gradient(self, precision: int, ckpt: int, fp32_state: bool = False, solver: HO_2D | None = None) -> dict:
        """Adjoint gradient (dJ/d omega0, dJ/d a) and the wall time of its two sweeps."""
        s = solver if solver is not None else (self.s if precision == FP64 else self.solver(precision))
        s.set_adjoint_storage(fp32_state)
        self._start(s, self.w0, self.a)
        l0 = s.launch_count()
        t0 = time.perf_counter()
        s.adjoint_forward(self.steps, ckpt)
        t1 = time.perf_counter()
        wT = s.getallvorts_d()
        gw, gpv = s.adjoint_backward(wT - self.target)
        t2 = time.perf_counter()
        it, res = s.adjoint_stats()
        ga = np.einsum("ekm,ek->m", self.dpv_da, gpv)
        return dict(gw=gw, ga=ga, J=0.5 * float(np.sum((wT - self.target) ** 2)), forward_s=t1 - t0,
                    backward_s=t2 - t1, launches=s.launch_count() - l0, last_transposed_iterations=it,
                    last_transposed_residual=res)

    def directions(self, ndir: int, seed: int = 43):
        rng = np.random.Generator(np.random.PCG64(seed))
        return [(rng.standard_normal(self.w0.shape), rng.standard_normal(self.a.shape)) for _ in range(ndir)]

    def finite_differences(self, dirs, h: float = 1e-6):
        out = []
        for dw, da in dirs:
            jp = self.J(self.w0 + h * dw, self.a + h * da)
            jm = self.J(self.w0 - h * dw, self.a - h * da)
            out.append((jp - jm) / (2.0 * h))
        return np.array(out)

    @staticmethod
    def directional(g: dict, dirs) -> np.ndarray:
        return np.array([float(np.vdot(g["gw"], dw) + np.vdot(g["ga"], da)) for dw, da in dirs])

    def state_bytes(self, ckpt: int) -> int:
        """Device bytes the adjoint keeps for the time loop: FP64 checkpoints and one
        segment of RK4 stage inputs and streamfunctions."""
        nv = self.s.N_el * self.knod ** 2
        nck = (self.steps + ckpt - 1) // ckpt
        return 8 * nv * (nck + 2 * ckpt * 4)


def run(workdir: str, n: int = 64, knod: int = 5, steps: int = 500, ckpt: int = 25, ndir: int = 20,
        h: float = 1e-6) -> dict:
    """FP64 and mixed-precision adjoint gradients of the case against FP64 central
    differences; returns the errors and timings."""
    c = DifferentiationCase(workdir, n=n, knod=knod, steps=steps)
    dirs = c.directions(ndir)
    t0 = time.perf_counter()
    fd = c.finite_differences(dirs, h)
    fd_s = time.perf_counter() - t0
    out = {"n_el": c.s.N_el, "dof": c.s.N_el * knod * knod, "dt": c.dt, "steps": steps, "ckpt_every": ckpt,
           "directions": ndir, "h": h, "fd_seconds": fd_s, "adjoint_state_bytes": c.state_bytes(ckpt)}
    for name, prec in (("fp64", FP64), ("mixed", MIXED_KRYLOV)):
        g = c.gradient(prec, ckpt)
        ad = c.directional(g, dirs)
        err = np.abs(ad - fd) / np.maximum(np.abs(fd), 1e-300)
        out[name] = {"max_rel_error": float(err.max()), "median_rel_error": float(np.median(err)),
                     "J": g["J"], "forward_s": g["forward_s"], "backward_s": g["backward_s"],
                     "launches": g["launches"], "last_transposed_iterations": g["last_transposed_iterations"],
                     "grad_lid": [float(x) for x in g["ga"]]}
    return out


def device_memory_used() -> float | None:
    """Bytes in use on the current device (all allocations of this process), or None."""
    try:
        import torch

        free, total = torch.cuda.mem_get_info()
        return float(total - free)
    except Exception:
        return None


def host_memory_available() -> float:
    for line in open("/proc/meminfo"):
        if line.startswith("MemAvailable:"):
            return float(line.split()[1]) * 1024.0
    return 0.0


def run_large(workdir: str, n: int = 512, knod: int = 7, steps: int = 200, ckpt: int = 20, coarse: int = 4,
              host_bytes_needed: float = 24e9) -> dict:
    """The combined large case: jittered cavity n x n (+/-0.1h, seed 5), K = 7, Re = 5000,
    omega0 from the seeded spectrum (seed 3), lid and target as in the differentiation
    case. (1) On the n/coarse mesh: the mixed-precision adjoint with FP32 state storage
    against the FP64 adjoint with FP64 states (relative L2 difference of both gradients).
    (2) On the full mesh: mixed forward + adjoint sweep, FP32 states, checkpoints every
    `ckpt` steps: wall times and device memory. The full mesh is skipped (and the reason
    reported) when the host has too little free memory for its setup: the inverse diagonal
    Poisson blocks (K^4 FP64 values per element, briefly twice), their FP32 copy and the
    metrics, about 15 GB at n = 512, K = 7."""
    import os

    out = {"n": n, "knod": knod, "steps": steps, "ckpt_every": ckpt}
    nc = n // coarse
    cdir = os.path.join(workdir, "coarse")
    c = DifferentiationCase(cdir, n=nc, knod=knod, reyn=5000.0, steps=steps, tol=1e-12, max_iter=500, jitter=0.1,
                            w0_seed=3)
    g64 = c.gradient(FP64, ckpt, fp32_state=False)
    g32 = c.gradient(MIXED_KRYLOV, ckpt, fp32_state=True)
    out["coarse"] = {"n": nc, "dof": c.s.N_el * knod * knod, "dt": c.dt,
                     "omega0_grad_rel_l2": float(np.linalg.norm(g32["gw"] - g64["gw"]) / np.linalg.norm(g64["gw"])),
                     "lid_grad_rel_l2": float(np.linalg.norm(g32["ga"] - g64["ga"]) / np.linalg.norm(g64["ga"])),
                     "fp64": {k: g64[k] for k in ("J", "forward_s", "backward_s")},
                     "mixed_fp32_state": {k: g32[k] for k in ("J", "forward_s", "backward_s")}}
    import json
    import sys

    print(json.dumps({"coarse": out["coarse"]}), file=sys.stderr, flush=True)
    avail = host_memory_available()
    out["host_memory_available"] = avail
    if avail < host_bytes_needed:
        out["full"] = {"skipped": f"host memory available {avail / 1e9:.0f} GB < {host_bytes_needed / 1e9:.0f} GB "
                                  f"needed for the host setup"}
        return out
    fdir = os.path.join(workdir, "full")
    t0 = time.perf_counter()
    f = DifferentiationCase(fdir, n=n, knod=knod, reyn=5000.0, steps=steps, tol=1e-12, max_iter=500, jitter=0.1,
                            w0_seed=3, precision=MIXED_KRYLOV)
    setup_s = time.perf_counter() - t0
    m0 = device_memory_used()
    g = f.gradient(MIXED_KRYLOV, ckpt, fp32_state=True, solver=f.s)
    m1 = device_memory_used()
    out["full"] = {"n_el": f.s.N_el, "dof": f.s.N_el * knod * knod, "dt": f.dt, "setup_and_target_s": setup_s,
                   "forward_s": g["forward_s"], "backward_s": g["backward_s"], "J": g["J"],
                   "grad_lid": [float(x) for x in g["ga"]], "omega0_grad_norm": float(np.linalg.norm(g["gw"])),
                   "device_bytes_before_adjoint": m0, "device_bytes_after_adjoint": m1,
                   "adjoint_state_bytes_fp32": f.state_bytes(ckpt) // 2,
                   "last_transposed_iterations": g["last_transposed_iterations"]}
    return out
