"""Benchmark: DOF-updates/s and Poisson ms/step of the FR time step on one B200.

Headline workload (default): flow around a cylinder on a 256 x 512 O-grid (radial stretch
1.02, r in [0.5, 20]; 131,072 quads), K = P+1 = 6 (4,718,592 DOF), Re = 100, RK4 at the
smaller of the CFL-0.5 and the viscous step, impulsive start -- a seeded synthetic mesh of
the stated shape (no dataset is involved). Each rank is an independent replica (the path
has no data-path collective); `value` sums DOF updates over ranks and divides by the
slowest rank's device time.

The headline precision is HO2D_MIXED: the FR stage kernels in FP32 (velocity from the FP64
streamfunction, RK accumulation in FP64) and FP32 BiCGSTAB with the FP32 preconditioner
inside FP64 iterative refinement of the Poisson solve (the device-resident refinement
loop). The FP64 plain path (every array and operation in FP64, exact FP64 inverse blocks)
is timed on the same workload under "fp64", and HO2D_MIXED_KRYLOV (FP64 FR stage, the same
mixed Poisson solve) under "mixed_fp64_stage", each with its relative L2 vorticity
difference from FP64 after the same steps and after --l2-steps steps.

usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""

from __future__ import annotations

import argparse
import json
import os
import shutil
import statistics
import subprocess
import sys
import tempfile
import time

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(REPO, "ho-cxx_b200"))

METRIC = "DOF-updates/s + Poisson ms/step, mixed vs FP64 on one B200 at stated L2 error"
UNIT = "DOF-updates/s"
REF_BIN = os.path.join(REPO, "oracle", "_ref", "ho2d_ref")
TRAFFIC = os.path.join(REPO, "profiles", "dram_traffic.json")
SMOOTHERS = {"blocks": 0, "bf16": 1, "kron": 2}
# algorithmic bytes per DOF-update of the FP64 FR stage kernels (trace, velocity, residual
# with the RK update), four stages of an RK4 step: per element and stage, velocity pass
# psi + 5 volume metrics + 3 face metrics + table -> u, v; residual pass omega, u, v,
# metrics, face metrics, table, omega_n and the RK accumulator
STAGE_BYTES_PER_DOF_UPDATE = {4: 848, 5: 804, 6: 775, 7: 755}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--case", default="cyl256x512")
    ap.add_argument("--knod", type=int, default=None, help="K = P + 1 (default 6 for cylinders, 5 for the step)")
    ap.add_argument("--smoother", default="kron", choices=sorted(SMOOTHERS),
                    help="smoother of the FP32 preconditioner in the mixed modes")
    ap.add_argument("--t0", type=float, default=None, help="start time (default 1.5 for the step's pulsatile inlet)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--l2-steps", type=int, default=1000,
                    help="continue every precision mode to this many steps (outside the timed region) and report "
                         "the relative vorticity L2 difference from FP64 there (0: off)")
    ap.add_argument("--no-secondary", action="store_true",
                    help="skip the secondary workloads (the step's 1000-step error, the 512^2 K=7 cavity)")
    ap.add_argument("--adjoint", action="store_true",
                    help="the differentiation case instead of the step benchmark: lid-driven cavity, K=5, Re=1000, "
                         "RK4; adjoint gradient (FP64 and mixed) against central differences")
    ap.add_argument("--adj-n", type=int, default=64, help="cavity elements per side (differentiation case)")
    ap.add_argument("--adj-steps", type=int, default=500)
    ap.add_argument("--adj-ckpt", type=int, default=25)
    ap.add_argument("--adj-dirs", type=int, default=20)
    ap.add_argument("--adjoint-large", action="store_true",
                    help="the combined large case: 512x512 jittered cavity, K=7, Re=5000, 200 RK4 steps, mixed "
                         "forward + adjoint with FP32 states; gradient error against FP64 on the 128x128 mesh")
    ap.add_argument("--large-n", type=int, default=512)
    ap.add_argument("--large-steps", type=int, default=200)
    ap.add_argument("--strouhal", action="store_true",
                    help="vortex shedding behind the cylinder (problem type 3, Re=100, 48x96 O-grid to the channel "
                         "[-15, 44] x [-15, 15], K=4): "
                         "Strouhal number, mean drag and lift amplitude in FP64 and mixed, and their differences")
    ap.add_argument("--profile-solve", action="store_true",
                    help="one solver of the headline precision on --case: --warmup steps, then --steps graph-free "
                         "BiCGSTAB iterations with per-kernel CUDA-event times (the command of the ncu captures "
                         "summarised in profiles/)")
    ap.add_argument("--t-end", type=float, default=30.0,
                    help="time units simulated for --strouhal (the pulsatile inflow peaks at t = 20)")
    ap.add_argument("--shed-knod", type=int, default=4, help="Knod of the --strouhal case")
    ap.add_argument("--long-steps", type=int, default=0,
                    help="run the backward-facing step (14,625 quads, K = 5) this many steps in FP64, HO2D_MIXED "
                         "and HO2D_MIXED_KRYLOV and report the vorticity L2 differences every 1000 steps")
    a = ap.parse_args()
    if a.knod is None:
        a.knod = 6 if a.case.startswith("cyl") else (5 if a.case.startswith("bfs") else 4)
    if a.t0 is None:
        a.t0 = 1.5 if a.case.startswith("bfs") else 0.0
    return a


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class Dist:
    """Barrier and max/sum-reduce of host floats across replicas (gloo; nothing GPU-side)."""

    def __init__(self, world):
        self.world = world
        if world > 1:
            import datetime

            import torch.distributed as td

            td.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))
            self.td = td

    def barrier(self):
        if self.world > 1:
            self.td.barrier()

    def _reduce(self, x, op):
        if self.world == 1:
            return x
        import torch

        t = torch.tensor([x], dtype=torch.float64)
        self.td.all_reduce(t, op=op)
        return float(t.item())

    def max(self, x: float) -> float:
        return self._reduce(x, self.td.ReduceOp.MAX) if self.world > 1 else x

    def sum(self, x: float) -> float:
        return self._reduce(x, self.td.ReduceOp.SUM) if self.world > 1 else x

    def close(self):
        if self.world > 1:
            self.td.destroy_process_group()


def workload_name(case, knod, t0=0.0):
    if case == "bfs":
        return (f"backward-facing step, 14,625 jittered quads (+/-0.15h, seed 2), K={knod}, Re=400, RK4, "
                f"CFL-0.5 dt, pulsatile parabolic inlet from t={t0}")
    if case.startswith("cyl"):
        nr, nt = case[3:].split("x")
        return (f"cylinder O-grid {nr} x {nt} (radial stretch 1.02, r in [0.5, 20]), K={knod}, Re=100, RK4 at the "
                f"smaller of the CFL-0.5 and viscous steps, impulsive start")
    if case.startswith("cavityj"):
        return f"lid-driven cavity {case[7:]}^2 jittered (+/-0.1h), K={knod}, RK4"
    return f"{case}, K={knod}"


class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: str):
        self.proc = None
        if shutil.which("nvidia-smi") is None:
            return
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        self.f = open(self.path, "w")
        self.proc = subprocess.Popen(["nvidia-smi", "-i", str(gpu_index), f"--query-gpu={self.FIELDS}",
                                      "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                     stderr=subprocess.DEVNULL)

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.f.close()
        with open(self.path) as f:
            out = summarize_clocks(f)
        os.remove(self.path)
        return out


def summarize_clocks(lines):
    """Median SM clock, the largest max clock and the throttle reasons seen Active in
    nvidia-smi CSV rows of ClockSampler.FIELDS (noheader, nounits); None without samples."""
    sm, smax, reasons = [], 0.0, set()
    names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    for line in lines:
        p = [x.strip() for x in line.split(",")]
        if len(p) < 9:
            continue
        try:
            sm.append(float(p[1]))
            smax = max(smax, float(p[2]))
        except ValueError:
            continue
        for nm, v in zip(names, p[5:9]):
            if v.lower().startswith("active"):
                reasons.add(nm)
    if not sm:
        return None
    return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax, "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get("hbm_gbs"), "measured"
    return 6650.0, "fallback"


def measured_traffic(kernel, case, knod, precision):
    """DRAM bytes (read + write) per element of one launch of `kernel` on this workload, from
    the ncu capture recorded in profiles/dram_traffic.json; None when there is none."""
    if not os.path.exists(TRAFFIC):
        return None
    for e in json.load(open(TRAFFIC)).get("captures", []):
        if (e["kernel"], e["case"], e["knod"], e["precision"]) == (kernel, case, knod, precision):
            return e
    return None


def _cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def reference_sample(case, knod, stages, t0, tmp):
    """The reference's own CPU step (oracle/_ref: src/HO_2D.cpp + src/Mesh.cpp built against
    the oracle's Eigen/AMGCL API shim), single thread, timed over `stages` RK4 stages.

    The reference stops at Knod = 5 and its mesh processing is quadratic in the element
    count, so the cylinder workloads are sampled on the 32 x 64 O-grid of the same shape at
    K = 5 (the K = 5 substitute), from a seeded N(0, 1) vorticity (PCG64 seed 3) -- from
    rest its first Poisson solves are trivial. Other workloads run on their own mesh (K
    capped at 5) from rest at t0. Returns a dict, or None when the binary is missing or
    fails."""
    import numpy as np

    from ho2d import meshgen

    if not os.path.exists(REF_BIN):
        return None
    k = min(knod, 5)
    if case.startswith("cyl"):
        sub = "cyl32x64"
        inp = meshgen.make_case(sub, os.path.join(tmp, "ref_" + sub), knod=k, steps=1)
        w0 = np.random.Generator(np.random.PCG64(3)).standard_normal((32 * 64, k, k))
        w0p = os.path.join(tmp, "ref_w0.npy")
        np.save(w0p, w0)
        extra = ["--init-vort", w0p]
        what = (f"K=5 substitute: the 32 x 64 O-grid of the same shape (2,048 quads) at K={k}, seeded N(0,1) "
                f"vorticity (PCG64 seed 3); the reference rejects K > 5 and its quadratic mesh processing "
                f"rules out the 131,072-quad mesh")
    else:
        inp = meshgen.make_case(case, os.path.join(tmp, "ref_" + case), knod=k, steps=1)
        extra = []
        what = f"the same mesh at K={k}, omega=0 from t={t0}"
    r = subprocess.run([REF_BIN, inp, os.path.join(tmp, "refout"), "--time-stages", str(stages), "--t0", str(t0)]
                       + extra, capture_output=True, text=True, timeout=3600)
    if r.returncode != 0:
        return None
    # the reference's destructor prints a line after the harness's JSON record
    d = json.loads([ln for ln in r.stdout.splitlines() if ln.startswith("{")][-1])
    per_stage = d["seconds"] / d["stages"]
    return {"value": d["dof"] / (4.0 * per_stage), "unit": UNIT, "cores": 1, "kind": "reference",
            "sample": f"{d['stages']} RK4 stage(s) ({d['stages'] / 4:g} step), {what}; reference setup excluded; "
                      f"Poisson {d['poisson_seconds']:.1f} s of {d['seconds']:.1f} s, {d['poisson_iterations']} "
                      f"BiCGSTAB iterations (shim solver, not AMGCL 1.4.0; tol 1e-15, maxiter 150)",
            "stages_timed": d["stages"], "seconds": d["seconds"],
            "poisson_ms_per_step": 4.0 * d["poisson_seconds"] / d["stages"] * 1e3,
            "ms_per_step": 4.0 * per_stage * 1e3, "dof": d["dof"], "cpu": _cpu_model(), "nproc": os.cpu_count()}


def run_reference(args, rank, world):
    """Reference arm: one full RK4 step (4 stages) of the reference's CPU path on the
    workload's reference sample, rank 0 only."""
    if rank != 0:
        return
    with tempfile.TemporaryDirectory() as tmp:
        if not os.path.exists(REF_BIN):
            print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/ho2d_ref was not built"}))
            return
        cb = reference_sample(args.case, args.knod, 4, args.t0, tmp)
        if cb is None:
            print(json.dumps({"impl": "reference", "unavailable": "reference run failed"}))
            return
        line = {"metric": METRIC, "value": cb["value"], "unit": UNIT, "n_gpus": world, "steps": 1, "warmup": 0,
                "ms_per_step": cb["ms_per_step"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f64", "data": "synthetic", "impl": "reference",
                "config": {"workload": workload_name(args.case, args.knod, args.t0), "reference_dof": cb["dof"],
                           "stages_timed": cb["stages_timed"]},
                "poisson_ms_per_step": cb["poisson_ms_per_step"],
                "cpu_baseline": cb,
                "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))


def pinned_like(n):
    """float64 host buffer in page-locked memory (cudaMallocHost of the runtime libho2d uses)."""
    import ctypes

    import numpy as np

    from ho2d import capi

    capi.load()
    rt = ctypes.CDLL("libcudart.so.12")
    p = ctypes.c_void_p()
    if rt.cudaMallocHost(ctypes.byref(p), ctypes.c_size_t(n * 8)) != 0:
        return np.zeros(n)
    buf = (ctypes.c_double * n).from_address(p.value)
    return np.frombuffer(buf, dtype=np.float64)


def make_solver(inp, mode, smoother, t0):
    import ho2d

    s = ho2d.HO_2D()
    s.read_input_file(inp)
    s.set_precision(mode)
    s.set_smoother(smoother)
    s.setup()
    s.set_time(t0)
    return s


def rel_l2(a, b):
    import numpy as np

    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def step_bytes(prof, iters_per_step, sweeps_per_step, solves_per_step, dof, knod, n_el, mixed, stage32=False):
    """Algorithmic bytes of one time step: the Krylov iterations (two smoothing steps, two
    operator applications, the x/r update and two coarse cycles each), the per-sweep FP64
    residual and FP32 restart of the mixed modes (or the FP64 initial residual), and the
    stage kernels: FP64, or with FP32 stage arrays (stage32) the FP64 count scaled by 0.58 --
    of the ~24 eight-byte values a stage moves per DOF, the streamfunction, the vorticity,
    the stage-start vorticity and the RK accumulator stay FP64 and the rest become FP32."""
    it = (2 * prof["smoother"][1] + 2 * prof["smoother_combine"][1] + 2 * prof["operator"][1] + prof["xr_update"][1]
          + 2 * prof["coarse_cycle"][1])
    op64 = n_el * ((6 * knod * knod + 24 * knod) * 8 + 24)  # one FP64 operator launch
    per_sweep = (op64 + prof["operator"][1] + 4 * dof * 4) if mixed else 0.0
    per_solve = op64 if not mixed else 0.0
    stage = STAGE_BYTES_PER_DOF_UPDATE.get(knod, 775) * dof * (0.58 if stage32 else 1.0)
    return iters_per_step * it + sweeps_per_step * per_sweep + solves_per_step * per_solve + stage


def time_mode(s, args, dist, phys, sample_clocks):
    n_dof = s.N_el * s.Knod * s.Knod
    s.solve_advection_diffusion(args.warmup)
    # the state the timed steps start from, for the end-to-end run over the same steps
    start = (s.get_vorticity(), s.time()[0]) if sample_clocks else None
    dist.barrier()
    sampler = ClockSampler(phys) if sample_clocks else None
    l0 = s.launch_count()
    c0 = s.solve_counters()
    tot_ms, pois_ms = s.time_steps(args.steps)
    c1 = s.solve_counters()
    launches = s.launch_count() - l0
    clocks = sampler.stop() if sampler else None
    dist.barrier()
    tmax = dist.max(tot_ms)
    pmax = dist.max(pois_ms)
    return {"ms_per_step": tmax / args.steps, "poisson_ms_per_step": pmax / args.steps,
            "value": dist.sum(n_dof * args.steps) / (tmax / 1e3), "launches": launches,
            "iters_per_step": (c1[1] - c0[1]) / args.steps, "sweeps_per_step": (c1[2] - c0[2]) / args.steps,
            "solves_per_step": (c1[0] - c0[0]) / args.steps, "iters_last_solve": s.poisson_stats()[0],
            "clocks": clocks, "start": start}


def run_long(args, rank):
    """The backward-facing step (14,625 jittered quads, K = 5, Re = 400, RK4 at CFL 0.5,
    pulsatile inlet from t = 1.5) for --long-steps steps in the three modes, with the
    relative vorticity L2 difference of both mixed modes from FP64 every 1000 steps and
    each mode's device time per step."""
    import ho2d
    from ho2d import meshgen

    if rank != 0:
        return
    with tempfile.TemporaryDirectory() as tmp:
        inp = meshgen.make_case("bfs", tmp, knod=5, steps=10)
        modes = (("fp64", ho2d.FP64), ("mixed", ho2d.MIXED), ("mixed_fp64_stage", ho2d.MIXED_KRYLOV))
        sv = {m: make_solver(inp, mode, SMOOTHERS[args.smoother], 1.5) for m, mode in modes}
        hist, ms = [], {m: 0.0 for m in sv}
        done = 0
        while done < args.long_steps:
            n = min(1000, args.long_steps - done)
            per = {}
            for m, s in sv.items():
                c0 = s.solve_counters()
                tot, pois = s.time_steps(n)
                c1 = s.solve_counters()
                ms[m] += tot
                per[m] = {"ms_per_step": tot / n, "poisson_ms_per_step": pois / n,
                          "iters_per_step": (c1[1] - c0[1]) / n, "sweeps_per_step": (c1[2] - c0[2]) / n,
                          "fp64_finishes": s.fp64_finishes()}
            done += n
            wf = sv["fp64"].get_vorticity()
            hist.append({"steps": done, "time": sv["fp64"].time()[0],
                         "mixed": rel_l2(sv["mixed"].get_vorticity(), wf),
                         "mixed_fp64_stage": rel_l2(sv["mixed_fp64_stage"].get_vorticity(), wf), "cost": per})
        print(json.dumps({"metric": "relative vorticity L2 difference from FP64 (backward-facing step)",
                          "value": hist[-1]["mixed"], "unit": "relative L2", "higher_is_better": False,
                          "n_gpus": 1, "steps": done, "dtype": "f32+f64", "data": "synthetic (seeded jitter)",
                          "config": {"workload": workload_name("bfs", 5, 1.5)},
                          "ms_per_step": {m: v / max(1, done) for m, v in ms.items()}, "history": hist}))


def secondary_workloads(args, tmp):
    """Outside the timed region of the headline: the step (14,625 quads, K = 5) after 1000
    steps in both mixed modes against FP64, and the 512^2 jittered cavity at K = 7 (mixed and
    FP64 step times)."""
    import ho2d
    from ho2d import meshgen

    out = {}
    inp = meshgen.make_case("bfs", os.path.join(tmp, "bfs"), knod=5, steps=10)
    sv = {m: make_solver(inp, mode, SMOOTHERS[args.smoother], 1.5)
          for m, mode in (("fp64", ho2d.FP64), ("mixed", ho2d.MIXED), ("mixed_fp64_stage", ho2d.MIXED_KRYLOV))}
    for s in sv.values():
        s.solve_advection_diffusion(1000)
    wf = sv["fp64"].get_vorticity()
    out["bfs14625_k5_l2_after_1000_steps"] = {"workload": workload_name("bfs", 5, 1.5),
                                              "mixed": rel_l2(sv["mixed"].get_vorticity(), wf),
                                              "mixed_fp64_stage": rel_l2(sv["mixed_fp64_stage"].get_vorticity(), wf)}
    del sv
    from ho2d.adjoint_case import cavity_dt

    dt = cavity_dt(512, 7, reyn=5000.0, jitter=0.1)
    inp = meshgen.make_case("cavityj512", os.path.join(tmp, "cav512"), knod=7, steps=10, dt=dt, reyn=5000.0,
                            jitter=0.1, seed=5)
    res = {}
    for m, mode in (("mixed", ho2d.MIXED), ("fp64", ho2d.FP64)):
        s = make_solver(inp, mode, SMOOTHERS[args.smoother], 0.0)
        s.set_vorticity(meshgen.sine_spectrum(s.getsolnpts_d(), seed=3))
        s.solve_advection_diffusion(2)
        tot, pois = s.time_steps(4)
        n_dof = s.N_el * s.Knod * s.Knod
        res[m] = {"ms_per_step": tot / 4, "poisson_ms_per_step": pois / 4, "value": n_dof * 4 / (tot / 1e3),
                  "iters_last_solve": s.poisson_stats()[0]}
        del s
    res["mixed_over_fp64"] = res["mixed"]["value"] / res["fp64"]["value"]
    res["workload"] = ("lid-driven cavity 512^2, interior jitter +/-0.1h (seed 5), K=7 (12,845,056 DOF), Re=5000, "
                       f"dt={dt:.3g}, seeded sine-spectrum vorticity (seed 3), 4 timed steps after 2")
    out["cavity512_k7"] = res
    return out


def run_ours(args, rank, world, local, phys):
    dist = Dist(world)
    import numpy as np

    import ho2d
    from ho2d import meshgen

    with tempfile.TemporaryDirectory() as tmp:
        inp = meshgen.make_case(args.case, tmp, knod=args.knod, steps=args.steps)
        sm = SMOOTHERS[args.smoother]
        modes = {"mixed": ho2d.MIXED, "fp64": ho2d.FP64, "mixed_fp64_stage": ho2d.MIXED_KRYLOV}
        solvers = {m: make_solver(inp, mode, sm, args.t0) for m, mode in modes.items()}
        s0 = solvers["mixed"]
        n_el, knod = s0.N_el, s0.Knod
        n_dof = n_el * knod * knod
        results = {m: time_mode(solvers[m], args, dist, phys, m == "mixed") for m in modes}
        # per-kernel times inside BiCGSTAB iterations on the state the timed steps left
        prof = {m: solvers[m].profile_krylov(30) for m in ("mixed", "fp64")}
        w = {m: solvers[m].get_vorticity() for m in modes}
        forces = None
        try:  # meshes with a body ("object" boundary): FP64 drag and lift of each mode
            fm, ff = solvers["mixed"].forces(), solvers["fp64"].forces()
            forces = {"mixed": fm, "fp64": ff,
                      "rel_diff_mixed_vs_fp64": float(np.hypot(fm[0] - ff[0], fm[1] - ff[1]) /
                                                      max(np.hypot(*ff), 1e-300))}
        except ho2d.HO2DError:
            pass
        # end to end through the public API with host buffers, over the same steps as the
        # timed region (from the state after warm-up): H2D of the step's input vorticity
        # from pinned memory, the step, D2H of the resulting vorticity
        s = solvers["mixed"]
        w_start, t_start = results["mixed"].pop("start")
        for r_ in results.values():
            r_.pop("start", None)
        host_in = pinned_like(n_dof)
        host_in[:] = w_start.ravel()
        host_out = pinned_like(n_dof)
        s.set_time(t_start)
        e2e_steps = args.steps
        dist.barrier()
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            s.set_vorticity(host_in)
            s.solve_advection_diffusion(1)
            s._check(s._lib.ho2d_get_vort(s._h, n_dof, ho2d.capi.dptr(host_out)))
            host_in[:] = host_out
        e2e_s = dist.max(time.perf_counter() - t0)
        e2e = {"value": dist.sum(n_dof * e2e_steps) / e2e_s, "unit": UNIT, "h2d_bytes_per_step": n_dof * 8,
               "d2h_bytes_per_step": n_dof * 8}
        # the same steps in every mode from here on (the e2e steps advanced only "mixed"):
        # the long differences start from the state after warm-up + timed steps
        l2_long = None
        done = args.warmup + args.steps
        if args.l2_steps > done:
            solvers["mixed"].set_vorticity(w["mixed"])
            solvers["mixed"].set_time(solvers["fp64"].time()[0])
            for s_ in solvers.values():
                s_.solve_advection_diffusion(args.l2_steps - done)
            wf = solvers["fp64"].get_vorticity()
            l2_long = {"steps": args.l2_steps, "mixed": rel_l2(solvers["mixed"].get_vorticity(), wf),
                       "mixed_fp64_stage": rel_l2(solvers["mixed_fp64_stage"].get_vorticity(), wf),
                       "note": "mixed restarted from its own state after the e2e steps, at the FP64 run's time"}
        del solvers, s
        peak, peak_kind = measured_peaks()
        m, f = results["mixed"], results["fp64"]
        # roofline of the kernel with the largest share of an iteration's main-stream time (the
        # coarse cycle runs on a second stream beside the fine smoothing, in the timed solves)
        launches_per_it = {"smoother": 2, "smoother_combine": 2, "operator": 2, "xr_update": 1, "coarse_cycle": 2}
        pm = prof["mixed"]
        share = {k: pm[k][0] * n for k, n in launches_per_it.items()}
        top = max((k for k in share if k != "coarse_cycle"), key=share.get)
        names = {"smoother": "k_post_a", "smoother_combine": "k_post_b", "operator": "k_mf_v/k_mf_t",
                 "xr_update": "k_xr_update",
                 "coarse_cycle": "coarse cycle (k_coarse_rows_f0, k_coarse_rows, k_dense_gemv16, k_coarse_up0)"}
        ms_top, by_top = pm[top]
        achieved = by_top / (ms_top * 1e-3) / 1e9
        tr = measured_traffic(names[top], args.case, knod, f"mixed/{args.smoother}")
        roofline = {"bound": "hbm", "kernel": names[top], "achieved": achieved, "peak": peak, "unit": "GB/s",
                    "frac": achieved / peak, "peak_kind": peak_kind,
                    "traffic": tr["dram_bytes_per_element"] * n_el if tr else None,
                    "traffic_source": tr["source"] if tr else None,
                    "launch_ms": ms_top, "algorithmic_bytes_per_launch": by_top,
                    "timing": "CUDA events between launches on the handle's stream, 30 BiCGSTAB iterations "
                              "on the state after the timed steps (no graph, launches in order: in the timed "
                              "solves each coarse cycle runs on a second stream beside k_post_a)",
                    "iteration_share": share[top] / sum(share.values()),
                    "kernels": {k: {"ms": v[0], "bytes": v[1], "gbs": v[1] / (v[0] * 1e-3) / 1e9,
                                    "frac": v[1] / (v[0] * 1e-3) / 1e9 / peak} for k, v in pm.items()}}
        for key, r_, mixed in (("mixed", m, True), ("fp64", f, False)):
            sb = step_bytes(prof[key], r_["iters_per_step"], r_["sweeps_per_step"], r_["solves_per_step"], n_dof,
                            knod, n_el, mixed, stage32=mixed)
            r_["step_level"] = {"algorithmic_bytes_per_step": sb,
                                "achieved_gbs": sb / (r_["ms_per_step"] * 1e-3) / 1e9,
                                "frac": sb / (r_["ms_per_step"] * 1e-3) / 1e9 / peak}
        fk = prof["fp64"]
        roofline_fp64 = {k: {"ms": v[0], "bytes": v[1], "frac": v[1] / (v[0] * 1e-3) / 1e9 / peak}
                         for k, v in fk.items()}
        cb = None
        if rank == 0 and world == 1 and not args.no_cpu_baseline:
            cb = reference_sample(args.case, knod, 1, args.t0, tmp)
        secondary = None
        if rank == 0 and world == 1 and not args.no_secondary and args.case == "cyl256x512":
            secondary = secondary_workloads(args, tmp)
        if rank == 0:
            def mode_out(r_):
                return {k: r_[k] for k in ("value", "ms_per_step", "poisson_ms_per_step", "iters_per_step",
                                           "sweeps_per_step", "iters_last_solve", "launches")
                        } | {"step_level": r_.get("step_level")}

            line = {"metric": METRIC, "value": m["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
                    "warmup": args.warmup, "ms_per_step": m["ms_per_step"], "higher_is_better": True,
                    "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64",
                    "data": "synthetic (seeded mesh of the stated shape)",
                    "config": {"workload": workload_name(args.case, knod, args.t0), "dof": n_dof, "n_el": n_el,
                               "parallelism": f"replicas x{world}",
                               "l2": "L2 flushed between timed steps (256 MiB device write outside the per-step "
                                     "CUDA events); working set larger than L2",
                               "poisson_tol": 1e-12, "t0": args.t0, "omega0": 0.0,
                               "smoother": args.smoother},
                    "poisson_ms_per_step": m["poisson_ms_per_step"],
                    "precision": "HO2D_MIXED: FR stage kernels in FP32 (velocity from the FP64 streamfunction, "
                                 "RK accumulation in FP64), FP32 BiCGSTAB with FP32 preconditioner "
                                 f"({args.smoother} smoother) inside FP64 iterative refinement of the Poisson solve, "
                                 "refinement loop on the device",
                    "mixed": mode_out(m),
                    "fp64": mode_out(f) | {"kernels": roofline_fp64},
                    "mixed_fp64_stage": mode_out(results["mixed_fp64_stage"]) | {
                        "precision": "HO2D_MIXED_KRYLOV: FR stage in FP64, the same mixed Poisson solve",
                        "l2_rel_vorticity_vs_fp64": rel_l2(w["mixed_fp64_stage"], w["fp64"])},
                    "mixed_over_fp64": m["value"] / f["value"],
                    "l2_rel_vorticity_mixed_vs_fp64": rel_l2(w["mixed"], w["fp64"]),
                    "l2_after_steps": args.warmup + args.steps,
                    "l2_rel_vorticity_vs_fp64_long": l2_long,
                    "body_force": forces,
                    "clocks": m["clocks"], "e2e": e2e, "gpu_launches": m["launches"], "roofline": roofline,
                    "cpu_baseline": cb, "secondary": secondary}
            print(json.dumps(line))
    dist.close()


def run_profile(args, rank):
    """The headline solver alone on --case: --warmup time steps (CUDA graphs), then --steps
    BiCGSTAB iterations launched in order without a graph, timed per kernel with CUDA events
    (Solver::profile_krylov). Kernels inside CUDA graphs with conditional nodes are not
    visible to ncu; these in-order iterations run the same kernels on the same state."""
    if rank != 0:
        return
    import ho2d
    from ho2d import meshgen

    with tempfile.TemporaryDirectory() as tmp:
        inp = meshgen.make_case(args.case, tmp, knod=args.knod, steps=args.warmup)
        s = make_solver(inp, ho2d.MIXED, SMOOTHERS[args.smoother], args.t0)
        s.solve_advection_diffusion(args.warmup)
        prof = s.profile_krylov(max(1, args.steps))
        print(json.dumps({"profile": "BiCGSTAB iterations in order, no graph", "case": args.case,
                          "knod": s.Knod, "n_el": s.N_el, "smoother": args.smoother, "iterations": args.steps,
                          "kernels": {k: {"ms": v[0], "bytes": v[1]} for k, v in prof.items()}}))


def run_adjoint(args, rank):
    """One JSON line: the adjoint gradient's largest relative error against central
    differences over the seeded directions (FP64 headline, mixed beside it), and the
    wall time of the forward and backward sweeps."""
    from ho2d import adjoint_case

    if rank != 0:
        return
    knod = 5 if args.knod is None else args.knod
    with tempfile.TemporaryDirectory() as tmp:
        r = adjoint_case.run(tmp, n=args.adj_n, knod=knod, steps=args.adj_steps, ckpt=args.adj_ckpt,
                             ndir=args.adj_dirs)
    f = r["fp64"]
    line = {"metric": "adjoint gradient relative error vs central differences (h=1e-6)",
            "value": f["max_rel_error"], "unit": "relative error", "n_gpus": 1, "higher_is_better": False,
            "dtype": "f64", "data": "synthetic (seeded sine-mode vorticity, seeded lid profile)",
            "config": {"workload": f"lid-driven cavity {args.adj_n}x{args.adj_n}, K={knod}, Re=1000, RK4, "
                                   f"{args.adj_steps} steps, checkpoints every {args.adj_ckpt}, "
                                   f"{args.adj_dirs} directions in (omega0, lid coefficients)",
                       "n_el": r["n_el"], "dof": r["dof"], "dt": r["dt"]},
            "gradient_s": f["forward_s"] + f["backward_s"],
            "gradient_over_forward": (f["forward_s"] + f["backward_s"]) / max(f["forward_s"], 1e-12),
            "adjoint_state_bytes": r["adjoint_state_bytes"], "fd_seconds": r["fd_seconds"],
            "fp64": f, "mixed": r["mixed"]}
    print(json.dumps(line))


def main():
    args = parse()
    rank, world, local = dist_env()
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if args.adjoint_large:
        from ho2d import adjoint_case

        if rank == 0:
            with tempfile.TemporaryDirectory() as tmp:
                r = adjoint_case.run_large(tmp, n=args.large_n, knod=7, steps=args.large_steps, ckpt=20)
            print(json.dumps({"metric": "combined large case: adjoint gradient error (mixed, FP32 states) vs FP64 "
                                        "adjoint on the 4x coarser mesh", "value": r["coarse"]["omega0_grad_rel_l2"],
                              "unit": "relative L2", "higher_is_better": False, "n_gpus": 1,
                              "data": "synthetic (seeded jitter, spectrum and lid)", "result": r}))
        return
    if args.strouhal:
        from ho2d import shedding

        if rank == 0:
            with tempfile.TemporaryDirectory() as tmp:
                r = shedding.run(tmp, t_end=args.t_end, knod=args.shed_knod)
            print(json.dumps({"metric": "Strouhal number of the cylinder wake (lift frequency x D / mean inflow "
                                        "speed over the analysed window)",
                              "value": r["fp64"]["St"], "unit": "St", "higher_is_better": None, "n_gpus": 1,
                              "dtype": "f64", "data": "synthetic (generated O-grid; Gaussian-vortex start)",
                              "config": {"workload": "cylinder wake, problem type 3 (pulsatile inflow "
                                                     "2|sin(pi t/40)|, Re=100 on U=1), O-grid from r=0.5 to the "
                                                     f"channel [-15, 44] x [-15, 15], t_end={args.t_end}",
                                         **r["case"]},
                              "fp64": r["fp64"], "mixed": r["mixed"], "difference": r["difference"]}))
        return
    # one GPU per rank: each replica sees only its own device
    visible = os.environ.get("CUDA_VISIBLE_DEVICES")
    devs = [d for d in visible.split(",") if d.strip()] if visible else None
    phys = devs[local % len(devs)] if devs else str(local)
    os.environ["CUDA_VISIBLE_DEVICES"] = phys
    if args.adjoint:
        run_adjoint(args, rank)
        return
    if args.profile_solve:
        run_profile(args, rank)
        return
    if args.long_steps > 0:
        run_long(args, rank)
        return
    run_ours(args, rank, world, local, phys)


if __name__ == "__main__":
    main()
