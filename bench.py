"""Benchmark: DOF-updates/s and Poisson ms/step of the FR time step on one B200.

Workload (default): the backward-facing step with ~15,000 jittered quads (14,625
elements, h = 1/15, +/-0.15h interior jitter, seed 2), K = P+1 = 5 (365,625 DOF),
Re = 400, RK4 at CFL 0.5, parabolic pulsatile inlet -- synthetic mesh of the stated
shape (no dataset is involved). Each rank is an independent replica (the path has no
data-path collective); `value` sums DOF updates over ranks and divides by the slowest
rank's device time.

The headline precision is mixed (FP32 FR residual + FP32 BiCGSTAB inside FP64 iterative
refinement, FP64 RK accumulation); the FP64 plain path is timed on the same workload and
reported under "fp64", with the relative L2 vorticity difference between the two after
the same steps.

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


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--case", default="bfs")
    ap.add_argument("--knod", type=int, default=5)
    ap.add_argument("--cpu-stages", type=int, default=1, help="RK stages timed for the CPU baseline sample")
    ap.add_argument("--t0", type=float, default=1.5, help="start time inside the pulsatile inflow cycle")
    ap.add_argument("--no-cpu-baseline", action="store_true")
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
                    help="vortex shedding behind the cylinder (problem type 3, Re=100, 48x96 O-grid, K=4): "
                         "Strouhal number, mean drag and lift amplitude in FP64 and mixed, and their differences")
    ap.add_argument("--t-end", type=float, default=80.0, help="time units simulated for --strouhal")
    ap.add_argument("--shed-knod", type=int, default=4, help="Knod of the --strouhal case")
    ap.add_argument("--l2-steps", type=int, default=0,
                    help="also continue every precision mode to this many steps (outside the timed region) and "
                         "report the relative vorticity L2 difference from FP64 there")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class Dist:
    """Barrier and max-reduce of host floats across replicas (gloo; nothing GPU-side)."""

    def __init__(self, world):
        self.world = world
        self.pg = None
        if world > 1:
            import datetime

            import torch.distributed as td

            td.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))
            self.td = td

    def barrier(self):
        if self.world > 1:
            self.td.barrier()

    def max(self, x: float) -> float:
        if self.world == 1:
            return x
        import torch

        t = torch.tensor([x], dtype=torch.float64)
        self.td.all_reduce(t, op=self.td.ReduceOp.MAX)
        return float(t.item())

    def sum(self, x: float) -> float:
        if self.world == 1:
            return x
        import torch

        t = torch.tensor([x], dtype=torch.float64)
        self.td.all_reduce(t, op=self.td.ReduceOp.SUM)
        return float(t.item())

    def close(self):
        if self.world > 1:
            self.td.destroy_process_group()


def make_workload(tmp, case, knod, steps):
    from ho2d import meshgen

    return meshgen.make_case(case, tmp, knod=knod, steps=steps)


class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.proc = None
        self.path = None
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


def cpu_baseline(inp, stages, t0=1.5):
    """The reference's own CPU step (oracle/_ref: src/HO_2D.cpp + src/Mesh.cpp built against
    the oracle's Eigen/AMGCL API shim), single thread, timed over `stages` RK stages of
    the same workload; DOF-updates/s = DOF / (4 * seconds per stage)."""
    if not os.path.exists(REF_BIN):
        return None
    r = subprocess.run([REF_BIN, inp, os.path.join(os.path.dirname(inp), "refout"), "--time-stages", str(stages),
                        "--t0", str(t0)],
                       capture_output=True, text=True, timeout=1800)
    if r.returncode != 0:
        return None
    # the reference's destructor prints a line after the harness's JSON record
    d = json.loads([ln for ln in r.stdout.splitlines() if ln.startswith("{")][-1])
    per_stage = d["seconds"] / d["stages"]
    value = d["dof"] / (4.0 * per_stage)
    return {"value": value, "unit": UNIT, "cores": 1, "kind": "reference",
            "sample": f"{d['stages']} RK4 stage(s) of the same mesh (DOF {d['dof']}) from t={t0}, omega=0, "
                      f"reference setup excluded; "
                      f"Poisson solve {d['poisson_seconds']:.1f} s of {d['seconds']:.1f} s "
                      f"({d['poisson_iterations']} shim BiCGSTAB iterations, tol 1e-15, maxiter 150; "
                      f"shim solver, not AMGCL 1.4.0)",
            "poisson_ms_per_step": 4.0 * d["poisson_seconds"] / d["stages"] * 1e3,
            "ms_per_step": 4.0 * per_stage * 1e3, "dof": d["dof"],
            "cpu": _cpu_model(), "nproc": os.cpu_count()}


def _cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def run_reference(args, rank, world):
    if rank != 0:
        return
    with tempfile.TemporaryDirectory() as tmp:
        inp = make_workload(tmp, args.case, args.knod, 1)
        if not os.path.exists(REF_BIN):
            print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/ho2d_ref was not built"}))
            return
        # one bounded sample (a full RK4 stage of the reference takes ~80 s on this mesh)
        cb = cpu_baseline(inp, args.cpu_stages, args.t0)
        if cb is None:
            print(json.dumps({"impl": "reference", "unavailable": "reference run failed"}))
            return
        vals = [cb["value"]]
        value = statistics.median(vals)
        dof = cb["dof"]
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": 0, "ms_per_step": cb["ms_per_step"], "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None,
                "dtype": "f64", "data": "synthetic", "impl": "reference",
                "config": {"workload": workload_name(args), "dof": dof},
                "cpu_baseline": dict(cb, value=value),
                "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))


def workload_name(args):
    if args.case == "bfs":
        return (f"backward-facing step, 14,625 jittered quads (+/-0.15h, seed 2), K={args.knod}, Re=400, RK4, "
                f"CFL-0.5 dt, pulsatile parabolic inlet")
    return f"{args.case}, K={args.knod}"


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


def run_ours(args, rank, world, local, phys):
    dist = Dist(world)
    import numpy as np

    import ho2d

    with tempfile.TemporaryDirectory() as tmp:
        inp = make_workload(tmp, args.case, args.knod, args.steps)
        solvers = {}
        # headline: FP64 FR stage with the FP32 Krylov inside FP64 refinement (meets the
        # 1e-6 vorticity target); "mixed_fp32_stage" also runs the FR stage in FP32
        modes = {"mixed": ho2d.MIXED_KRYLOV, "fp64": ho2d.FP64, "mixed_fp32_stage": ho2d.MIXED}
        for prec, mode in modes.items():
            s = ho2d.HO_2D()
            s.read_input_file(inp)
            s.set_precision(mode)
            s.setup()
            s.set_time(args.t0)
            solvers[prec] = s
        s0 = solvers["mixed"]
        n_dof = s0.N_el * s0.Knod * s0.Knod
        results = {}
        clocks = None
        for prec in modes:
            s = solvers[prec]
            s.solve_advection_diffusion(args.warmup)
            dist.barrier()
            sampler = ClockSampler(phys) if prec == "mixed" else None
            l0 = s.launch_count()
            tot_ms, pois_ms = s.time_steps(args.steps)
            launches = s.launch_count() - l0
            if sampler:
                clocks = sampler.stop()
            dist.barrier()
            tmax = dist.max(tot_ms)
            pmax = dist.max(pois_ms)
            spmv_ms, spmv_bytes = s.profile_spmv(30)
            results[prec] = {"ms_per_step": tmax / args.steps, "poisson_ms_per_step": pmax / args.steps,
                             "value": dist.sum(n_dof * args.steps) / (tmax / 1e3), "launches": launches,
                             "spmv_ms": spmv_ms, "spmv_bytes": spmv_bytes, "iters": s.poisson_stats()[0]}
        w_mixed = solvers["mixed"].get_vorticity()
        w_fp64 = solvers["fp64"].get_vorticity()
        l2 = float(np.linalg.norm(w_mixed - w_fp64) / max(np.linalg.norm(w_fp64), 1e-300))
        forces = None
        try:  # meshes with a body ("object" boundary): FP64 drag and lift of each mode
            fm, ff = solvers["mixed"].forces(), solvers["fp64"].forces()
            forces = {"mixed": fm, "fp64": ff,
                      "rel_diff_mixed_vs_fp64": float(np.hypot(fm[0] - ff[0], fm[1] - ff[1]) /
                                                      max(np.hypot(*ff), 1e-300))}
        except ho2d.HO2DError:
            pass
        w_f32 = solvers["mixed_fp32_stage"].get_vorticity()
        l2_f32 = float(np.linalg.norm(w_f32 - w_fp64) / max(np.linalg.norm(w_fp64), 1e-300))
        l2_long = None
        done = args.warmup + args.steps
        if args.l2_steps > done:  # the same steps in every mode, then the differences from FP64
            for s_ in solvers.values():
                s_.solve_advection_diffusion(args.l2_steps - done)
            wf = solvers["fp64"].get_vorticity()
            nf = max(np.linalg.norm(wf), 1e-300)
            l2_long = {"steps": args.l2_steps,
                       "mixed": float(np.linalg.norm(solvers["mixed"].get_vorticity() - wf) / nf),
                       "mixed_fp32_stage": float(np.linalg.norm(solvers["mixed_fp32_stage"].get_vorticity() - wf) / nf)}
        # end to end through the public API with host buffers: H2D of the step's input
        # vorticity from pinned memory, the step, D2H of the resulting vorticity
        s = solvers["mixed"]
        host_in = pinned_like(n_dof)
        host_in[:] = w_mixed.ravel()
        host_out = pinned_like(n_dof)
        e2e_steps = max(3, args.steps // 2)
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
        peak, peak_kind = measured_peaks()
        # DRAM bytes (read + write) of one k_mf_apply<5, float> launch on this workload, from
        # the ncu capture summarised in profiles/k_mf_apply_bfs14625_k5_fp32.md
        traffic = 13118720 if (args.case == "bfs" and args.knod == 5) else None
        m = results["mixed"]
        achieved = m["spmv_bytes"] / (m["spmv_ms"] * 1e-3) / 1e9
        roofline = {"bound": "hbm", "kernel": "k_mf_apply (matrix-free Poisson operator, FP32 inner Krylov)",
                    "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                    "peak_kind": peak_kind, "traffic": traffic,
                    "launch_ms": m["spmv_ms"], "algorithmic_bytes_per_launch": m["spmv_bytes"]}
        f = results["fp64"]
        roofline_fp64 = {"kernel": "k_mf_apply (FP64)", "achieved": f["spmv_bytes"] / (f["spmv_ms"] * 1e-3) / 1e9,
                         "launch_ms": f["spmv_ms"], "algorithmic_bytes_per_launch": f["spmv_bytes"]}
        roofline_fp64["frac"] = roofline_fp64["achieved"] / peak
        cb = None
        if rank == 0 and world == 1 and not args.no_cpu_baseline:
            cb = cpu_baseline(inp, args.cpu_stages, args.t0)
        if rank == 0:
            line = {"metric": METRIC, "value": m["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
                    "warmup": args.warmup, "ms_per_step": m["ms_per_step"], "higher_is_better": True,
                    "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64",
                    "data": "synthetic (seeded mesh of the stated shape)",
                    "config": {"workload": workload_name(args), "dof": n_dof, "n_el": s0.N_el,
                               "parallelism": f"replicas x{world}", "l2": "L2 flushed between timed steps (256 MiB device "
                               "write outside the per-step CUDA events)",
                               "poisson_tol": 1e-12, "t0": args.t0, "omega0": 0.0},
                    "poisson_ms_per_step": m["poisson_ms_per_step"],
                    "poisson_iterations_last_solve": m["iters"],
                    "fp64": {"value": f["value"], "ms_per_step": f["ms_per_step"],
                             "poisson_ms_per_step": f["poisson_ms_per_step"], "roofline": roofline_fp64,
                             "poisson_iterations_last_solve": f["iters"]},
                    "precision": "HO2D_MIXED_KRYLOV: FP64 FR stage and RK update, FP32 BiCGSTAB with FP32 "
                                 "preconditioner inside FP64 iterative refinement of the Poisson solve",
                    "mixed_fp32_stage": {"precision": "HO2D_MIXED: FR stage also in FP32",
                                         "value": results["mixed_fp32_stage"]["value"],
                                         "ms_per_step": results["mixed_fp32_stage"]["ms_per_step"],
                                         "poisson_ms_per_step": results["mixed_fp32_stage"]["poisson_ms_per_step"],
                                         "poisson_iterations_last_solve": results["mixed_fp32_stage"]["iters"],
                                         "l2_rel_vorticity_vs_fp64": l2_f32},
                    "mixed_over_fp64": m["value"] / f["value"],
                    "l2_rel_vorticity_mixed_vs_fp64": l2,
                    "l2_after_steps": args.warmup + args.steps,
                    "l2_rel_vorticity_vs_fp64_long": l2_long,
                    "body_force": forces,
                    "clocks": clocks, "e2e": e2e, "gpu_launches": m["launches"], "roofline": roofline,
                    "cpu_baseline": cb}
            print(json.dumps(line))
    dist.close()


def run_adjoint(args, rank):
    """One JSON line: the adjoint gradient's largest relative error against central
    differences over the seeded directions (FP64 headline, mixed beside it), and the
    wall time of the forward and backward sweeps."""
    from ho2d import adjoint_case

    if rank != 0:
        return
    with tempfile.TemporaryDirectory() as tmp:
        r = adjoint_case.run(tmp, n=args.adj_n, knod=args.knod, steps=args.adj_steps, ckpt=args.adj_ckpt,
                             ndir=args.adj_dirs)
    f = r["fp64"]
    line = {"metric": "adjoint gradient relative error vs central differences (h=1e-6)",
            "value": f["max_rel_error"], "unit": "relative error", "n_gpus": 1, "higher_is_better": False,
            "dtype": "f64", "data": "synthetic (seeded sine-mode vorticity, seeded lid profile)",
            "config": {"workload": f"lid-driven cavity {args.adj_n}x{args.adj_n}, K={args.knod}, Re=1000, RK4, "
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
            print(json.dumps({"metric": "Strouhal number of the cylinder wake (lift frequency x D / U)",
                              "value": r["fp64"]["St"], "unit": "St", "higher_is_better": None, "n_gpus": 1,
                              "dtype": "f64", "data": "synthetic (generated O-grid; Gaussian-vortex start)",
                              "config": {"workload": "cylinder wake, Re=100, O-grid r in [0.5, 15], "
                                                     f"t_end={args.t_end}", **r["case"]},
                              "fp64": r["fp64"], "mixed": r["mixed"], "difference": r["difference"]}))
        return
    if args.adjoint:
        visible = os.environ.get("CUDA_VISIBLE_DEVICES")
        devs = [d for d in visible.split(",") if d.strip()] if visible else None
        os.environ["CUDA_VISIBLE_DEVICES"] = devs[local % len(devs)] if devs else str(local)
        run_adjoint(args, rank)
        return
    # one GPU per rank: each replica sees only its own device
    visible = os.environ.get("CUDA_VISIBLE_DEVICES")
    devs = [d for d in visible.split(",") if d.strip()] if visible else None
    phys = devs[local % len(devs)] if devs else str(local)
    os.environ["CUDA_VISIBLE_DEVICES"] = phys
    run_ours(args, rank, world, local, phys)


if __name__ == "__main__":
    main()
