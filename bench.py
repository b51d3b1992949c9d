#!/usr/bin/env python
"""UAAMG-PCG benchmark: ms per pressure solve on the plain Poisson workload.

Workload (one "step" = one solve, as in FLIP_vdb's solve_pressure_simd,
FLIP_vdb.cpp:3118-3168): 128^3 voxels, dx = 1/128, liquid = {y < 0.4} U
sphere(r 0.15 at (0.5, 0.7, 0.5)), walls solid, face velocities U[-1,1]
(seed 0), dt = 1; build the level-0 matrix and the multigrid hierarchy, build
the right-hand side, and run UAAMG-PCG to 1e-7 relative inf-norm residual.

  value      device-resident inputs (torch CUDA tensors) through the C ABI
  e2e        the same step through the host-pointer C ABI from pinned host
             memory, host<->device copies inside the timed region
  cpu_baseline / --impl reference
             the CPU restatement of the reference's SIMD solver (oracle/),
             OpenMP over all host cores, on a bounded sample of solves

Multi-GPU: every rank solves its own independent instances (replicas; no
collective on the solve path); the step time is the max over ranks and value
is the whole-job ms per solve.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "UAAMG-PCG ms/solve to 1e-7 rel-res (plain vs batched/mixed), p99 served latency"
UNIT = "ms/solve"
WORKLOAD = "plain pressure Poisson 128^3, liquid y<0.4 + sphere r0.15, walls solid, U[-1,1] face velocities seed 0"


def _peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def _traffic_from_profile(kernel_tag: str):
    """DRAM bytes per launch of the dominant kernel from the committed ncu summary."""
    d = os.path.join(ROOT, "profiles")
    if not os.path.isdir(d):
        return None
    for fn in sorted(os.listdir(d)):
        if not fn.endswith(".md"):
            continue
        for line in open(os.path.join(d, fn)):
            if line.startswith("traffic_bytes_per_launch") and kernel_tag in line:
                try:
                    return float(line.split(":")[1].split()[0])
                except (IndexError, ValueError):
                    return None
    return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = os.path.join("/tmp", f"uaamg_clocks_{os.getpid()}.csv")

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], 0.0, set()
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except ValueError:
                continue
            for name, val in zip(("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"), f[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    if ws == 1:
        return 0, 1, 0, None
    import torch.distributed as dist
    import datetime
    rank = int(os.environ["RANK"])
    local = int(os.environ.get("LOCAL_RANK", rank))
    return rank, ws, local, dist


def cpu_solve_once(sc, threads: int):
    """One full solve with the CPU restatement (build + rhs + PCG); seconds."""
    from oracle.oracle import OraclePoisson, set_threads
    set_threads(threads)
    t0 = time.perf_counter()
    o = OraclePoisson(sc.phi, sc.face_weights, sc.dt, sc.dx)
    rhs = o.build_rhs(sc.face_weights, sc.vx, sc.vy, sc.vz, sc.solid_velocity)
    x, st, it, _ = o.solve_pcg(o.zeros(), rhs, tol=1e-7)
    dt = time.perf_counter() - t0
    return dt, it, st


def cpu_baseline(sc, budget_s: float = 12.0, min_samples: int = 3, max_samples: int = 30):
    threads = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    cpu_solve_once(sc, threads)  # warm-up
    times, iters = [], []
    t0 = time.perf_counter()
    while len(times) < max_samples and (len(times) < min_samples or time.perf_counter() - t0 < budget_s):
        dt, it, _ = cpu_solve_once(sc, threads)
        times.append(dt)
        iters.append(it)
    return {"value": round(statistics.median(times) * 1e3, 3), "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{len(times)} full solves (build+rhs+PCG) of the same 128^3 workload, median; "
                      f"oracle/poisson_oracle.c, OpenMP, {threads} threads; iterations {iters[0]}"}


def run_reference(args, rank, ws):
    """--impl reference: the CPU restatement of the reference's solver (rank 0 only)."""
    if rank != 0:
        return
    from uaamg_b200 import scenes
    sc = scenes.plain_poisson_scene(n=args.n, seed=0)
    threads = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    for _ in range(args.warmup):
        cpu_solve_once(sc, threads)
    times, iters = [], []
    for _ in range(args.steps):
        dt, it, _ = cpu_solve_once(sc, threads)
        times.append(dt)
        iters.append(it)
    ms = sum(times) / len(times) * 1e3
    line = {"metric": METRIC, "value": round(ms, 3), "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms, 3), "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic", "impl": "reference",
            "config": {"workload": WORKLOAD, "n": args.n, "iterations": iters[0]},
            "cpu_baseline": {"value": round(ms, 3), "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": f"{args.steps} full solves (build+rhs+PCG), mean; CPU restatement "
                                       f"oracle/poisson_oracle.c (the reference needs OpenVDB/TBB/Eigen, absent)"},
            "e2e": {"value": round(ms, 3), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def _gbytes(g) -> int:
    return int(g.values.nbytes + g.origins.nbytes)


def _pinned(a: np.ndarray):
    import torch
    t = torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
    return t


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=128)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-graph", action="store_true", help="host-driven PCG loop instead of the CUDA graph")
    ap.add_argument("--profile", choices=["solve", "sweep"], default=None,
                    help="short fixed sequence for ncu: 'solve' = build + 2 graph solves, "
                         "'sweep' = build + 3 level-0 Jacobi sweeps")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3) if args.impl == "ours" else args.warmup

    rank, ws, local, dist = _dist()
    if args.impl == "reference":
        run_reference(args, rank, ws)
        return

    import torch
    torch.cuda.set_device(local)
    if dist is not None:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    from uaamg_b200 import scenes
    from uaamg_b200.grids import LeafGrid
    from uaamg_b200.poisson import LaplacianWithLevel, PoissonSolver

    sc = scenes.plain_poisson_scene(n=args.n, seed=0)
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream(dev)

    def on_device(g: LeafGrid) -> LeafGrid:
        d = LeafGrid(origins=g.origins, values=g.values, background=g.background, masks=g.masks)
        d.values = torch.from_numpy(g.values).to(dev)
        return d

    def pinned(g: LeafGrid) -> LeafGrid:
        d = LeafGrid(origins=g.origins, values=g.values, background=g.background, masks=g.masks)
        t = _pinned(g.values)
        d.values = t.numpy()  # numpy view of pinned memory: host pointer path
        d._pin = t
        return d

    dgr = {k: on_device(getattr(sc, k)) for k in ("phi", "face_weights", "vx", "vy", "vz", "solid_velocity")}
    if args.profile:
        lap = LaplacianWithLevel.createPressurePoissonLaplacian(dgr["phi"], dgr["face_weights"], sc.dt, sc.dx)
        rhs = torch.empty((lap.leaf_count(0), 512), dtype=torch.float32, device=dev)
        lap.createPressurePoissonRightHandSide(dgr["face_weights"], dgr["vx"], dgr["vy"], dgr["vz"],
                                              dgr["solid_velocity"], sc.dt, out=rhs)
        if args.profile == "solve":
            solver = PoissonSolver(lap)
            solver.use_graph = not args.no_graph
            for _ in range(2):
                p = torch.zeros_like(rhs)
                st = solver.solveMultigridPCG(p, rhs)
            print(json.dumps({"profile": "solve", "status": st, "iterations": solver.mIterationTaken}))
        else:
            b = rhs.cpu().numpy()
            x = np.zeros_like(b)
            for _ in range(3):
                x = lap.apply(0, "jacobi", x, b, weight=0.8571)
            print(json.dumps({"profile": "sweep", "leaves": lap.leaf_count(0)}))
        return
    hgr = {k: pinned(getattr(sc, k)) for k in ("phi", "face_weights", "vx", "vy", "vz", "solid_velocity")}
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    stats = {"launches": 0, "iters": [], "status": []}

    def step_device():
        lap = LaplacianWithLevel.createPressurePoissonLaplacian(dgr["phi"], dgr["face_weights"], sc.dt, sc.dx)
        solver = PoissonSolver(lap)
        solver.set_stream(stream.cuda_stream)
        rhs = torch.empty((lap.leaf_count(0), 512), dtype=torch.float32, device=dev)
        lap.createPressurePoissonRightHandSide(dgr["face_weights"], dgr["vx"], dgr["vy"], dgr["vz"],
                                              dgr["solid_velocity"], sc.dt, out=rhs)
        p = torch.zeros_like(rhs)
        st = solver.solveMultigridPCG(p, rhs)
        stats["launches"] += solver.kernel_launches
        stats["iters"].append(solver.mIterationTaken)
        stats["status"].append(st)
        return lap, p

    host_p = {}

    def step_host():
        lap = LaplacianWithLevel.createPressurePoissonLaplacian(hgr["phi"], hgr["face_weights"], sc.dt, sc.dx)
        solver = PoissonSolver(lap)
        n = lap.leaf_count(0)
        if "rhs" not in host_p or host_p["rhs"].shape[0] != n:
            host_p["rhs_t"] = torch.empty((n, 512), dtype=torch.float32).pin_memory()
            host_p["p_t"] = torch.empty((n, 512), dtype=torch.float32).pin_memory()
            host_p["rhs"] = host_p["rhs_t"].numpy()
            host_p["p"] = host_p["p_t"].numpy()
        lap.createPressurePoissonRightHandSide(hgr["face_weights"], hgr["vx"], hgr["vy"], hgr["vz"],
                                              hgr["solid_velocity"], sc.dt, out=host_p["rhs"])
        host_p["p"][:] = 0.0
        st = solver.solveMultigridPCG(host_p["p"], host_p["rhs"])
        stats["launches"] += solver.kernel_launches
        return lap, st

    def timed(fn, steps, warmup):
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        total = 0.0
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        for _ in range(steps):
            flush.fill_(1.0)  # evict L2 between timed steps (256 MiB > 126 MB L2)
            torch.cuda.synchronize()
            e0.record(stream)
            fn()
            e1.record(stream)
            torch.cuda.synchronize()
            total += e0.elapsed_time(e1)
        if dist is not None:
            dist.barrier()
        return total

    # ---- headline: device-resident inputs
    clk = ClockSampler(local)
    stats.update(launches=0, iters=[], status=[])
    for _ in range(args.warmup):
        step_device()
    stats.update(launches=0, iters=[], status=[])
    clk.start()
    t_dev = timed(step_device, args.steps, 0)
    clocks = clk.stop()
    launches = stats["launches"]
    iters = list(stats["iters"])
    statuses = list(stats["status"])
    # ---- e2e through the host-pointer C ABI
    for _ in range(args.warmup):
        step_host()
    t_host = timed(step_host, args.steps, 0)

    if dist is not None:
        tt = torch.tensor([t_dev, t_host], dtype=torch.float64, device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t_dev, t_host = float(tt[0]), float(tt[1])
    total_solves = args.steps * ws
    value = t_dev / total_solves
    e2e = t_host / total_solves

    # ---- per-kernel device times (event pairs, host-driven loop) for the roofline
    lap, p = step_device()
    solver = PoissonSolver(lap)
    solver.set_stream(stream.cuda_stream)
    rhs = torch.empty((lap.leaf_count(0), 512), dtype=torch.float32, device=dev)
    lap.createPressurePoissonRightHandSide(dgr["face_weights"], dgr["vx"], dgr["vy"], dgr["vz"],
                                          dgr["solid_velocity"], sc.dt, out=rhs)
    prof = solver.profile_pcg(torch.zeros_like(rhs), rhs)
    levels = lap.num_levels()
    vec_bytes = 4 * 512 * lap.leaf_count(0)
    ndof = [lap.num_dof(l) for l in range(levels)]
    # algorithmic bytes of a level-0 Jacobi sweep: x, b, out for every DOF plus
    # diag, 1/diag, c_x, c_y, c_z for DOF in leaves whose array is stored
    # (trimmed leaves hold the default and are not read), 4 B each
    (diag, cx, cy, cz), flags = lap.coefficients(0)
    _, masks = lap.dof_topology(0)
    from uaamg_b200.grids import unpack_masks
    per_leaf = unpack_masks(masks).sum(axis=1)
    stored = lambda bit: int(per_leaf[(flags & bit) == 0].sum())
    jac_bytes = 4 * (3 * ndof[0] + 2 * stored(1) + stored(2) + stored(4) + stored(8))
    # the level-0 plain Jacobi sweep (staged or not); the fused variants move
    # the same bytes plus small extras and are reported in kernel_profile_ms
    tags = [k for k in prof if k.startswith("L0 jacobi") and "+" not in k]
    tag = tags[0] if tags else "L0 jacobi"
    t_ms, cnt = prof.get(tag, (0.0, 0))
    achieved = jac_bytes / (t_ms / cnt * 1e-3) / 1e9 if cnt else None
    peak, peak_kind = _peaks()
    traffic = _traffic_from_profile("k_sweep_staged<0>")
    dominant = max(prof.items(), key=lambda kv: kv[1][0])
    cpu = None
    if rank == 0 and not args.no_cpu_baseline and ws == 1:
        cpu = cpu_baseline(sc)
    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 4), "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(t_dev / args.steps, 4), "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "n": args.n, "ndof": ndof, "levels": levels,
                       "pcg_iterations": iters[0], "status": "SUCCESS" if all(s == 0 for s in statuses) else "FAILED",
                       "step": "create matrix+hierarchy, rhs, UAAMG-PCG (device-resident inputs)",
                       "l2": "flushed before every timed step (256 MiB write)",
                       "parallelism": f"replicas x{ws}", "solves_per_s": round(1e3 / value, 2),
                       "voxel_updates_per_s": round(ndof[0] * iters[0] * 1e3 / value, 1)},
            "e2e": {"value": round(e2e, 4), "unit": UNIT,
                    # create: phi (+mask) and face weights; rhs: face weights and
                    # three velocity channels; solve: pressure guess and rhs
                    "h2d_bytes_per_step": int(_gbytes(sc.phi) + sc.phi.masks.nbytes + 2 * _gbytes(sc.face_weights)
                                              + sum(_gbytes(getattr(sc, k)) for k in ("vx", "vy", "vz"))
                                              + 2 * vec_bytes),
                    # rhs returned to the caller, solved pressure
                    "d2h_bytes_per_step": int(2 * vec_bytes)},
            "gpu_launches": int(launches),
            "roofline": {"bound": "hbm", "kernel": f"level-0 Jacobi sweep ({tag})",
                         "achieved": round(achieved, 1) if achieved else None, "peak": peak,
                         "peak_kind": peak_kind, "unit": "GB/s",
                         "frac": round(achieved / peak, 4) if achieved else None,
                         "traffic": traffic, "algorithmic_bytes": jac_bytes,
                         "avg_launch_us": round(t_ms / cnt * 1e3, 2) if cnt else None},
            "kernel_profile_ms": {k: [round(v[0], 4), v[1]] for k, v in sorted(prof.items(), key=lambda kv: -kv[1][0])},
            "dominant_kernel": dominant[0],
            "clocks": clocks,
        }
        if cpu is not None:
            line["cpu_baseline"] = cpu
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
