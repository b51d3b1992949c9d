#!/usr/bin/env python
"""UAAMG-PCG benchmark: ms per solve.

Headline workload (one "step" = one pressure projection solve as at FLIP_vdb's
call site, FLIP_vdb.cpp:3118-3168): the 128^3 domain, dx = 1/128, liquid =
{y < 0.4} U sphere(r 0.15 at (0.5, 0.7, 0.5)), domain walls solid (face
fraction 0), free surface as Dirichlet p = 0 with ghost-fluid fractions from the
SDF, rhs = negative divergence of face velocities U[-1,1] (seed 0), dt = 1; build
the level-0 matrix, the multigrid hierarchy and the right-hand side, and run
UAAMG-PCG (scheduled relaxed Jacobi) from a zero pressure to 1e-7 relative
inf-norm residual (PoissonSolver::solveMultigridPCG).

Secondary objects of the same line: the plain variational viscosity solve on
the same geometry ("viscosity"), the batched, mixed-precision and served forms,
and the projection steps around the solve.

  value      device-resident inputs (torch CUDA tensors) through the C ABI
             (uaamg_poisson_create_with_rhs, uaamg_poisson_solve_pcg_resident_device)
  e2e        the same step through the host-pointer C ABI from pinned host
             memory (uaamg_poisson_create_with_rhs with host grids, then
             uaamg_poisson_solve_pcg_resident: the pressure back to the host),
             host<->device copies inside the timed region
  cpu_baseline / --impl reference
             the CPU restatement of the reference's SIMD solver (oracle/),
             OpenMP over all host cores, full solves of the same workload

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
POISSON_WORKLOAD = ("plain pressure Poisson 128^3, dx 1/128, liquid y<0.4 + sphere r0.15 at (0.5,0.7,0.5), walls solid, "
                    "ghost-fluid free surface, rhs = -div of U[-1,1] face velocities seed 0, dt 1, rel-res 1e-7, "
                    "zero initial pressure")


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


def _threads() -> int:
    return len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()


def cpu_solve_once(sc, threads: int):
    """One full Poisson solve with the CPU restatement (build + rhs + PCG); seconds."""
    from oracle.oracle import OraclePoisson, set_threads
    set_threads(threads)
    t0 = time.perf_counter()
    o = OraclePoisson(sc.phi, sc.face_weights, sc.dt, sc.dx)
    rhs = o.build_rhs(sc.face_weights, sc.vx, sc.vy, sc.vz, sc.solid_velocity)
    x, st, it, _ = o.solve_pcg(o.zeros(), rhs, tol=1e-7)
    dt = time.perf_counter() - t0
    return dt, it, st


def _visc_warm_start(o, sc):
    """The velocity at every DOF (FLIP_vdb.cpp:3188-3198), from the oracle's
    topology: each DOF leaf is matched to the velocity grid's leaf at the same
    origin by a sorted-key search, then the values are copied under the DOF
    masks, all as whole-array operations."""
    org, _ = o.topology(0)
    idx = o.dof_index(0)
    out = o.zeros(0)

    def keys(a):
        a = a.astype(np.int64) + (1 << 20)
        return (a[:, 0] << 42) | (a[:, 1] << 21) | a[:, 2]

    k0 = keys(org)
    for c, g in enumerate((sc.u, sc.v, sc.w)):
        kg = keys(g.origins)
        order = np.argsort(kg)
        pos = np.searchsorted(kg[order], k0)
        pos = np.minimum(pos, len(kg) - 1)
        j = order[pos]
        hit = kg[j] == k0
        vals = np.zeros((org.shape[0], 512), np.float32)
        vals[hit] = g.values[j[hit]].reshape(-1, 512)
        m = idx[c] >= 0
        out[c][m] = vals[m]
    return out


def cpu_visc_solve_once(sc, threads: int):
    """One full viscosity solve with the CPU restatement (build + rhs + warm
    start + PCG); seconds."""
    from oracle.oracle import OracleViscosity, set_threads
    set_threads(threads)
    t0 = time.perf_counter()
    o = OracleViscosity(sc.liquid_phi, sc.solid_phi, sc.viscosity, sc.dt, sc.rho, sc.dx)
    rhs = o.build_rhs(sc.u, sc.v, sc.w, sc.solid_velocity)
    x0 = _visc_warm_start(o, sc)
    x, st, it, _ = o.solve_pcg(x0, rhs, 1e-6, 100)
    dt = time.perf_counter() - t0
    return dt, it, st


def cpu_baseline(fn, sc, what: str, budget_s: float = 12.0, min_samples: int = 3, max_samples: int = 30):
    threads = _threads()
    fn(sc, threads)  # warm-up
    times, iters = [], []
    t0 = time.perf_counter()
    while len(times) < max_samples and (len(times) < min_samples or time.perf_counter() - t0 < budget_s):
        dt, it, _ = fn(sc, threads)
        times.append(dt)
        iters.append(it)
    return {"value": round(statistics.median(times) * 1e3, 3), "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{len(times)} full solves of the same 128^3 workload, median; {what}, OpenMP, "
                      f"{threads} threads; iterations {iters[0]}"}


def run_reference(args, rank, ws):
    """--impl reference: the CPU restatement of the reference's solver on the
    headline workload (rank 0 only; the other ranks exit without work)."""
    if rank != 0:
        return
    from uaamg_b200 import scenes
    sc = scenes.plain_poisson_scene(n=args.n, seed=0)
    threads = _threads()
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
            "config": poisson_config(args),
            "solve": {"pcg_iterations": iters[0]},
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


def _grid_bytes(*gs) -> int:
    return int(sum(_gbytes(g) + (g.masks.nbytes if g.masks is not None else 0) for g in gs))


def _map_bytes(g) -> int:
    """The dense leaf map the library uploads for a grid (one int32 per leaf
    cell of the origins' bounding box)."""
    if g.leaf_count == 0:
        return 0
    c = np.asarray(g.origins).reshape(-1, 3) >> 3
    return int(np.prod(c.max(0) - c.min(0) + 1)) * 4


def _pressure_h2d_bytes(phi, fw, vels) -> int:
    """Bytes uaamg_poisson_create_with_rhs moves host->device for pinned
    inputs: the liquid SDF whole (values, origins, active masks, leaf map); of
    each face grid only the leaves the construction reads (at a liquid leaf
    or the next leaf above one along x, y or z), with its origins and leaf map
    (the velocity channels share the face weights' map and read flags when
    their leaves are the same)."""
    po = np.asarray(phi.origins).reshape(-1, 3)
    vals = np.asarray(phi.values).reshape(phi.leaf_count, 512)
    liq = vals < 0
    if phi.masks is not None:
        bits = np.unpackbits(np.asarray(phi.masks, np.uint64).reshape(-1, 8).view(np.uint8), axis=1,
                             bitorder="little").astype(bool)
        liq &= bits
    liquid = {tuple(o) for o in po[liq.any(1)]}
    total = _gbytes(phi) + po.nbytes + (phi.masks.nbytes if phi.masks is not None else 0) + _map_bytes(phi)
    shared = None
    for i, g in enumerate([fw] + list(vels)):
        if g.leaf_count == 0:
            continue
        org = np.asarray(g.origins).reshape(-1, 3)
        if i > 0 and shared is not None and np.array_equal(org, shared):
            pass  # map and read flags of the face weights
        else:
            total += _map_bytes(g) + org.nbytes
            if i == 0:
                shared = org
        read = np.array([any(tuple(o - d) in liquid for d in ((0, 0, 0), (8, 0, 0), (0, 8, 0), (0, 0, 8)))
                         for o in org])
        total += int(read.sum()) * 512 * 4 * g.components
    return int(total)


# algorithmic bytes of one pass per DOF it updates (canonical model: every array
# read or written once at 4 B, halos excluded): GS colour pass of one channel =
# half of the 44 B two-colour channel sweep; residual 44 B and A.x 40 B per
# channel DOF; restriction 4.5 B and prolong-add 8.5 B per fine DOF
def _visc_pass_bytes(label: str, ndof_level: list[int], ndof_c: list[list[int]]) -> float | None:
    parts = label.split()
    if not parts or not parts[0].startswith("L") or not parts[0][1:].isdigit():
        return None
    lv = int(parts[0][1:])
    if len(parts) >= 3 and parts[1] in ("red_gs", "black_gs"):
        c = int(parts[2][1:])
        return 22.0 * ndof_c[lv][c]
    if len(parts) >= 4 and parts[1] == "rbgs" and parts[2] == "step":  # fused red+black: one pass's bytes
        c = int(parts[3][1:])
        return 22.0 * ndof_c[lv][c]
    if parts[1] == "residual":
        return 44.0 * ndof_level[lv]
    if parts[1] == "normal":
        return 40.0 * ndof_level[lv]
    if parts[1] == "restrict":
        return 4.5 * ndof_level[lv]
    if parts[1] == "prolong":
        return 8.5 * ndof_level[lv]
    return None


def poisson_config(args) -> dict:
    """The headline workload's configuration; both arms print the same dict."""
    return {"workload": POISSON_WORKLOAD, "n": args.n, "rel_tol": 1e-7, "smoother": "scheduled relaxed Jacobi",
            "step": "build level-0 matrix + multigrid hierarchy + rhs, UAAMG-PCG from a zero pressure",
            "l2": "flushed before every timed step (256 MiB write)", "parallelism": "replicas"}


class PoissonBytes:
    """Algorithmic bytes per launch of the Poisson solve's kernel classes (the
    labels of the event-timed profile): every array a kernel must touch,
    counted once per DOF of its level at 4 B; the coefficient arrays (diag,
    1/diag, c_x, c_y, c_z) only for DOF in leaves where they are stored (a
    trimmed leaf holds the default and is not read); halo re-reads and
    inactive voxels not credited; a restriction writes 4 B per 8 fine DOF, a
    prolongation reads as much."""

    TRIM_DIAG, TRIM_X, TRIM_Y, TRIM_Z = 1, 2, 4, 8

    def __init__(self, lap):
        self.levels = []
        for l in range(lap.num_levels()):
            _, masks = lap.dof_topology(l)
            dof = np.array([sum(bin(int(w)).count("1") for w in row) for row in masks], np.int64)
            _, flags = lap.coefficients(l)
            fl = flags.astype(np.int64)
            stored = {k: int(dof[(fl & bit) == 0].sum()) for k, bit in
                      (("diag", self.TRIM_DIAG), ("cx", self.TRIM_X), ("cy", self.TRIM_Y), ("cz", self.TRIM_Z))}
            self.levels.append((int(dof.sum()), stored))

    def _coef(self, l, with_inv: bool) -> float:
        n, st = self.levels[l]
        b = 4.0 * (st["diag"] + st["cx"] + st["cy"] + st["cz"])
        return b + (4.0 * st["diag"] if with_inv else 0.0)

    def launch_bytes(self, label: str):
        parts = label.split()
        if not parts or not parts[0].startswith("L") or not parts[0][1:].isdigit():
            return None
        l = int(parts[0][1:])
        if l >= len(self.levels):
            return None
        n = float(self.levels[l][0])
        kind = " ".join(parts[1:]).replace(" staged", "")
        dot = 4.0 * n if kind.endswith("+dot") else 0.0
        kind = kind.replace("+dot", "")
        if kind == "jacobi":                     # x, b, out + coefficients and 1/diag
            return 12.0 * n + self._coef(l, True) + dot
        if kind == "jacobi+first":               # b, out (x computed from b) + coefficients and 1/diag
            return 8.0 * n + self._coef(l, True) + dot
        if kind == "jacobi+prolong":             # x, b, out, coarse x + coefficients and 1/diag
            return 12.5 * n + self._coef(l, True) + dot
        if kind == "residual+restrict":          # x, b + coefficients, coarse rhs
            return 8.5 * n + self._coef(l, False)
        if kind == "materialize+first":          # b, 1/diag, out
            return 8.0 * n + 4.0 * self.levels[l][1]["diag"]
        if kind == "materialize+prolong":        # x in place, coarse x
            return 8.5 * n
        if kind == "pcg Ap":                     # p, q + coefficients (+ p.q)
            return 8.0 * n + self._coef(l, False)
        if kind == "pcg r update+absmax":        # q, r in place
            return 12.0 * n
        if kind == "pcg x,p update":             # z, p in place, x in place
            return 20.0 * n
        return None

    @staticmethod
    def ncu_tag(label: str, leaves: int) -> str:
        """The kernel name and level size the committed ncu summaries use for
        this class (a kernel's traffic depends on the level it sweeps)."""
        if "jacobi staged" in label and "+dot" not in label:
            return f"k_sweep_staged<0> ({leaves} leaves)"
        return label


VISC_WORKLOAD = ("plain variational viscosity 128^3, liquid y<0.4 + sphere r0.15, walls solid, U[-1,1] face velocities "
                 "seed 1, mu 1e3, dt 1/240, rho 1, rel-res 1e-6, warm start = velocity")


def run_viscosity(args, dev, stream, timed, max_over_ranks, ws, rank, vsc, vdg, pinned):
    """The plain variational viscosity solve (FLIP_vdb.cpp:3170-3208): build the
    level-0 matrix and the hierarchy, the rhs and the warm start (the velocity
    at the DOFs), UAAMG-PCG to 1e-6.  value: device-resident grids; e2e: the
    host-pointer C ABI from pinned memory (uaamg_viscosity_create, then
    uaamg_viscosity_solve_velocity: the velocity in, the solved velocity out)."""
    import torch
    from uaamg_b200.viscosity import L_with_level, simd_viscosity3d
    vstats = {"launches": 0, "iters": [], "status": []}

    def vstep_device():
        lv = L_with_level.create_viscosity_matrix(vdg["viscosity"], vdg["liquid_phi"], vdg["solid_phi"], vsc.dt,
                                                  vsc.rho, vsc.dx)
        lv.set_stream(stream.cuda_stream)
        n = lv.leaf_count(0)
        rhs = torch.empty((3, n, 512), dtype=torch.float32, device=dev)
        lv.build_rhs(vdg["u"], vdg["v"], vdg["w"], vdg["solid_velocity"], out=rhs)
        x = torch.empty_like(rhs)
        lv.gather_velocity(vdg["u"], vdg["v"], vdg["w"], out=x)
        s = simd_viscosity3d(lv)
        st = s.pcg_solve(x, 1e-6, rhs)
        vstats["launches"] += s.kernel_launches
        vstats["iters"].append(s.m_iteration)
        vstats["status"].append(st)
        return lv, x

    vkeys = ("liquid_phi", "solid_phi", "viscosity", "u", "v", "w", "solid_velocity")
    vhg = {k: pinned(getattr(vsc, k)) for k in vkeys}
    vhost = {}

    def vstep_host():
        lv = L_with_level.create_viscosity_matrix(vhg["viscosity"], vhg["liquid_phi"], vhg["solid_phi"], vsc.dt,
                                                  vsc.rho, vsc.dx)
        n = lv.leaf_count(0)
        if vhost.get("n") != n:
            vhost["x_t"] = torch.empty((3, n, 512), dtype=torch.float32).pin_memory()
            vhost["x"], vhost["n"] = vhost["x_t"].numpy(), n
        s = simd_viscosity3d(lv)
        st, _ = s.solve_velocity(vhg["u"], vhg["v"], vhg["w"], vhg["solid_velocity"], 1e-6, out=vhost["x"])
        vstats["launches"] += s.kernel_launches
        return lv, st

    for _ in range(args.warmup):
        vstep_device()
    vstats.update(launches=0, iters=[], status=[])
    t_dev = timed(vstep_device, args.steps)
    launches = vstats["launches"]
    viters, vstatus = list(vstats["iters"]), list(vstats["status"])
    for _ in range(args.warmup):
        vstep_host()
    t_host = timed(vstep_host, args.steps)
    t_dev, t_host = max_over_ranks(t_dev, t_host)
    total = args.steps * ws
    value, e2e = t_dev / total, t_host / total

    # per-kernel device times (event pairs, host-driven loop) for the roofline
    lv, _ = vstep_device()
    n0 = lv.leaf_count(0)
    rhs = torch.empty((3, n0, 512), dtype=torch.float32, device=dev)
    lv.build_rhs(vdg["u"], vdg["v"], vdg["w"], vdg["solid_velocity"], out=rhs)
    x0 = torch.empty_like(rhs)
    lv.gather_velocity(vdg["u"], vdg["v"], vdg["w"], out=x0)
    s = simd_viscosity3d(lv)
    prof = s.profile_pcg(x0.clone(), rhs, 1e-6)
    levels = lv.num_levels()
    ndof = [lv.num_dof(l) for l in range(levels)]
    ndof_c = []
    for l in range(levels):
        _, m = lv.topology(l)
        ndof_c.append([int(sum(bin(int(w)).count("1") for w in m[c].reshape(-1))) for c in range(3)])
    # The dominant kernel is the red/black GS pass (k_vapply_seq on levels 0-1, fused k_vrbgs steps below);
    # the roofline is quoted on the level-0 red pass of channel 0 (the launch
    # the committed ncu capture measures), the all-level aggregate beside it.
    gs = [(k, v) for k, v in prof.items() if " red_gs " in k or " black_gs " in k or " rbgs step " in k]
    gs_bytes = sum(_visc_pass_bytes(k, ndof, ndof_c) * v[1] for k, v in gs)
    gs_ms = sum(v[0] for k, v in gs)
    prof_ms = sum(v[0] for v in prof.values())
    dom_label = "L0 red_gs c0"
    dom_bytes = _visc_pass_bytes(dom_label, ndof, ndof_c)
    l0 = [(k, v) for k, v in gs if k.startswith("L0 ")]
    l0_bytes = sum(_visc_pass_bytes(k, ndof, ndof_c) * v[1] for k, v in l0)
    l0_ms = sum(v[0] for k, v in l0)
    peak, peak_kind = _peaks()
    t_ms, cnt = prof.get(dom_label, (0.0, 0))
    achieved = dom_bytes / (t_ms / cnt * 1e-3) / 1e9 if (dom_bytes and cnt) else None
    vec_bytes = 3 * 4 * 512 * n0
    out = {"workload": VISC_WORKLOAD, "value": round(value, 4), "unit": UNIT,
           "e2e": {"value": round(e2e, 4), "unit": UNIT,
                   # create: viscosity, liquid SDF (+mask), solid SDF; solve: the three velocity channels and the
                   # solid velocity, once
                   "h2d_bytes_per_step": int(_grid_bytes(vsc.viscosity, vsc.liquid_phi, vsc.solid_phi)
                                             + _grid_bytes(vsc.u, vsc.v, vsc.w, vsc.solid_velocity)),
                   "d2h_bytes_per_step": int(vec_bytes)},
           "ndof": ndof, "ndof_per_channel_l0": ndof_c[0], "levels": levels, "pcg_iterations": viters[0],
           "status": "SUCCESS" if all(x == 0 for x in vstatus) else "FAILED",
           "step": "create viscosity matrix+hierarchy, rhs, warm start, UAAMG-PCG",
           "solves_per_s": round(1e3 / value, 2),
           "roofline": {"bound": "hbm",
                        "kernel": f"k_vapply_seq<RED_GS> level 0, channel 0 ({n0} leaves over 3 CTAs per SM)",
                        "achieved": round(achieved, 1) if achieved else None, "peak": peak,
                        "peak_kind": peak_kind, "unit": "GB/s",
                        "frac": round(achieved / peak, 4) if achieved else None,
                        "traffic": _traffic_from_profile("k_vapply_seq<3>"), "algorithmic_bytes_per_launch": dom_bytes,
                        "avg_launch_us": round(t_ms / cnt * 1e3, 2) if cnt else None,
                        "level0_rbgs_GBps": round(l0_bytes / (l0_ms * 1e-3) / 1e9, 1) if l0_ms else None,
                        "all_levels_rbgs_GBps": round(gs_bytes / (gs_ms * 1e-3) / 1e9, 1) if gs_ms else None,
                        "rbgs_share_of_solve": round(gs_ms / prof_ms, 3) if prof_ms else None},
           "kernel_profile_ms": {k: [round(v[0], 4), v[1]] for k, v in sorted(prof.items(), key=lambda kv: -kv[1][0])},
           "_launches": int(launches)}
    if rank == 0 and not args.no_cpu_baseline and ws == 1:
        out["cpu_baseline"] = cpu_baseline(cpu_visc_solve_once, vsc,
                                           "oracle/viscosity_oracle.c (build+rhs+warm start+PCG)",
                                           budget_s=20.0, min_samples=2, max_samples=10)
    return out


BATCH_WORKLOAD = ("batched Poisson: instance i = cubic box of side from {32,64,96,128,192} (seed i), 1-6 spheres "
                  "with radii log-uniform [0.05,0.3] and centres uniform in the box, walls solid, U[-1,1] face "
                  "velocities seed i, rel-res 1e-7, zero initial guess")


def run_batched(args, dev, stream, timed, max_over_ranks, ws):
    """All instances in one batched graph launch vs the same instances solved
    one after another through the plain API (each handle with its own graph).
    Hierarchies and right-hand sides are built once, outside the timed region
    (they stay resident, as in a serving loop); a step resets the initial
    guesses to zero and solves every instance."""
    import torch
    from uaamg_b200 import scenes
    from uaamg_b200.batch import PoissonBatch
    from uaamg_b200.poisson import LaplacianWithLevel, PoissonSolver
    t0 = time.perf_counter()
    laps, solvers, rhss, xs = [], [], [], []
    sides = []
    for i in range(args.batch):
        sc = scenes.random_balls_scene(i)
        sides.append(sc.n)
        lap = LaplacianWithLevel.createPressurePoissonLaplacian(sc.phi, sc.face_weights, sc.dt, sc.dx)
        n = lap.leaf_count(0)
        r = torch.empty((n, 512), dtype=torch.float32, device=dev)
        lap.createPressurePoissonRightHandSide(sc.face_weights, sc.vx, sc.vy, sc.vz, sc.solid_velocity, sc.dt,
                                              out=r)
        laps.append(lap)
        solvers.append(PoissonSolver(lap))
        rhss.append(r)
        xs.append(torch.zeros_like(r))
    torch.cuda.synchronize()
    setup_s = time.perf_counter() - t0
    batch = PoissonBatch(solvers)
    batch.set_stream(stream.cuda_stream)
    for s_ in solvers:
        s_.set_stream(stream.cuda_stream)
    ndof = [lap.num_dof(0) for lap in laps]
    levels = [lap.num_levels() for lap in laps]
    launches = {"batch": 0, "plain": 0}

    def step_batch():
        torch._foreach_zero_(xs)
        batch.solveMultigridPCG(xs, rhss)
        launches["batch"] += batch.kernel_launches

    def step_plain():
        torch._foreach_zero_(xs)
        for s_, x, r in zip(solvers, xs, rhss):
            s_.solveMultigridPCG(x, r)

    for _ in range(args.warmup):
        step_plain()
    plain_iters = list(s_.mIterationTaken for s_ in solvers)
    plain_x = [x.clone() for x in xs]
    for _ in range(args.warmup):
        step_batch()
    same = all(torch.equal(a, b) for a, b in zip(plain_x, xs)) and batch.mIterationTaken == plain_iters
    steps = max(2, min(args.steps, 5))
    launches.update(batch=0, plain=0)
    t_b = timed(step_batch, steps)
    base = sum(s_.kernel_launches for s_ in solvers)
    t_p = timed(step_plain, steps)
    launches["plain"] = sum(s_.kernel_launches for s_ in solvers) - base
    t_b, t_p = max_over_ranks(t_b, t_p)
    ms_b, ms_p = t_b / steps, t_p / steps
    n = args.batch
    return {
        "workload": BATCH_WORKLOAD, "instances": n, "sides": sorted(sides), "total_dof": int(sum(ndof)),
        "levels": [min(levels), max(levels)], "iterations": [min(plain_iters), max(plain_iters)],
        "status": "SUCCESS" if all(v == 0 for v in batch.status) else "FAILED",
        "ms_per_batch": round(ms_b, 3), "ms_per_solve": round(ms_b / n, 4), "solves_per_s": round(n * 1e3 / ms_b, 1),
        "plain_sequential": {"ms_per_batch": round(ms_p, 3), "ms_per_solve": round(ms_p / n, 4),
                             "solves_per_s": round(n * 1e3 / ms_p, 1)},
        "speedup_vs_plain": round(ms_p / ms_b, 3),
        "identical_to_plain": bool(same),
        "dof_updates_per_s": round(sum(d * (it + 1) for d, it in zip(ndof, plain_iters)) * 1e3 / ms_b, 1),
        "setup_s_host_wall": round(setup_s, 2),
        "step": "zero initial guesses, solve every instance to rel-res 1e-7 (hierarchies and rhs resident)",
        "gpu_launches_per_batch": int(launches["batch"] // steps),
        "_launches": int(launches["batch"] + launches["plain"]),
    }


MIXED_WORKLOAD = ("mixed-precision large Poisson: {n}^3, dx = 1/{n}, liquid y<0.45 + 4 spheres r0.1 (seed 2), walls "
                  "solid, U[-1,1] face velocities (seed 2), rel-res 1e-7, zero initial guess")


def run_mixed(args, dev, stream, timed, max_over_ranks, ws):
    """One large Poisson system solved by the FP32 UAAMG-PCG and by the
    mixed-precision form (FP16 and BF16 hierarchy storage, FP32 arithmetic and
    outer CG, FP64 dots, residual replacement every 25 iterations, FP64
    coarsest solve).  The hierarchy and rhs are built once (setup, reported
    apart); a step resets the initial guess to zero and solves.  Accuracy: the
    FP64 true relative residual |b - A x|_inf / |b|_inf of every solution, and
    the relative 2-norm difference of each mixed solution to the FP32 one."""
    import torch
    from uaamg_b200 import scenes
    from uaamg_b200.poisson import LaplacianWithLevel, PoissonSolver
    n = args.mixed_n
    t0 = time.perf_counter()
    with torch.cuda.stream(stream):
        phi, fw, vx, vy, vz, sv, dt, dx = scenes.device_large_poisson(n, 2, dev)
    stream.synchronize()
    lap = LaplacianWithLevel.createPressurePoissonLaplacian(phi, fw, dt, dx, stream=stream.cuda_stream)
    nl = lap.leaf_count(0)
    rhs = torch.empty((nl, 512), dtype=torch.float32, device=dev)
    lap.createPressurePoissonRightHandSide(fw, vx, vy, vz, sv, dt, out=rhs)
    del phi, fw, vx, vy, vz
    solver = PoissonSolver(lap)
    solver.set_stream(stream.cuda_stream)
    torch.cuda.synchronize()
    setup_s = time.perf_counter() - t0
    x = torch.zeros_like(rhs)
    out = {"workload": MIXED_WORKLOAD.format(n=n), "ndof": [lap.num_dof(l) for l in range(lap.num_levels())],
           "hierarchy_setup_s_host_wall": round(setup_s, 3)}
    steps = max(2, min(args.steps, 5))
    launches = 0
    sols = {}
    for form in ("fp32", "fp16", "bf16"):
        if form == "fp32":
            fn = lambda: solver.solveMultigridPCG(x, rhs)  # noqa: E731
            setup_ms = 0.0
        else:
            setup_ms = solver.prepare_mixed(form)
            fn = lambda f=form: solver.solveMultigridPCGMixed(x, rhs, f)  # noqa: E731
        for _ in range(args.warmup):
            x.zero_()
            fn()
        base = solver.kernel_launches

        def step():
            x.zero_()
            fn()

        t = timed(step, steps)
        launches += solver.kernel_launches - base
        (t,) = max_over_ranks(t)
        x.zero_()
        st = fn()
        rmax, bmax = solver.true_residual_fp64(x, rhs)
        sols[form] = x.clone()
        out[form] = {"ms_per_solve": round(t / steps, 3), "solves_per_s": round(steps * 1e3 / t, 2),
                     "iterations": solver.mIterationTaken, "status": "SUCCESS" if st == 0 else "FAILED",
                     "true_rel_residual_fp64": rmax / bmax if bmax > 0 else 0.0}
        if form != "fp32":
            out[form]["setup_ms"] = round(setup_ms, 1)
    for form in ("fp16", "bf16"):
        d = torch.linalg.vector_norm((sols[form] - sols["fp32"]).double())
        out[form]["rel_diff_vs_fp32"] = float(d / torch.linalg.vector_norm(sols["fp32"].double()))
        out[form]["speedup_vs_fp32"] = round(out["fp32"]["ms_per_solve"] / out[form]["ms_per_solve"], 3)
    # every form's error against the FP64 reference solution of the same system (flexible FP64 PCG to a true
    # relative 2-norm residual of 1e-12, uaamg_poisson_solve_fp64_reference)
    x64 = torch.empty(rhs.shape, dtype=torch.float64, device=dev)
    t0 = time.perf_counter()
    st64, it64, res64 = solver.solve_fp64_reference(rhs, x64, 1e-12, 200)
    torch.cuda.synchronize()
    out["fp64_reference"] = {"status": "SUCCESS" if st64 == 0 else "FAILED", "iterations": it64,
                             "true_rel_residual_2norm": res64, "s_host_wall": round(time.perf_counter() - t0, 3),
                             "method": "flexible FP64 PCG on the FP32-assembled level-0 matrix, FP32 W-cycle "
                                       "preconditioner on the scaled residual, stop at |b-Ax|_2 <= 1e-12 |b|_2"}
    n64 = torch.linalg.vector_norm(x64)
    for form in ("fp32", "fp16", "bf16"):
        out[form]["rel_err_vs_fp64"] = float(torch.linalg.vector_norm(sols[form].double() - x64) / n64)
    del x64
    out["step"] = "zero initial guess, solve to rel-res 1e-7 (hierarchy, rhs resident)"
    out["_launches"] = int(launches)
    del lap, solver, sols
    torch.cuda.empty_cache()
    return out


SERVE_WORKLOAD = ("served stream: Poisson arrivals 200/s and viscosity arrivals 50/s (Poisson process), sides "
                  "log-uniform in [48,384] voxels, geometry as the batched workload (seeded per request), 1-24 "
                  "substeps with new face velocities each, pressure warm-started across substeps, hierarchies "
                  "resident, admission by HBM budget")


def run_projection(args, dev, stream, timed, max_over_ranks, ws, rank):
    """The steps either side of the pressure solve on the plain Poisson
    workload (128^3): the solid face weights on the liquid's dilated topology
    (walls 1.5 voxels thick and a sphere obstacle of radius n/8 as the solid
    SDF), the liquid SDF immersed in the solid, the pressure-gradient update of
    the three velocity channels with the solved pressure, and the velocity
    extrapolation after it.  Inputs device-resident, L2 flushed before each step;
    the CPU oracle (OpenMP) is timed on the same inputs."""
    import ctypes as C
    import torch
    from uaamg_b200 import _lib, scenes
    from uaamg_b200.grids import LeafGrid, dense_to_leaves
    from uaamg_b200.poisson import LaplacianWithLevel, PoissonSolver, _as_c
    from uaamg_b200.projection import face_weight_topology
    sc = scenes.plain_poisson_scene(n=args.n, seed=0)
    n, dx = sc.n, sc.dx
    lo, size = -8, n + 16
    c = np.arange(size, dtype=np.float64) + lo
    X, Y, Z = np.meshgrid(c, c, c, indexing="ij")
    wall = np.minimum.reduce([X - 1.5, n - 1.5 - X, Y - 1.5, n - 1.5 - Y, Z - 1.5, n - 1.5 - Z])
    sph = np.sqrt((X - n / 2) ** 2 + (Y - n / 4) ** 2 + (Z - n / 2) ** 2) - n / 8
    solid = dense_to_leaves((np.minimum(wall, sph) * dx).astype(np.float32), origin=(lo, lo, lo),
                            background=-3.0 * dx)
    del X, Y, Z, wall, sph
    origins, masks = face_weight_topology(sc.phi)
    nfw = origins.shape[0]
    keep = []

    def dev_grid(g):
        d = LeafGrid(origins=g.origins, values=g.values, background=g.background, masks=g.masks)
        d.values = torch.from_numpy(np.ascontiguousarray(g.values)).to(dev)
        return d

    solid_d = dev_grid(solid)
    gs = _as_c(solid_d, keep)
    w_d = torch.empty((nfw, 512, 3), dtype=torch.float32, device=dev)
    L = _lib.lib()

    def fw_step():
        _lib.check(L.uaamg_face_weights_device(C.byref(gs), nfw, origins.ctypes.data, masks.ctypes.data,
                                               w_d.data_ptr(), C.c_void_p(stream.cuda_stream)), "face_weights")

    for _ in range(args.warmup):
        fw_step()
    t_fw = timed(fw_step, args.steps)
    torch.cuda.synchronize()

    # the liquid SDF immersed in the solid (FLIP_vdb.cpp:2856-2942): both value passes on the device, liquid and
    # solid resident
    liq_d = dev_grid(sc.phi)
    gl = _as_c(liq_d, keep)
    im_out = torch.empty((sc.phi.leaf_count, 512), dtype=torch.float32, device=dev)

    def im_step():
        _lib.check(L.uaamg_immerse_liquid_phi_device(C.byref(gs), C.byref(gl), float(dx), im_out.data_ptr(),
                                                     C.c_void_p(stream.cuda_stream)), "immerse_liquid_phi")

    for _ in range(args.warmup):
        im_step()
    t_im = timed(im_step, args.steps)
    torch.cuda.synchronize()
    fw = LeafGrid(origins=origins, values=w_d.cpu().numpy(), background=np.ones(3, np.float32), masks=masks)
    fw_d = dev_grid(fw)
    phi_d = dev_grid(sc.phi)
    lap = LaplacianWithLevel.createPressurePoissonLaplacian(phi_d, fw_d, sc.dt, sc.dx, stream=stream.cuda_stream)
    rhs = torch.empty((lap.leaf_count(0), 512), dtype=torch.float32, device=dev)
    lap.createPressurePoissonRightHandSide(fw_d, dev_grid(sc.vx), dev_grid(sc.vy), dev_grid(sc.vz),
                                          sc.solid_velocity, sc.dt, out=rhs)
    solver = PoissonSolver(lap)
    solver.set_stream(stream.cuda_stream)
    p = torch.zeros_like(rhs)
    st = solver.solveMultigridPCG(p, rhs)
    m = n + 1
    sv = dense_to_leaves(np.random.default_rng(11).uniform(-1, 1, (m, m, m, 3)).astype(np.float32),
                         background=np.zeros(3, np.float32))
    sv_d = dev_grid(sv)
    vels = [sc.vx, sc.vy, sc.vz]
    vin = [torch.from_numpy(np.ascontiguousarray(v.values)).to(dev) for v in vels]
    vwork = [x.clone() for x in vin]
    nv = [v.leaf_count for v in vels]
    mk = [torch.empty(k * 8, dtype=torch.int64, device=dev) for k in nv]
    up = [torch.empty_like(x) for x in vin]
    rf = [torch.empty_like(x) for x in vin]
    gphi, gfw, gsv = _as_c(phi_d, keep), _as_c(fw_d, keep), _as_c(sv_d, keep)
    gv = [_as_c(v, keep) for v in vels]
    friction = 0.5

    def pg_step():
        for ch in range(3):
            vwork[ch].copy_(vin[ch])
            _lib.check(L.uaamg_poisson_apply_pressure_gradient_device(
                lap._h, C.byref(gphi), C.byref(gfw), C.byref(gsv), p.data_ptr(), float(sc.dt), friction, ch,
                C.byref(gv[ch]), vwork[ch].data_ptr(), mk[ch].data_ptr(), up[ch].data_ptr(), rf[ch].data_ptr()),
                "apply_pressure_gradient")

    for _ in range(args.warmup):
        pg_step()
    t_pg = timed(pg_step, args.steps)
    torch.cuda.synchronize()

    # velocity extrapolation after the gradient update (FLIP_vdb.cpp:2379): the updated voxels of each channel
    # extrapolated 3 layers into the liquid SDF's topology; the topology set operations run on the host (timed
    # apart), the layers on the device with the channel values and masks resident
    from uaamg_b200.extrapolate import prepare_channel, run_layers_device, topology_of
    import time as _time
    n_layer = 3
    target = topology_of(sc.phi)
    ex_in = [LeafGrid(origins=vels[ch].origins, values=vwork[ch].cpu().numpy(), background=vels[ch].background,
                      masks=mk[ch].cpu().numpy().view(np.uint64).reshape(-1, 8).copy()) for ch in range(3)]
    tp0 = _time.perf_counter()
    preps = [prepare_channel(g, target) for g in ex_in]
    prep_ms = (_time.perf_counter() - tp0) * 1e3
    xv_in = [torch.from_numpy(pr[1]).to(dev) for pr in preps]
    xm_in = [torch.from_numpy(pr[2].view(np.int64)).to(dev) for pr in preps]
    xv, xm = [x.clone() for x in xv_in], [x.clone() for x in xm_in]

    def ex_step():
        for ch in range(3):
            xv[ch].copy_(xv_in[ch])
            xm[ch].copy_(xm_in[ch])
            org, _, _, fl, fm = preps[ch]
            run_layers_device(n_layer, org, xv[ch], xm[ch], fl, fm, stream=stream.cuda_stream)

    for _ in range(args.warmup):
        ex_step()
    t_ex = timed(ex_step, args.steps)
    t_fw, t_pg, t_ex, t_im = max_over_ranks(t_fw, t_pg, t_ex, t_im)
    fw_ms, pg_ms, ex_ms, im_ms = t_fw / args.steps, t_pg / args.steps, t_ex / args.steps, t_im / args.steps
    ex_fill = int(sum(int(np.unpackbits(pr[4].view(np.uint8)).sum()) for pr in preps))
    ex_leaves = int(sum(pr[0].shape[0] for pr in preps))
    ex_filled = int(sum(int(np.unpackbits(xm[ch].cpu().numpy().view(np.uint8)).sum())
                        - int(np.unpackbits(preps[ch][2].view(np.uint8)).sum()) for ch in range(3)))
    fw_vox = int(np.unpackbits(masks.view(np.uint8)).sum())
    v_vox = int(sum(k * 512 for k in nv))
    # algorithmic bytes: face weights read the solid SDF once per voxel (4 B) and write 3 weights (12 B); the
    # gradient update reads u, w, phi, p (two cells each for phi and p) and the solid velocity and writes u, the
    # update, the reflected value and the mask (36 B per velocity voxel, the copy of u included)
    out = {"workload": f"projection steps on the plain Poisson workload {n}^3: face weights on the liquid SDF "
                       f"dilated by 2 voxels (solid = walls + sphere r=n/8), the liquid SDF immersed in the solid, "
                       f"pressure-gradient update of the 3 velocity channels (friction {friction}), velocity "
                       f"extrapolation ({n_layer} layers into the liquid SDF topology)",
           "face_weights": {"ms": round(fw_ms, 4), "voxels": fw_vox, "leaves": nfw,
                            "GBps_algorithmic": round(16.0 * nfw * 512 / (fw_ms * 1e-3) / 1e9, 1)},
           "immerse_liquid_phi": {"ms": round(im_ms, 4), "voxels": int(sc.phi.leaf_count * 512),
                                  "leaves": int(sc.phi.leaf_count),
                                  "note": "both value passes (2 launches); the two topology dilations are host work"},
           "pressure_gradient": {"ms_3_channels": round(pg_ms, 4), "voxels": v_vox, "solve_status": int(st),
                                 "GBps_algorithmic": round(36.0 * v_vox / (pg_ms * 1e-3) / 1e9, 1)},
           "extrapolation": {"ms_3_channels": round(ex_ms, 4), "layers": n_layer,
                             "target": "liquid SDF active voxels", "fill_set_voxels": ex_fill,
                             "voxels_filled": ex_filled, "fill_leaves": int(sum(pr[3].size for pr in preps)),
                             "output_leaves": ex_leaves, "host_topology_ms": round(prep_ms, 2),
                             "note": "per channel: upload of the fill set and leaf map, 3 layer launches"},
           "l2": "flushed before every timed step (256 MiB write)"}
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:  # the oracle as the timed CPU baseline
        import os
        import time as _t
        from oracle import oracle as orc
        pc = p.cpu().numpy()
        ref = orc.OraclePoisson(sc.phi, fw, sc.dt, sc.dx, hierarchy=False)
        po, pm = ref.topology(0)
        t0 = _t.perf_counter()
        orc.face_weights(solid, origins, masks)
        t1 = _t.perf_counter()
        orc.immerse_liquid_phi(sc.phi, solid, dx)
        t_imm = (_t.perf_counter() - t1) * 1e3
        t1 = _t.perf_counter()
        for ch in range(3):
            orc.pressure_gradient(sc.phi, fw, sv, po, pm, pc, sc.dt, sc.dx, friction, ch, vels[ch])
        t2 = _t.perf_counter()
        for pr in preps:
            orc.extrapolate_channel(n_layer, *pr)
        t3 = _t.perf_counter()
        out["cpu_oracle_ms"] = {"face_weights": round((t1 - t0) * 1e3, 2), "immerse_liquid_phi": round(t_imm, 2),
                                "pressure_gradient_3_channels": round((t2 - t1) * 1e3, 2),
                                "extrapolation_3_channels": round((t3 - t2) * 1e3, 2),
                                "threads": os.cpu_count()}
    out["_launches"] = (6 + 3 * n_layer) * args.steps
    return out


def run_served(args, ws):
    """The served stream through the native server (uaamg_server_*): requests
    are submitted at their arrival times; each simulation pushes its next
    substep's face velocities once its previous substep is solved (a closed
    loop, as a FLIP substep needs the previous solution), so requests arrive
    and progress while others are being served.  Batched (pressure rounds in
    one graph) vs plain (every pressure solve alone); viscosity requests run
    on lanes of their own in both.  Latency: arrival to the last substep.
    Every pressure result carries its FP64 relative residual."""
    import torch
    from uaamg_b200 import scenes
    from uaamg_b200.serve import make_stream
    from uaamg_b200.server import NativeServer
    dev = torch.device("cuda", torch.cuda.current_device())
    free, _ = torch.cuda.mem_get_info()
    out = {"workload": SERVE_WORKLOAD, "window_s": args.serve_window, "server": "native (uaamg_server_*)"}
    for mode in ("batched", "plain"):
        reqs = make_stream(args.serve_window, seed=4)
        srv = NativeServer(batching=(mode == "batched"), budget_bytes=int(0.5 * free))
        t0 = time.perf_counter()
        pending = sorted(reqs, key=lambda r: r.arrival)
        live = []  # [request, server id, next substep to push, substeps waited]
        lat, res64, it_p, stat_ok, solves = [], [], [], True, 0
        by_kind = {"poisson": [], "viscosity": []}
        while pending or live:
            now = time.perf_counter() - t0
            if now > args.serve_limit:
                break
            while pending and pending[0].arrival <= now:
                r = pending.pop(0)
                if r.kind == "poisson":
                    phi, fw, sv, dt, dx = scenes.device_poisson_instance(r.side, r.seed, dev)
                    rid = srv.submit_poisson(phi, fw, sv, dt, dx, r.substeps)
                else:
                    liq, sol, mu, sv, dt, rho, dx = scenes.device_viscosity_instance(r.side, r.seed, dev)
                    rid = srv.submit_viscosity(mu, liq, sol, sv, dt, rho, dx, r.substeps)
                srv.push_velocity(rid, *scenes.device_face_velocities(r.side, r.seed * 1000003, dev))
                live.append([r, rid, 1, 0])
            progressed = False
            for e in list(live):
                r, rid, nxt, got = e
                try:
                    w = srv.wait(rid, got, 0.0)
                except Exception:
                    continue  # not solved yet
                progressed = True
                e[3] = got = got + 1
                solves += 1
                stat_ok &= w["status"] == 0
                if r.kind == "poisson":
                    res64.append(w["fp64_residual"])
                    it_p.append(w["iterations"])
                if nxt < r.substeps:
                    srv.push_velocity(rid, *scenes.device_face_velocities(r.side, r.seed * 1000003 + nxt, dev))
                    e[2] = nxt + 1
                if got == r.substeps:
                    live.remove(e)
                    lat.append(w["latency_s"])
                    by_kind[r.kind].append(w["latency_s"])
            if not progressed:
                time.sleep(0.0005)
        elapsed = time.perf_counter() - t0
        st = srv.stats()
        srv.close()
        torch.cuda.synchronize()

        def pct(a, q):
            return round(float(np.percentile(np.array(a), q)) * 1e3, 2) if a else None

        out[mode] = {"requests": len(reqs), "completed": st["done"], "solves": solves, "elapsed_s": round(elapsed, 3),
                     "solves_per_s": round(solves / elapsed, 1), "p50_ms": pct(lat, 50), "p99_ms": pct(lat, 99),
                     "by_kind": {k: {"completed": len(v), "p50_ms": pct(v, 50), "p99_ms": pct(v, 99)}
                                 for k, v in by_kind.items()},
                     "pressure_rounds": st["rounds"], "batch_graphs_built": st["batch_builds"],
                     # what batching changes: pressure solves per second of pressure rounds (the rounds share the
                     # GPU with the viscosity lanes in both forms)
                     "pressure_solves_per_busy_s": round(st["pressure_solves"] / (st["pressure_busy_us"] * 1e-6), 1)
                     if st["pressure_busy_us"] else None,
                     "peak_budget_GB": round(st["peak_bytes"] / 1e9, 2), "all_status_success": bool(stat_ok),
                     "pressure_fp64_rel_residual_max": max(res64) if res64 else None,
                     "pressure_iterations_mean": round(float(np.mean(it_p)), 2) if it_p else None}
        del srv
    b, p = out["batched"], out["plain"]
    out["solves_per_s_vs_plain"] = round(b["solves_per_s"] / p["solves_per_s"], 3) if p["solves_per_s"] else None
    if b.get("pressure_solves_per_busy_s") and p.get("pressure_solves_per_busy_s"):
        out["pressure_round_throughput_vs_plain"] = round(b["pressure_solves_per_busy_s"] /
                                                          p["pressure_solves_per_busy_s"], 3)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=128)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-viscosity", action="store_true", help="skip the secondary viscosity measurement")
    ap.add_argument("--no-projection", action="store_true",
                    help="skip the face-weight and pressure-gradient measurement")
    ap.add_argument("--batch", type=int, default=64, help="instances of the batched Poisson measurement (0 = skip)")
    ap.add_argument("--mixed-n", type=int, default=512, help="domain side of the mixed-precision measurement (0 = skip)")
    ap.add_argument("--serve-window", type=float, default=0.2,
                    help="seconds of arrivals of the served request stream (0 = skip)")
    ap.add_argument("--serve-limit", type=float, default=60.0, help="time limit of each served run (s)")
    ap.add_argument("--no-graph", action="store_true", help="host-driven PCG loop instead of the CUDA graph")
    ap.add_argument("--profile", choices=["solve", "sweep", "vsolve", "vbuild", "large"], default=None,
                    help="short fixed sequence for ncu: 'vsolve' = viscosity build + 2 solves, 'vbuild' = "
                         "3 viscosity matrix + hierarchy builds, "
                         "'solve' = Poisson build + 2 graph solves, 'sweep' = Poisson build + 3 level-0 sweeps, "
                         "'large' = the mixed-precision workload at --mixed-n, one host-driven solve in "
                         "--profile-form")
    ap.add_argument("--profile-form", choices=["fp32", "fp16", "bf16"], default="fp32",
                    help="precision of the 'large' profile solve")
    ap.add_argument("--profile-events", action="store_true",
                    help="'large' profile: time every kernel of the solve with CUDA event pairs and print the "
                         "per-kernel-class table (ms, launches) as JSON")
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
    from uaamg_b200.viscosity import L_with_level, simd_viscosity3d

    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream(dev)
    # the autotuner's kernel-shape table for this GPU, when one is committed (results do not depend on it)
    from uaamg_b200 import autotune
    tuning_table = autotune.apply(device=local)
    tuning = {"setting": autotune.get(),
              "source": os.path.relpath(autotune.table_path(tuning_table["gpu"], tuning_table["sm_count"]), ROOT)
              if tuning_table else "built-in defaults"}

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

    if args.profile == "large":
        with torch.cuda.stream(stream):
            phi, fw, vx, vy, vz, sv, dt, dx = scenes.device_large_poisson(args.mixed_n, 2, dev)
        stream.synchronize()
        lap = LaplacianWithLevel.createPressurePoissonLaplacian(phi, fw, dt, dx, stream=stream.cuda_stream)
        rhs = torch.empty((lap.leaf_count(0), 512), dtype=torch.float32, device=dev)
        lap.createPressurePoissonRightHandSide(fw, vx, vy, vz, sv, dt, out=rhs)
        del phi, fw, vx, vy, vz
        torch.cuda.synchronize()
        solver = PoissonSolver(lap)
        solver.use_graph = 0
        p = torch.zeros_like(rhs)
        out = {"profile": "large", "form": args.profile_form, "n": args.mixed_n,
               "leaves": [lap.leaf_count(l) for l in range(lap.num_levels())]}
        if args.profile_form != "fp32":
            solver.prepare_mixed(args.profile_form)
        if args.profile_events:
            for _ in range(2):  # the second run is reported
                p.zero_()
                if args.profile_form == "fp32":
                    table = solver.profile_pcg(p, rhs)
                else:
                    table = solver.profile_pcg_mixed(p, rhs, args.profile_form)
            out["kernel_ms"] = {k: [round(v[0], 4), v[1]]
                                for k, v in sorted(table.items(), key=lambda kv: -kv[1][0])}
            out["total_ms"] = round(sum(v[0] for v in table.values()), 3)
        elif args.profile_form == "fp32":
            solver.solveMultigridPCG(p, rhs)
        else:
            solver.solveMultigridPCGMixed(p, rhs, args.profile_form)
        out["iterations"] = solver.mIterationTaken
        print(json.dumps(out))
        return

    vsc = scenes.plain_viscosity_scene(n=args.n, seed=1)
    vkeys = ("liquid_phi", "solid_phi", "viscosity", "u", "v", "w", "solid_velocity")
    vdg = {k: on_device(getattr(vsc, k)) for k in vkeys}

    if args.profile == "vbuild":
        for _ in range(3):
            lv = L_with_level.create_viscosity_matrix(vdg["viscosity"], vdg["liquid_phi"], vdg["solid_phi"], vsc.dt,
                                                      vsc.rho, vsc.dx)
            torch.cuda.synchronize()
            del lv
        print(json.dumps({"profile": "vbuild", "builds": 3}))
        return

    if args.profile == "vsolve":
        lv = L_with_level.create_viscosity_matrix(vdg["viscosity"], vdg["liquid_phi"], vdg["solid_phi"], vsc.dt,
                                                  vsc.rho, vsc.dx)
        rhs = torch.empty((3, lv.leaf_count(0), 512), dtype=torch.float32, device=dev)
        lv.build_rhs(vdg["u"], vdg["v"], vdg["w"], vdg["solid_velocity"], out=rhs)
        x0 = torch.empty_like(rhs)
        lv.gather_velocity(vdg["u"], vdg["v"], vdg["w"], out=x0)
        s = simd_viscosity3d(lv)
        s.use_graph = 0 if args.no_graph else 1
        for _ in range(2):
            x = x0.clone()
            st = s.pcg_solve(x, 1e-6, rhs)
        print(json.dumps({"profile": "vsolve", "status": st, "iterations": s.m_iteration}))
        return

    psc = scenes.plain_poisson_scene(n=args.n, seed=0)
    pkeys = ("phi", "face_weights", "vx", "vy", "vz", "solid_velocity")
    pdg = {k: on_device(getattr(psc, k)) for k in pkeys}
    if args.profile:
        lap = LaplacianWithLevel.createPressurePoissonLaplacian(pdg["phi"], pdg["face_weights"], psc.dt, psc.dx)
        rhs = torch.empty((lap.leaf_count(0), 512), dtype=torch.float32, device=dev)
        lap.createPressurePoissonRightHandSide(pdg["face_weights"], pdg["vx"], pdg["vy"], pdg["vz"],
                                              pdg["solid_velocity"], psc.dt, out=rhs)
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

    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    step_log: dict[str, list[float]] = {}

    def timed(fn, steps, name=None):
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        total = 0.0
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        each = []
        for _ in range(steps):
            flush.fill_(1.0)  # evict L2 between timed steps (256 MiB > 126 MB L2)
            torch.cuda.synchronize()
            e0.record(stream)
            fn()
            e1.record(stream)
            torch.cuda.synchronize()
            each.append(e0.elapsed_time(e1))
            total += each[-1]
        if name:
            step_log[name] = each
        if dist is not None:
            dist.barrier()
        return total

    def max_over_ranks(*vals):
        if dist is None:
            return vals
        tt = torch.tensor(vals, dtype=torch.float64, device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        return tuple(float(v) for v in tt)

    # ================= headline: plain pressure Poisson (the metric's configuration) =================
    pstats = {"launches": 0, "iters": [], "status": []}

    def pstep_device():
        # createPressurePoissonLaplacian + PoissonSolver + createPressurePoissonRightHandSide in one call
        # (device-resident grids), then solveMultigridPCG from a zero pressure
        lap = LaplacianWithLevel.createPressurePoissonLaplacianWithRhs(
            pdg["phi"], pdg["face_weights"], pdg["vx"], pdg["vy"], pdg["vz"], pdg["solid_velocity"], psc.dt,
            psc.dx, stream=stream.cuda_stream)
        solver = PoissonSolver(lap)
        p = torch.empty((lap.leaf_count(0), 512), dtype=torch.float32, device=dev)
        st = solver.solveMultigridPCGResident(p)
        pstats["launches"] += solver.kernel_launches
        pstats["iters"].append(solver.mIterationTaken)
        pstats["status"].append(st)
        return lap, p

    phg = {k: pinned(getattr(psc, k)) for k in pkeys}
    phost = {}

    def pstep_host():
        # the same step through the host-pointer C ABI: the pinned input grids go up once each, the pressure
        # comes back to pinned host memory
        lap = LaplacianWithLevel.createPressurePoissonLaplacianWithRhs(
            phg["phi"], phg["face_weights"], phg["vx"], phg["vy"], phg["vz"], phg["solid_velocity"], psc.dt,
            psc.dx, stream=stream.cuda_stream)
        solver = PoissonSolver(lap)
        n = lap.leaf_count(0)
        if phost.get("n") != n:
            phost["p_t"] = torch.empty((n, 512), dtype=torch.float32).pin_memory()
            phost["p"], phost["n"] = phost["p_t"].numpy(), n
        st = solver.solveMultigridPCGResident(phost["p"])
        pstats["launches"] += solver.kernel_launches
        return lap, st

    for _ in range(args.warmup):
        pstep_device()
    pstats.update(launches=0, iters=[], status=[])
    clk = ClockSampler(local)
    clk.start()
    tp_dev = timed(pstep_device, args.steps, "device")
    clocks = clk.stop()
    launches = pstats["launches"]
    piters, pstatus = list(pstats["iters"]), list(pstats["status"])
    for _ in range(args.warmup):
        pstep_host()
    tp_host = timed(pstep_host, args.steps, "e2e")
    tp_dev, tp_host = max_over_ranks(tp_dev, tp_host)
    total = args.steps * ws
    value, e2e = tp_dev / total, tp_host / total

    # per-kernel device times of one solve (event pairs around every launch, host-driven loop) for the roofline
    lap, p_ref = pstep_device()
    solver = PoissonSolver(lap)
    rhs_d = lap.copy_rhs(torch.empty_like(p_ref))
    pprof = solver.profile_pcg(torch.zeros_like(rhs_d), rhs_d)
    pndof = [lap.num_dof(l) for l in range(lap.num_levels())]
    pleaves = [lap.leaf_count(l) for l in range(lap.num_levels())]
    pbytes = PoissonBytes(lap)
    peak, peak_kind = _peaks()
    prof_ms = sum(v[0] for v in pprof.values())
    # The dominant bandwidth kernel class: the most algorithmic bytes per solve.  (Event pairs around every launch
    # add each launch's latency, so ranking by event time would favour the many small coarse-level launches; the
    # ncu launch list, with device times, ranks the level-0 Jacobi sweep first among the bandwidth kernels.)
    ranked = sorted(((k, v) for k, v in pprof.items() if pbytes.launch_bytes(k) is not None),
                    key=lambda kv: -pbytes.launch_bytes(kv[0]) * kv[1][1])
    top_label, (top_ms, top_cnt) = max(pprof.items(), key=lambda kv: kv[1][0])
    dom_label, (dom_ms, dom_cnt) = ranked[0]
    dom_bytes = pbytes.launch_bytes(dom_label)
    dom_us = dom_ms / dom_cnt * 1e3
    achieved = dom_bytes / (dom_us * 1e-6) / 1e9
    agg_bytes = sum(pbytes.launch_bytes(k) * v[1] for k, v in ranked)
    agg_ms = sum(v[0] for k, v in ranked)
    pvec = 4 * 512 * pleaves[0]
    pcpu = None
    if rank == 0 and not args.no_cpu_baseline and ws == 1:
        pcpu = cpu_baseline(cpu_solve_once, psc, "oracle/poisson_oracle.c (build+rhs+PCG)")

    # ================= secondary: plain variational viscosity =================
    viscosity = None
    if not args.no_viscosity:
        viscosity = run_viscosity(args, dev, stream, timed, max_over_ranks, ws, rank, vsc, vdg, pinned)
        launches += viscosity.pop("_launches")

    # ================= batched Poisson: many instances in one graph =================
    batched = None
    if args.batch > 0:
        batched = run_batched(args, dev, stream, timed, max_over_ranks, ws)

    # ================= mixed precision: large Poisson solve =================
    mixed = None
    if args.mixed_n > 0:
        mixed = run_mixed(args, dev, stream, timed, max_over_ranks, ws)

    # ================= the steps either side of the pressure solve =================
    projection = None
    if not args.no_projection:
        projection = run_projection(args, dev, stream, timed, max_over_ranks, ws, rank)

    # ================= served request stream (continuous batching) =================
    served = None
    if args.serve_window > 0:
        served = run_served(args, ws)

    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 4), "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(tp_dev / args.steps, 4), "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": poisson_config(args),
            "solve": {"ndof": pndof, "leaves": pleaves, "levels": len(pndof), "pcg_iterations": piters[0],
                      "status": "SUCCESS" if all(x == 0 for x in pstatus) else "FAILED",
                      "solves_per_s": round(1e3 / value, 2),
                      "voxel_updates_per_s": round(pndof[0] * piters[0] * 1e3 / value, 1),
                      "step": "create level-0 matrix + hierarchy + rhs (uaamg_poisson_create_with_rhs, device-"
                              "resident grids), then UAAMG-PCG from a zero pressure "
                              "(uaamg_poisson_solve_pcg_resident_device)",
                      # per-step spread (the step has host phases: topology, the first solve's host-driven loop)
                      "step_ms": {k: {"min": round(min(v), 4), "median": round(float(np.median(v)), 4),
                                      "max": round(max(v), 4)} for k, v in step_log.items()}},
            "e2e": {"value": round(e2e, 4), "unit": UNIT,
                    # uaamg_poisson_create_with_rhs from pinned grids: the liquid SDF whole, the face weights
                    # and the three velocity channels at the leaves the construction reads; the solid velocity
                    # grid is empty here
                    "h2d_bytes_per_step": _pressure_h2d_bytes(psc.phi, psc.face_weights,
                                                              (psc.vx, psc.vy, psc.vz, psc.solid_velocity)),
                    # the pressure
                    "d2h_bytes_per_step": int(pvec)},
            "gpu_launches": int(launches),
            "roofline": {"bound": "hbm", "kernel": f"{dom_label} ({pleaves[int(dom_label[1])]} leaves)",
                         "achieved": round(achieved, 1), "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                         "frac": round(achieved / peak, 4),
                         "traffic": _traffic_from_profile(pbytes.ncu_tag(dom_label, pleaves[int(dom_label[1])])),
                         "algorithmic_bytes_per_launch": round(dom_bytes),
                         "avg_launch_us": round(dom_us, 2), "launches": dom_cnt,
                         "share_of_solve": round(dom_ms / prof_ms, 3),
                         "all_bandwidth_kernels_GBps": round(agg_bytes / (agg_ms * 1e-3) / 1e9, 1),
                         "top_kernel_by_time": {"label": top_label, "share_of_solve": round(top_ms / prof_ms, 3),
                                                "avg_launch_us": round(top_ms / top_cnt * 1e3, 2)},
                         "note": "the bandwidth kernel class moving the most algorithmic bytes in one solve (the "
                                 "ncu launch list ranks it first of the bandwidth kernels by device time, "
                                 "profiles/poisson128_pcg_solve_launch_list.md); duration from CUDA event pairs "
                                 "around every launch of a host-driven solve (they include the launch latency); "
                                 "algorithmic bytes: every array the kernel must touch once per DOF at 4 B, "
                                 "coefficient arrays only where stored; traffic: ncu DRAM bytes of one launch of the "
                                 "same kernel on the same level; top_kernel_by_time may be a latency-bound one (the "
                                 "cluster bottom-cycle kernel with the coarsest CG)"},
            "tuning": tuning,
            "kernel_profile_ms": {k: [round(v[0], 4), v[1]] for k, v in sorted(pprof.items(), key=lambda kv: -kv[1][0])},
            "clocks": clocks,
        }
        if pcpu is not None:
            line["cpu_baseline"] = pcpu
        if viscosity is not None:
            line["viscosity"] = viscosity
        if served is not None:
            line["served"] = served
        if mixed is not None:
            line["mixed"] = mixed
            line["gpu_launches"] = int(line["gpu_launches"] + mixed.pop("_launches"))
        if projection is not None:
            line["projection"] = projection
            line["gpu_launches"] = int(line["gpu_launches"] + projection.pop("_launches"))
        if batched is not None:
            line["batched"] = batched
            line["gpu_launches"] = int(line["gpu_launches"] + batched.pop("_launches"))
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
