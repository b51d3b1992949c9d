"""Autotuner of the solver's kernel shapes (no counterpart in the reference).

The C library picks, per multigrid level, which kernel form sweeps it: the
one-leaf kernels, the bulk-copy staged kernels (from ``staged_min_leaves``
leaves), stored computed sources (from ``split_min_leaves``), the grid of the
grid-stride passes (``elem_ctas_per_sm``), and whether the bottom of the
W-cycle runs as one thread-block-cluster launch (``bottom_cycle``).  All of
these give the same results; they only move time.  This module measures
candidate settings on representative solves and keeps the fastest:

* ``search`` is a coordinate descent over a discrete space: starting from a
  base setting it tries every value of one knob with the others held, keeps
  the best, moves to the next knob, and repeats whole rounds until a round
  improves nothing (or a round limit).  A candidate must beat the incumbent
  by ``min_gain`` (relative) to replace it, so timing noise does not churn
  the table.
* ``tune`` measures on the GPU: a candidate's cost is the sum over the
  workloads of the median device time of a few graph solves.
* A table (JSON, keyed by GPU name and SM count) records the chosen setting,
  the workloads and every trial; ``apply`` loads the table for the current GPU
  and sets it with ``uaamg_set_tuning``.  Nothing applies a table implicitly:
  the library starts from its built-in defaults.

``pipe_min_leaves`` moves only the passes without a dot product: the passes
that carry the PCG's level-0 dot products switch to the pipelined kernels at a
fixed size (their per-CTA partials set the summation order), so no setting
changes a result.

    python -m uaamg_b200.autotune --out uaamg_b200/tuning/NVIDIA_B200.json
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import time
from typing import Callable

from . import _lib

KNOBS = ("staged_min_leaves", "split_min_leaves", "pipe_min_leaves", "elem_ctas_per_sm", "bottom_cycle")
NEVER = 1 << 30  # a leaf threshold no level reaches

# the searched values of each result-neutral knob
SPACE = {
    "bottom_cycle": [0, 1],
    "pipe_min_leaves": [1024, 2048, 4096, 8192, 16384],
    "staged_min_leaves": [16, 32, 64, 128, 256, 512],
    "split_min_leaves": [256, 512, 1024, 2048, 4096, NEVER],
    "elem_ctas_per_sm": [4, 8, 16, 32],
}

TABLE_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tuning")


# ----------------------------------------------------------------------------- library access
def get() -> dict:
    t = _lib.TuningC()
    _lib.check(_lib.lib().uaamg_get_tuning(C.byref(t)), "uaamg_get_tuning")
    return {k: int(getattr(t, k)) for k in KNOBS}


def set(setting: dict) -> None:  # noqa: A001 - mirrors the C entry point's name
    cur = get()
    cur.update({k: int(v) for k, v in setting.items() if k in KNOBS})
    t = _lib.TuningC(*[cur[k] for k in KNOBS])
    _lib.check(_lib.lib().uaamg_set_tuning(C.byref(t)), "uaamg_set_tuning")


# ----------------------------------------------------------------------------- search
def search(measure: Callable[[dict], float], space: dict, base: dict, max_rounds: int = 3,
           min_gain: float = 0.01, log: list | None = None) -> tuple[dict, float]:
    """Coordinate descent: returns (best setting, its cost).  ``measure``
    maps a full setting to a cost (lower is better); every evaluation is
    appended to ``log`` as {"setting", "cost"}.  Settings already measured are
    not measured again."""
    cache: dict[tuple, float] = {}

    def cost(s: dict) -> float:
        key = tuple(sorted(s.items()))
        if key not in cache:
            cache[key] = float(measure(dict(s)))
            if log is not None:
                log.append({"setting": dict(s), "cost": cache[key]})
        return cache[key]

    best = dict(base)
    best_cost = cost(best)
    for _ in range(max_rounds):
        improved = False
        for knob, values in space.items():
            for v in values:
                if v == best.get(knob):
                    continue
                cand = dict(best)
                cand[knob] = v
                c = cost(cand)
                if c < best_cost * (1.0 - min_gain):
                    best, best_cost, improved = cand, c, True
        if not improved:
            break
    return best, best_cost


# ----------------------------------------------------------------------------- tables
def gpu_key(name: str, sms: int) -> str:
    return "".join(ch if ch.isalnum() else "_" for ch in name).strip("_") + f"_{sms}sm"


def table_path(name: str, sms: int, directory: str = TABLE_DIR) -> str:
    return os.path.join(directory, gpu_key(name, sms) + ".json")


def load(path: str) -> dict:
    with open(path) as f:
        table = json.load(f)
    setting = table["tuning"]
    missing = [k for k in KNOBS if k not in setting]
    if missing:
        raise ValueError(f"tuning table {path} lacks {missing}")
    return table


def apply(path: str | None = None, device: int = 0) -> dict | None:
    """Set the table for this GPU (or the one at ``path``); returns the table,
    or None when there is none for this GPU."""
    if path is None:
        import torch
        p = torch.cuda.get_device_properties(device)
        path = table_path(p.name, p.multi_processor_count)
        if not os.path.exists(path):
            return None
    table = load(path)
    set(table["tuning"])
    return table


# ----------------------------------------------------------------------------- measurement
def _workloads(sizes):
    """Device-resident Poisson hierarchies and right-hand sides of the plain
    workload geometry (slab y < 0.4 plus a sphere) at the given sizes."""
    import torch
    from . import scenes
    from .grids import LeafGrid
    from .poisson import LaplacianWithLevel, PoissonSolver
    dev = torch.device("cuda", torch.cuda.current_device())
    out = []
    for n in sizes:
        sc = scenes.plain_poisson_scene(n=n, seed=0)

        def on_device(g):
            d = LeafGrid(origins=g.origins, values=g.values, background=g.background, masks=g.masks)
            d.values = torch.from_numpy(g.values).to(dev)
            return d

        gr = [on_device(getattr(sc, k)) for k in ("phi", "face_weights", "vx", "vy", "vz", "solid_velocity")]
        lap = LaplacianWithLevel.createPressurePoissonLaplacianWithRhs(*gr, sc.dt, sc.dx)
        rhs = lap.copy_rhs(torch.empty((lap.leaf_count(0), 512), dtype=torch.float32, device=dev))
        s = PoissonSolver(lap)
        s.use_graph = 2
        out.append({"n": n, "lap": lap, "solver": s, "rhs": rhs, "x": torch.zeros_like(rhs),
                    "leaves": [lap.leaf_count(l) for l in range(lap.num_levels())]})
    return out


def tune(sizes=(96, 128, 192), solves: int = 7, max_rounds: int = 3) -> dict:
    import torch
    works = _workloads(sizes)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=works[0]["rhs"].device)

    def measure(setting: dict) -> float:
        set(setting)
        total = 0.0
        for w in works:
            ts = []
            for i in range(solves + 2):
                w["x"].zero_()
                flush.zero_()
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record()
                w["solver"].solveMultigridPCG(w["x"], w["rhs"])
                b.record()
                torch.cuda.synchronize()
                if i >= 2:  # the first solves capture the graph
                    ts.append(a.elapsed_time(b))
            total += statistics.median(ts)
        return total

    base = get()
    log: list = []
    t0 = time.perf_counter()
    best, cost = search(measure, SPACE, base, max_rounds=max_rounds, log=log)
    set(best)
    p = torch.cuda.get_device_properties(torch.cuda.current_device())
    return {"gpu": p.name, "sm_count": p.multi_processor_count, "tuning": best, "cost_ms": round(cost, 4),
            "default_cost_ms": round(log[0]["cost"], 4),
            "objective": f"sum over the workloads of the median device time of {solves} graph solves (ms), "
                         "L2 flushed before each",
            "workloads": [{"n": w["n"], "leaves": w["leaves"]} for w in works],
            "trials": [{"setting": t["setting"], "cost_ms": round(t["cost"], 4)} for t in log],
            "search_s": round(time.perf_counter() - t0, 1),
            "when": time.strftime("%Y-%m-%dT%H:%M:%SZ", time.gmtime())}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=None, help="table path (default: tuning/<gpu>_<sms>sm.json)")
    ap.add_argument("--sizes", default="96,128,192")
    ap.add_argument("--solves", type=int, default=7)
    args = ap.parse_args()
    from . import build
    build.build()
    table = tune(tuple(int(x) for x in args.sizes.split(",")), args.solves)
    out = args.out or table_path(table["gpu"], table["sm_count"])
    os.makedirs(os.path.dirname(out), exist_ok=True)
    with open(out, "w") as f:
        json.dump(table, f, indent=1)
    print(json.dumps({k: table[k] for k in ("gpu", "tuning", "cost_ms", "default_cost_ms", "search_s")}))
    print("wrote", out)


if __name__ == "__main__":
    main()
