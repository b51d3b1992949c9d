"""Served solves: a request loop for streams of pressure and viscosity solves.

A FLIP substep calls the pressure solve (FLIP_vdb.cpp:3118-3168) and, for
viscous liquids, the viscosity solve (FLIP_vdb.cpp:3170-3216).  A server runs
many such simulations at once: each request is one simulation domain that
asks for ``substeps`` solves of its kind, each substep with new face
velocities.  Pressure substeps warm-start from the previous pressure.

What the server does
 * admission by HBM budget: a queued request is admitted (its hierarchy built
   on the device) as soon as its estimated footprint fits next to the
   requests already resident; requests are admitted in arrival order;
 * hierarchies and warm starts stay on the device across a request's
   substeps and are released when it completes;
 * continuous batching: every round runs one substep of every resident
   pressure request, all of them in one batched CUDA graph (PoissonBatch);
   requests that arrive during a round join at the next round.  Each
   viscosity request runs on a lane of its own (a host thread and a CUDA
   stream) that does its substeps back to back, so viscosity work overlaps
   the pressure rounds on the device instead of holding them up.  At most
   ``admit_per_round`` requests are admitted (hierarchy built) per round, so
   resident requests keep moving while a burst is admitted.
 * each result is the same alone and in the mix: the batched pressure solve
   is bit-identical to a standalone solve, and viscosity solves are
   independent.

The host logic (``Scheduler``) is independent of the device work
(``DeviceBackend``), so the admission and batching rules are testable on the
CPU with a fake backend.
"""
from __future__ import annotations

import math
import threading
import time
from dataclasses import dataclass, field

import numpy as np

from . import scenes


@dataclass
class Request:
    rid: int
    kind: str          # "poisson" | "viscosity"
    side: int          # cubic domain side in voxels
    seed: int          # geometry seed (velocities of substep k: seed * 1000003 + k)
    substeps: int
    arrival: float     # seconds after the start of the stream
    admitted_at: float | None = None
    done_at: float | None = None
    step: int = 0
    iterations: list = field(default_factory=list)
    status: list = field(default_factory=list)
    result: object = None  # final solution (host copy) when the backend keeps results

    @property
    def latency(self) -> float | None:
        return None if self.done_at is None else self.done_at - self.arrival


def make_stream(duration: float, poisson_rate: float = 200.0, viscosity_rate: float = 50.0, seed: int = 0,
                lo: int = 48, hi: int = 384, max_substeps: int = 24) -> list[Request]:
    """Poisson-process arrivals of pressure (``poisson_rate``/s) and viscosity
    (``viscosity_rate``/s) requests over ``duration`` seconds; sides
    log-uniform in [lo, hi]; 1..max_substeps substeps; per-request seeds."""
    reqs: list[Request] = []
    rid = 0
    for kind, rate, base in (("poisson", poisson_rate, 1), ("viscosity", viscosity_rate, 2)):
        if rate <= 0:
            continue
        t, k = 0.0, 0
        while True:
            u = float(scenes.uniform(seed * 7 + base, 1, 0.0, 1.0, start=k)[0])
            k += 1
            t += -math.log(max(1.0 - u, 1e-12)) / rate
            if t >= duration:
                break
            s = seed * 100003 + base * 1000000 + k
            v = scenes.uniform(s + 17, 2, 0.0, 1.0)
            side = scenes.served_side(s, lo, hi)
            sub = 1 + min(int(float(v[0]) * max_substeps), max_substeps - 1)
            reqs.append(Request(rid=-1, kind=kind, side=side, seed=s, substeps=sub, arrival=t))
    reqs.sort(key=lambda r: (r.arrival, r.kind))
    for i, r in enumerate(reqs):
        r.rid = i
    return reqs


class Scheduler:
    """Admission by memory budget, pressure rounds, viscosity lanes."""

    def __init__(self, backend, budget_bytes: int, max_poisson: int = 256, max_viscosity: int = 16,
                 admit_per_round: int = 8):
        self.backend = backend
        self.budget = int(budget_bytes)
        self.max_poisson = max_poisson
        self.max_viscosity = max_viscosity
        self.admit_per_round = admit_per_round
        self.queue: list[Request] = []
        self.active: list[Request] = []
        self.done: list[Request] = []
        self.used = 0
        self.peak_used = 0
        self.rounds = 0
        self.solves = 0
        self._cost: dict[int, int] = {}

    def submit(self, r: Request) -> None:
        self.queue.append(r)

    def admit(self, now: float, limit: int | None = None) -> list[Request]:
        """Admit queued requests in arrival order while they fit (at most
        ``limit``); a viscosity request starts its lane at once."""
        out = []
        while self.queue and (limit is None or len(out) < limit):
            r = self.queue[0]
            cost = int(self.backend.estimate_bytes(r))
            if cost > self.budget:
                raise ValueError(f"request {r.rid} ({r.kind} {r.side}^3) needs {cost} B, budget {self.budget} B")
            n_kind = sum(1 for a in self.active if a.kind == r.kind)
            cap = self.max_poisson if r.kind == "poisson" else self.max_viscosity
            if self.used + cost > self.budget or n_kind >= cap:
                break
            self.queue.pop(0)
            self.backend.admit(r)
            r.admitted_at = now
            self._cost[r.rid] = cost
            self.used += cost
            self.peak_used = max(self.peak_used, self.used)
            self.active.append(r)
            if r.kind == "viscosity":
                self.backend.start_viscosity(r)
            out.append(r)
        return out

    def _retire(self, r: Request, now: float) -> None:
        r.done_at = now
        self.active.remove(r)
        self.backend.release(r)
        self.used -= self._cost.pop(r.rid)
        self.done.append(r)

    def round(self, clock) -> list[Request]:
        """One substep of every resident pressure request; collect finished
        viscosity lanes.  Returns the requests completed in this round."""
        finished = []
        pois = [r for r in self.active if r.kind == "poisson"]
        if pois:
            self.backend.poisson_round(pois)
            self.rounds += 1
            now = clock()
            for r in pois:
                r.step += 1
                self.solves += 1
                if r.step >= r.substeps:
                    finished.append(r)
                    self._retire(r, now)
        for r in [a for a in self.active if a.kind == "viscosity"]:
            if self.backend.viscosity_done(r):
                self.solves += r.substeps
                r.step = r.substeps
                finished.append(r)
                self._retire(r, clock())
        return finished

    def run(self, requests: list[Request], clock=None, sleep=time.sleep, time_limit: float = 60.0) -> float:
        """Serve ``requests`` (arrival times relative to the start) until all
        are done or ``time_limit`` seconds have passed; returns the elapsed time."""
        pending = sorted(requests, key=lambda r: r.arrival)
        if clock is None:
            t0 = time.perf_counter()
            clock = lambda: time.perf_counter() - t0  # noqa: E731
        while pending or self.queue or self.active:
            now = clock()
            if now >= time_limit:
                break
            while pending and pending[0].arrival <= now:
                self.submit(pending.pop(0))
            self.admit(now, self.admit_per_round)
            if not self.active:
                if pending:
                    sleep(max(0.0, min(pending[0].arrival - now, 0.01)))
                    continue
                if self.queue:
                    raise RuntimeError("queued requests cannot be admitted")
                break
            busy = any(r.kind == "poisson" for r in self.active)
            self.round(clock)
            if not busy and self.active:
                self.backend.wait_viscosity(0.002)  # only viscosity lanes running: poll
        return clock()


def latency_summary(done: list[Request]) -> dict:
    lat = np.array([r.latency for r in done if r.latency is not None], dtype=np.float64)
    if lat.size == 0:
        return {"p50_ms": None, "p99_ms": None, "max_ms": None}
    return {"p50_ms": round(float(np.percentile(lat, 50)) * 1e3, 2),
            "p99_ms": round(float(np.percentile(lat, 99)) * 1e3, 2),
            "max_ms": round(float(lat.max()) * 1e3, 2)}


class DeviceBackend:
    """The device work of a served stream on one GPU.

    batching=True: every round solves all pressure requests in one batched
    graph (cached while the set of resident pressure requests is unchanged)
    while the viscosity requests run concurrently on their own streams.
    batching=False (the plain form): every solve runs alone, one after
    another, through the plain API."""

    def __init__(self, device=None, batching: bool = True, keep_results: bool = False, viscosity_tol: float = 1e-6,
                 pressure_tol: float = 1e-7):
        import torch
        self.torch = torch
        self.device = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
        self.batching = batching
        self.keep_results = keep_results
        self.vtol = viscosity_tol
        self.ptol = pressure_tol
        self.slots: dict[int, dict] = {}
        self._batch = None
        self._batch_key = None
        self.batch_builds = 0
        # pressure rounds are short and latency-bound: their stream has the
        # highest priority, so their kernels go ahead of the viscosity lanes'
        lo, hi = torch.cuda.Stream.priority_range()
        self.pstream = torch.cuda.Stream(self.device, priority=hi)
        self.vstreams: list = []
        self.times = {"admit_poisson": 0.0, "admit_viscosity": 0.0, "rhs": 0.0, "batch_build": 0.0, "solve": 0.0}

    # footprint estimates (inputs + hierarchy + vectors), conservative
    @staticmethod
    def estimate_bytes(r: Request) -> int:
        m = (r.side + 16) ** 3
        return int(m * 4 * (14 if r.kind == "poisson" else 64))

    def admit(self, r: Request) -> None:
        t0 = time.perf_counter()
        self._admit(r)
        self.times["admit_" + r.kind] += time.perf_counter() - t0

    def _admit(self, r: Request) -> None:
        """Pressure: build the hierarchy now, on the high-priority stream.
        Viscosity: reserve a stream; the request's lane builds its matrix."""
        torch = self.torch
        if r.kind == "poisson":
            from .poisson import LaplacianWithLevel, PoissonSolver
            with torch.cuda.stream(self.pstream):
                phi, fw, sv, dt, dx = scenes.device_poisson_instance(r.side, r.seed, self.device)
                # built on the same stream that produced the inputs
                lap = LaplacianWithLevel.createPressurePoissonLaplacian(phi, fw, dt, dx,
                                                                        stream=self.pstream.cuda_stream)
                s = PoissonSolver(lap)
                s.mRelativeTolerance = self.ptol
                n = lap.leaf_count(0)
                x = torch.zeros((n, 512), dtype=torch.float32, device=self.device)
                rhs = torch.empty_like(x)
            self.slots[r.rid] = dict(lap=lap, solver=s, fw=fw, sv=sv, dt=dt, x=x, rhs=rhs, inputs=(phi,))
        else:
            self.slots[r.rid] = dict(stream=self._vstream())

    def _viscosity_build(self, r: Request) -> None:
        torch = self.torch
        from .viscosity import L_with_level
        slot = self.slots[r.rid]
        st = slot["stream"]
        with torch.cuda.stream(st):
            liq, sol, mu, sv, dt, rho, dx = scenes.device_viscosity_instance(r.side, r.seed, self.device)
            lv = L_with_level.create_viscosity_matrix(mu, liq, sol, dt, rho, dx, stream=st.cuda_stream)
        slot.update(lv=lv, sv=sv, inputs=(liq, sol))

    def _vstream(self):
        if self.vstreams:
            return self.vstreams.pop()
        return self.torch.cuda.Stream(self.device)

    def release(self, r: Request) -> None:
        slot = self.slots.pop(r.rid)
        if self.keep_results:
            r.result = (slot["x"] if r.kind == "poisson" else slot["xv"]).cpu().numpy()
        if r.kind == "viscosity":
            self.vstreams.append(slot["stream"])
        if self._batch_key is not None and r.rid in self._batch_key:
            self._batch, self._batch_key = None, None

    # --- one substep of each kind
    def _poisson_rhs(self, r: Request) -> None:
        s = self.slots[r.rid]
        vx, vy, vz = scenes.device_face_velocities(r.side, r.seed * 1000003 + r.step, self.device)
        s["lap"].createPressurePoissonRightHandSide(s["fw"], vx, vy, vz, s["sv"], s["dt"], out=s["rhs"])

    def _poisson_round(self, reqs: list[Request]) -> None:
        torch = self.torch
        from .batch import PoissonBatch
        with torch.cuda.stream(self.pstream):
            t0 = time.perf_counter()
            for r in reqs:
                self._poisson_rhs(r)
            t1 = time.perf_counter()
            self.times["rhs"] += t1 - t0
            if self.batching:
                key = tuple(r.rid for r in reqs)
                if key != self._batch_key:
                    self._batch = PoissonBatch([self.slots[r.rid]["solver"] for r in reqs])
                    self._batch.mRelativeTolerance = self.ptol
                    self._batch.set_stream(self.pstream.cuda_stream)
                    self._batch_key = key
                    self.batch_builds += 1
                b = self._batch
                t2 = time.perf_counter()
                self.times["batch_build"] += t2 - t1
                b.solveMultigridPCG([self.slots[r.rid]["x"] for r in reqs], [self.slots[r.rid]["rhs"] for r in reqs])
                self.times["solve"] += time.perf_counter() - t2
                for i, r in enumerate(reqs):
                    r.iterations.append(b.mIterationTaken[i])
                    r.status.append(b.status[i])
            else:
                for r in reqs:
                    s = self.slots[r.rid]
                    st = s["solver"].solveMultigridPCG(s["x"], s["rhs"])
                    r.iterations.append(s["solver"].mIterationTaken)
                    r.status.append(st)
                self.times["solve"] += time.perf_counter() - t1

    def _viscosity_step(self, r: Request, k: int) -> None:
        torch = self.torch
        from .viscosity import simd_viscosity3d
        s = self.slots[r.rid]
        with torch.cuda.stream(s["stream"]):
            lv = s["lv"]
            u, v, w = scenes.device_face_velocities(r.side, r.seed * 1000003 + k, self.device)
            n = lv.leaf_count(0)
            rhs = s.get("rhs")
            if rhs is None:
                rhs = s["rhs"] = torch.empty((3, n, 512), dtype=torch.float32, device=self.device)
                s["xv"] = torch.empty_like(rhs)
            lv.build_rhs(u, v, w, s["sv"], out=rhs)
            lv.gather_velocity(u, v, w, out=s["xv"])
            solver = simd_viscosity3d(lv)
            st = solver.pcg_solve(s["xv"], self.vtol, rhs)
            r.iterations.append(solver.m_iteration)
            r.status.append(st)

    # --- viscosity lanes
    def start_viscosity(self, r: Request) -> None:
        """Run all substeps of a viscosity request: on a lane of its own
        (thread + stream) when batching, inline in the plain form."""
        slot = self.slots[r.rid]

        def lane():
            try:
                t0 = time.perf_counter()
                self._viscosity_build(r)
                self.times["admit_viscosity"] += time.perf_counter() - t0
                for k in range(r.substeps):
                    self._viscosity_step(r, k)
                slot["stream"].synchronize()
            except BaseException as e:  # reported by viscosity_done
                slot["error"] = e

        if not self.batching:
            lane()
            return
        t = threading.Thread(target=lane, daemon=True)
        slot["thread"] = t
        t.start()

    def viscosity_done(self, r: Request) -> bool:
        slot = self.slots[r.rid]
        t = slot.get("thread")
        if t is not None and t.is_alive():
            return False
        if "error" in slot:
            raise slot["error"]
        return True

    def wait_viscosity(self, seconds: float) -> None:
        time.sleep(seconds)

    def poisson_round(self, reqs: list[Request]) -> None:
        self._poisson_round(reqs)
