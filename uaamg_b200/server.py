"""Python mirror of the native served form (uaamg_server_* in include/uaamg.h).

The server runs in the library on a thread of its own: requests are submitted
with their operator inputs, each substep's face velocities are pushed as the
simulation produces them, and results are waited for per substep.  See the
header for the admission, batching and lane rules.  Grids may live on the host
(numpy) or on the device (torch CUDA tensors); the server copies them at the
call, after synchronising torch's current stream when a grid is on the device.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .grids import LeafGrid
from .poisson import _as_c

POISSON, VISCOSITY = 0, 1


class NativeServer:
    """A served-form instance on the current CUDA device."""

    def __init__(self, budget_bytes: int | None = None, max_poisson: int | None = None,
                 max_viscosity: int | None = None, admit_per_round: int | None = None, batching: bool = True,
                 keep_results: bool = False, pressure_tolerance: float | None = None,
                 viscosity_tolerance: float | None = None):
        L = _lib.lib()
        o = _lib.ServerOptionsC()
        _lib.check(L.uaamg_server_default_options(C.byref(o)), "uaamg_server_default_options")
        for name, val in (("budget_bytes", budget_bytes), ("max_poisson", max_poisson),
                          ("max_viscosity", max_viscosity), ("admit_per_round", admit_per_round),
                          ("pressure_tolerance", pressure_tolerance), ("viscosity_tolerance", viscosity_tolerance)):
            if val is not None:
                setattr(o, name, val)
        o.batching = 1 if batching else 0
        o.keep_results = 1 if keep_results else 0
        self.options = o
        h = C.c_void_p()
        _lib.check(L.uaamg_server_create(C.byref(o), C.byref(h)), "uaamg_server_create")
        self._h = h.value

    def close(self) -> None:
        h = getattr(self, "_h", None)
        if h:
            _lib.lib().uaamg_server_destroy(h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # interpreter shutdown
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # --- requests
    def submit_poisson(self, liquid_phi: LeafGrid, face_weights: LeafGrid, solid_velocity: LeafGrid, dt: float,
                       dx: float, substeps: int) -> int:
        keep: list = []
        gs = [_as_c(g, keep) for g in (liquid_phi, face_weights, solid_velocity)]
        _lib.torch_inputs_ready(None, liquid_phi, face_weights, solid_velocity)
        rid = C.c_int64(0)
        _lib.check(_lib.lib().uaamg_server_submit_poisson(self._h, *[C.byref(g) for g in gs], float(dt), float(dx),
                                                          int(substeps), C.byref(rid)), "uaamg_server_submit_poisson")
        return int(rid.value)

    def submit_viscosity(self, viscosity: LeafGrid, liquid_sdf: LeafGrid, solid_sdf: LeafGrid,
                         solid_velocity: LeafGrid, dt: float, rho: float, dx: float, substeps: int) -> int:
        keep: list = []
        gs = [_as_c(g, keep) for g in (viscosity, liquid_sdf, solid_sdf, solid_velocity)]
        _lib.torch_inputs_ready(None, viscosity, liquid_sdf, solid_sdf, solid_velocity)
        rid = C.c_int64(0)
        _lib.check(_lib.lib().uaamg_server_submit_viscosity(self._h, *[C.byref(g) for g in gs], float(dt), float(rho),
                                                            float(dx), int(substeps), C.byref(rid)),
                   "uaamg_server_submit_viscosity")
        return int(rid.value)

    def push_velocity(self, request: int, u: LeafGrid, v: LeafGrid, w: LeafGrid) -> None:
        keep: list = []
        gs = [_as_c(g, keep) for g in (u, v, w)]
        _lib.torch_inputs_ready(None, u, v, w)
        _lib.check(_lib.lib().uaamg_server_push_velocity(self._h, int(request), *[C.byref(g) for g in gs]),
                   "uaamg_server_push_velocity")

    def wait(self, request: int, substep: int, timeout_s: float = 60.0) -> dict:
        st, it = C.c_int(0), C.c_int(0)
        res, lat = C.c_double(0.0), C.c_double(0.0)
        _lib.check(_lib.lib().uaamg_server_wait(self._h, int(request), int(substep), float(timeout_s), C.byref(st),
                                                C.byref(it), C.byref(res), C.byref(lat)), "uaamg_server_wait")
        return {"status": int(st.value), "iterations": int(it.value), "fp64_residual": float(res.value),
                "latency_s": float(lat.value)}

    def result(self, request: int, substep: int, kind: int = POISSON) -> np.ndarray:
        n = C.c_int64(0)
        L = _lib.lib()
        _lib.check(L.uaamg_server_result(self._h, int(request), int(substep), C.byref(n), None), "uaamg_server_result")
        shape = (int(n.value), 512) if kind == POISSON else (3, int(n.value), 512)
        out = np.zeros(shape, np.float32)
        _lib.check(L.uaamg_server_result(self._h, int(request), int(substep), C.byref(n), out.ctypes.data),
                   "uaamg_server_result")
        return out

    def stats(self) -> dict:
        st = _lib.ServerStatsC()
        _lib.check(_lib.lib().uaamg_server_stats(self._h, C.byref(st)), "uaamg_server_stats")
        return {k: int(getattr(st, k)) for k, _ in _lib.ServerStatsC._fields_}
