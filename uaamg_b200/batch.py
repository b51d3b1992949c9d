"""Batched pressure solves: many ``PoissonSolver`` instances in one CUDA graph.

``PoissonBatch([solver_a, solver_b, ...]).solveMultigridPCG(pressures, rhss)``
runs ``PoissonSolver.solveMultigridPCG`` (SIMD_UAAMG/simd_vdb_poisson.cpp:
2155-2226) for every instance at once: each kernel of the batched W-cycle
covers the leaves of all instances that have work at that point, and an
instance that has converged stops updating while the others go on.  Each
instance's solution, iteration count and status are identical to its own
``solveMultigridPCG``.  The reference has no batched form; the class follows
``PoissonSolver``'s member names (``mMaxIteration``, ``mRelativeTolerance``,
``mSmoother``; ``mIterationTaken`` becomes a list).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .poisson import PoissonSolver


class PoissonBatch:
    SUCCESS = PoissonSolver.SUCCESS
    FAILED = PoissonSolver.FAILED

    def __init__(self, solvers: list[PoissonSolver]):
        if not solvers:
            raise ValueError("empty batch")
        self._solvers = list(solvers)  # the batch references their hierarchies
        n = len(self._solvers)
        handles = (C.c_void_p * n)(*[s.mMultigridHierarchy._h for s in self._solvers])
        h = C.c_void_p()
        _lib.check(_lib.lib().uaamg_batch_create(n, handles, C.byref(h)), "uaamg_batch_create")
        self._h = h.value
        s0 = self._solvers[0]
        self.mMaxIteration = s0.mMaxIteration
        self.mRelativeTolerance = s0.mRelativeTolerance
        self.mSmoother = s0.mSmoother
        self.mIterationTaken = [0] * n
        self.status = [self.SUCCESS] * n
        self.use_graph = True

    def __len__(self) -> int:
        return len(self._solvers)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            try:
                _lib.lib().uaamg_batch_destroy(h)
            except Exception:
                pass
            self._h = None

    def _configure(self):
        L = _lib.lib()
        _lib.check(L.uaamg_batch_set_smoother(self._h, int(self.mSmoother)), "batch set_smoother")
        _lib.check(L.uaamg_batch_set_max_iterations(self._h, int(self.mMaxIteration)), "batch set_max_iterations")
        _lib.check(L.uaamg_batch_set_relative_tolerance(self._h, float(self.mRelativeTolerance)),
                   "batch set_tolerance")
        mode = self.use_graph if isinstance(self.use_graph, int) and not isinstance(self.use_graph, bool) \
            else (1 if self.use_graph else 0)
        _lib.check(L.uaamg_batch_set_graph_mode(self._h, mode), "batch set_graph_mode")
        return L

    def solveMultigridPCG(self, in_out_pressures: list, rhss: list) -> int:
        """Solve instance i for pressure i (in: initial guess, out: solution)
        with right-hand side i; numpy arrays (host path) or torch CUDA tensors
        (device path), leaf-dense [leaves, 512] float32.  Returns SUCCESS when
        every instance succeeded; per-instance results in mIterationTaken and
        status."""
        n = len(self._solvers)
        if len(in_out_pressures) != n or len(rhss) != n:
            raise ValueError("one pressure and one rhs per instance")
        L = self._configure()
        keep = []
        xs, bs = (C.c_void_p * n)(), (C.c_void_p * n)()
        host = isinstance(in_out_pressures[0], np.ndarray)
        for i, (x, b) in enumerate(zip(in_out_pressures, rhss)):
            if host:
                assert isinstance(x, np.ndarray) and x.dtype == np.float32 and x.flags["C_CONTIGUOUS"]
                b = np.ascontiguousarray(b, np.float32)
                keep.append(b)
                xs[i], bs[i] = x.ctypes.data, b.ctypes.data
            else:
                xs[i], bs[i] = x.data_ptr(), b.data_ptr()
        its, sts = (C.c_int * n)(), (C.c_int * n)()
        fn = L.uaamg_batch_solve_pcg if host else L.uaamg_batch_solve_pcg_device
        with _lib.torch_ordered("batch", self._h, in_out_pressures, rhss):
            rc = _lib.check(fn(self._h, xs, bs, its, sts), "uaamg_batch_solve_pcg")
        self.mIterationTaken = [int(v) for v in its]
        self.status = [int(v) for v in sts]
        return int(rc)

    def final_residuals(self) -> list[float]:
        n = len(self._solvers)
        res = (C.c_float * n)()
        _lib.check(_lib.lib().uaamg_batch_results(self._h, None, None, res), "batch results")
        return [float(v) for v in res]

    @property
    def kernel_launches(self) -> int:
        return int(_lib.lib().uaamg_batch_kernel_launches(self._h))

    def set_stream(self, stream_ptr: int | None) -> None:
        _lib.check(_lib.lib().uaamg_batch_set_stream(self._h, stream_ptr), "batch set_stream")
