"""Python mirror of the reference's pressure-solver interface over the C ABI.

Names, argument meaning and status codes follow SIMD_UAAMG/simd_vdb_poisson.h:
``LaplacianWithLevel.createPressurePoissonLaplacian`` (h:54-57),
``createPressurePoissonRightHandSide`` (h:59-65), ``getZeroVectorGrid`` (h:98),
``PoissonSolver`` with ``mMaxIteration``/``mRelativeTolerance``/``mSmoother``/
``mIterationTaken`` and ``solveMultigridPCG``/``solvePureMultigrid`` returning
``SUCCESS`` (0) / ``FAILED`` (1) (h:141-169).  Grids are ``LeafGrid`` objects
(flattened OpenVDB leaves); vectors are leaf-dense float32 [leaves, 512] arrays
(numpy on the host, or torch CUDA tensors for the ``*_device`` path).
"""
from __future__ import annotations

import ctypes as C
import enum

import numpy as np

from . import _lib
from .grids import LeafGrid


def _as_c(grid: LeafGrid, keep: list) -> _lib.LeafGridC:
    """The C view of a leaf grid (pointers into its arrays).  A grid passed
    again with the same arrays (the same objects, the same tensor storage)
    reuses the view built the first time: a FLIP loop hands the same input
    grids to every substep."""
    vals = grid.values
    key = (id(grid.origins), id(grid.masks), id(vals), grid.leaf_count, grid.components,
           vals.data_ptr() if hasattr(vals, "data_ptr") else None,
           np.asarray(grid.background, np.float32).tobytes())
    cached = getattr(grid, "_c_view", None)
    if cached is not None and cached[0] == key:
        keep.extend(cached[2])
        return cached[1]
    mine: list = []
    g = _as_c_build(grid, mine)
    keep.extend(mine)
    # only a view of the grid's own arrays is kept: a converted copy would miss later in-place writes
    if all(a is grid.origins or a is grid.masks or a is vals for a in mine):
        try:
            grid._c_view = (key, g, mine)
        except AttributeError:  # a grid type without a writable __dict__
            pass
    return g


def _as_c_build(grid: LeafGrid, keep: list) -> _lib.LeafGridC:
    g = _lib.LeafGridC()
    g.leaf_count = grid.leaf_count
    org = np.ascontiguousarray(grid.origins, dtype=np.int32)
    keep.append(org)
    g.origins = org.ctypes.data if grid.leaf_count else None
    if grid.masks is not None and grid.leaf_count:
        m = np.ascontiguousarray(grid.masks, dtype=np.uint64)
        keep.append(m)
        g.masks = m.ctypes.data
    else:
        g.masks = None
    vals = grid.values
    if isinstance(vals, np.ndarray):
        v = np.ascontiguousarray(vals, dtype=np.float32)
        keep.append(v)
        g.values = v.ctypes.data if grid.leaf_count else None
        g.values_on_device = 0
    else:  # torch tensor
        keep.append(vals)
        g.values = vals.data_ptr() if grid.leaf_count else None
        g.values_on_device = 1 if vals.is_cuda else 0
    g.components = grid.components
    bg = np.zeros(3, np.float32)
    bg[: grid.background.size] = grid.background
    for i in range(3):
        g.background[i] = float(bg[i])
    return g


class LaplacianWithLevel:
    """The pressure Poisson operator with its multigrid hierarchy on the GPU."""

    def __init__(self, handle: int, dt: float, dx: float):
        self._h = handle
        self.mDt = dt
        self.mDxThisLevel = dx
        self.mLevel = 0
        # solver settings last applied to the handle (smoother, max iterations,
        # relative tolerance, graph mode): a new handle holds these defaults
        self._applied = (0, 100, 1e-7, 1)

    @staticmethod
    def createPressurePoissonLaplacian(liquid_phi: LeafGrid, face_weights: LeafGrid, dt: float,
                                       dx: float, stream: int | None = None) -> "LaplacianWithLevel":
        """``stream``: a cudaStream_t (int) to build on; the handle keeps it."""
        L = _lib.lib()
        keep: list = []
        a = _as_c(liquid_phi, keep)
        b = _as_c(face_weights, keep)
        h = C.c_void_p()
        _lib.torch_inputs_ready(stream, liquid_phi, face_weights)
        _lib.check(L.uaamg_poisson_create_on_stream(C.byref(a), C.byref(b), float(dt), float(dx), stream,
                                                    C.byref(h)), "uaamg_poisson_create")
        _lib.torch_after("poisson", h.value, liquid_phi, face_weights)
        return LaplacianWithLevel(h.value, dt, dx)

    @staticmethod
    def createPressurePoissonLaplacianWithRhs(liquid_phi: LeafGrid, face_weights: LeafGrid, vx: LeafGrid,
                                              vy: LeafGrid, vz: LeafGrid, solid_velocity: LeafGrid, dt: float,
                                              dx: float, stream: int | None = None) -> "LaplacianWithLevel":
        """createPressurePoissonLaplacian + createPressurePoissonRightHandSide
        in one C-ABI call (uaamg_poisson_create_with_rhs): every input crosses
        the bus once and the rhs stays on the device for
        ``PoissonSolver.solveMultigridPCGResident``."""
        L = _lib.lib()
        keep: list = []
        grids = (liquid_phi, face_weights, vx, vy, vz, solid_velocity)
        gs = [_as_c(g, keep) for g in grids]
        h = C.c_void_p()
        _lib.torch_inputs_ready(stream, grids)
        _lib.check(L.uaamg_poisson_create_with_rhs(*[C.byref(g) for g in gs], float(dt), float(dx), stream,
                                                   C.byref(h)), "uaamg_poisson_create_with_rhs")
        _lib.torch_after("poisson", h.value, grids)
        return LaplacianWithLevel(h.value, dt, dx)

    def copy_rhs(self, out=None):
        """The rhs built by createPressurePoissonLaplacianWithRhs (numpy, or
        into a torch CUDA tensor)."""
        rhs = self.getZeroVectorGrid() if out is None else out
        ptr = rhs.ctypes.data if isinstance(rhs, np.ndarray) else rhs.data_ptr()
        with _lib.torch_ordered("poisson", self._h, rhs):
            _lib.check(_lib.lib().uaamg_poisson_copy_rhs(self._h, ptr), "copy_rhs")
        return rhs

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            try:
                _lib.lib().uaamg_poisson_destroy(h)
            except Exception:  # interpreter shutdown
                pass
            self._h = None

    # --- topology / sizes
    @property
    def mNumDof(self) -> int:
        return int(_lib.lib().uaamg_poisson_num_dof(self._h, 0))

    def num_levels(self) -> int:
        return int(_lib.lib().uaamg_poisson_num_levels(self._h))

    def num_dof(self, level: int = 0) -> int:
        return int(_lib.lib().uaamg_poisson_num_dof(self._h, level))

    def leaf_count(self, level: int = 0) -> int:
        return int(_lib.lib().uaamg_poisson_leaf_count(self._h, level))

    def dof_topology(self, level: int = 0):
        n = self.leaf_count(level)
        o = np.zeros((n, 3), np.int32)
        m = np.zeros((n, 8), np.uint64)
        _lib.check(_lib.lib().uaamg_poisson_dof_topology(self._h, level, o.ctypes.data, m.ctypes.data),
                   "dof_topology")
        return o, m

    def dof_index(self, level: int = 0) -> np.ndarray:
        out = np.zeros((self.leaf_count(level), 512), np.int32)
        _lib.check(_lib.lib().uaamg_poisson_dof_index(self._h, level, out.ctypes.data), "dof_index")
        return out

    def getZeroVectorGrid(self, level: int = 0) -> np.ndarray:
        return np.zeros((self.leaf_count(level), 512), np.float32)

    # --- right-hand side
    def createPressurePoissonRightHandSide(self, face_weights, vx, vy, vz, solid_velocity, dt,
                                           out=None):
        keep: list = []
        gs = [_as_c(g, keep) for g in (face_weights, vx, vy, vz, solid_velocity)]
        L = _lib.lib()
        if out is not None and not isinstance(out, np.ndarray):
            with _lib.torch_ordered("poisson", self._h, out, face_weights, vx, vy, vz, solid_velocity):
                _lib.check(L.uaamg_poisson_build_rhs_device(self._h, *[C.byref(g) for g in gs], float(dt),
                                                            out.data_ptr()), "build_rhs_device")
            return out
        _lib.torch_inputs_ready(None, face_weights, vx, vy, vz, solid_velocity)
        rhs = self.getZeroVectorGrid() if out is None else out
        _lib.check(L.uaamg_poisson_build_rhs(self._h, *[C.byref(g) for g in gs], float(dt), rhs.ctypes.data),
                   "build_rhs")
        return rhs

    def residual_norm_device(self, d_x, d_b, d_r, d_norm) -> None:
        """r = b - A x and |r|_inf into device tensors (enqueued on the handle's stream)."""
        with _lib.torch_ordered("poisson", self._h, d_x, d_b, d_r, d_norm):
            _lib.check(_lib.lib().uaamg_poisson_residual_norm_device(self._h, d_x.data_ptr(), d_b.data_ptr(),
                                                                     d_r.data_ptr(), d_norm.data_ptr()),
                       "residual_norm_device")

    def set_stream(self, stream_ptr) -> None:
        _lib.check(_lib.lib().uaamg_poisson_set_stream(self._h, stream_ptr), "set_stream")

    # --- per-level operators (public methods of the reference class)
    def apply(self, level, mode, lhs, rhs=None, weight=6.0 / 7.0, w_sor=1.2):
        modes = {"jacobi": 0, "residual": 1, "laplacian": 2, "red_gs": 3, "black_gs": 4, "spai0": 5}
        out = np.zeros_like(lhs, dtype=np.float32)
        lhs = np.ascontiguousarray(lhs, np.float32)
        rhs = lhs if rhs is None else np.ascontiguousarray(rhs, np.float32)
        _lib.check(_lib.lib().uaamg_poisson_level_apply(self._h, level, modes[mode], weight, w_sor,
                                                        lhs.ctypes.data, rhs.ctypes.data, out.ctypes.data),
                   "level_apply")
        return out

    def residualApply(self, lhs, rhs, level=0):
        return self.apply(level, "residual", lhs, rhs)

    def laplacianApply(self, lhs, level=0):
        return self.apply(level, "laplacian", lhs)

    def weightedJacobiApply(self, lhs, rhs, weight=6.0 / 7.0, level=0):
        return self.apply(level, "jacobi", lhs, rhs, weight=weight)

    def first_sweep(self, level, kind, rhs, weight=6.0 / 7.0, w_sor=1.2):
        kinds = {"jacobi": 0, "spai0": 1, "rbgs": 2}
        out = np.zeros_like(rhs, dtype=np.float32)
        rhs = np.ascontiguousarray(rhs, np.float32)
        _lib.check(_lib.lib().uaamg_poisson_level_first_sweep(self._h, level, kinds[kind], weight, w_sor,
                                                              rhs.ctypes.data, out.ctypes.data), "first_sweep")
        return out

    def restriction(self, fine, fine_level=0):
        out = np.zeros((self.leaf_count(fine_level + 1), 512), np.float32)
        fine = np.ascontiguousarray(fine, np.float32)
        _lib.check(_lib.lib().uaamg_poisson_level_restrict(self._h, fine_level, fine.ctypes.data,
                                                           out.ctypes.data), "restrict")
        return out

    def prolongation(self, coarse, fine, fine_level=0, alpha=1.0):
        out = np.array(fine, dtype=np.float32, copy=True)
        coarse = np.ascontiguousarray(coarse, np.float32)
        _lib.check(_lib.lib().uaamg_poisson_level_prolongate(self._h, fine_level, coarse.ctypes.data,
                                                             out.ctypes.data, alpha), "prolongate")
        return out

    def coefficients(self, level=0):
        n = self.leaf_count(level)
        arr = [np.zeros((n, 512), np.float32) for _ in range(4)]
        flags = np.zeros(n, np.uint8)
        _lib.check(_lib.lib().uaamg_poisson_level_coefficients(self._h, level, *[a.ctypes.data for a in arr],
                                                                flags.ctypes.data), "coefficients")
        return arr, flags

    def coarsest_solve(self, rhs):
        out = np.zeros_like(rhs, dtype=np.float32)
        rhs = np.ascontiguousarray(rhs, np.float32)
        _lib.check(_lib.lib().uaamg_poisson_coarsest_solve(self._h, rhs.ctypes.data, out.ctypes.data),
                   "coarsest_solve")
        return out


def solve_graph_cache_stats() -> tuple[int, int]:
    """(hits, captures) of the process's solve-graph cache: first solves that
    replayed a graph captured for an earlier handle with the same launch
    sequence, and graphs captured into the cache (uaamg_solve_graph_cache_stats)."""
    hits, caps = C.c_int64(0), C.c_int64(0)
    _lib.check(_lib.lib().uaamg_solve_graph_cache_stats(C.byref(hits), C.byref(caps)), "solve_graph_cache_stats")
    return int(hits.value), int(caps.value)


class PoissonSolver:
    """PCG with the unsmoothed-aggregation mu-cycle (mu = 2) as preconditioner."""

    class SmootherOption(enum.IntEnum):
        ScheduledRelaxedJacobi = 0
        WeightedJacobi = 1
        RedBlackGaussSeidel = 2
        SPAI0 = 3

    SUCCESS = 0
    FAILED = 1

    def __init__(self, level0: LaplacianWithLevel):
        self.mMultigridHierarchy = level0
        self.mIterationTaken = 0
        self.mMaxIteration = 100
        self.mRelativeTolerance = 1e-7
        self.mSmoother = PoissonSolver.SmootherOption.ScheduledRelaxedJacobi
        self.use_graph = True

    def _configure(self):
        L = _lib.lib()
        lvl = self.mMultigridHierarchy
        h = lvl._h
        mode = self.use_graph if isinstance(self.use_graph, int) and not isinstance(self.use_graph, bool) \
            else (1 if self.use_graph else 0)
        want = (int(self.mSmoother), int(self.mMaxIteration), float(self.mRelativeTolerance), int(mode))
        if getattr(lvl, "_applied", None) != want:  # the handle keeps its settings between solves
            _lib.check(L.uaamg_poisson_set_smoother(h, want[0]), "set_smoother")
            _lib.check(L.uaamg_poisson_set_max_iterations(h, want[1]), "set_max_iterations")
            _lib.check(L.uaamg_poisson_set_relative_tolerance(h, want[2]), "set_tolerance")
            _lib.check(L.uaamg_poisson_set_graph_mode(h, want[3]), "set_graph_mode")
            lvl._applied = want
        return L, h

    def _solve(self, host_fn, dev_fn, pressure, rhs) -> int:
        L, h = self._configure()
        it = C.c_int(0)
        if isinstance(pressure, np.ndarray):
            assert pressure.dtype == np.float32 and pressure.flags["C_CONTIGUOUS"]
            rhs = np.ascontiguousarray(rhs, np.float32)
            rc = getattr(L, host_fn)(h, pressure.ctypes.data, rhs.ctypes.data, C.byref(it))
        else:
            with _lib.torch_ordered("poisson", h, pressure, rhs):
                rc = getattr(L, dev_fn)(h, pressure.data_ptr(), rhs.data_ptr(), C.byref(it))
        _lib.check(rc, host_fn)
        self.mIterationTaken = int(it.value)
        return int(rc)

    def solveMultigridPCG(self, in_out_pressure, in_rhs) -> int:
        return self._solve("uaamg_poisson_solve_pcg", "uaamg_poisson_solve_pcg_device", in_out_pressure, in_rhs)

    def solvePureMultigrid(self, in_out_pressure, in_rhs) -> int:
        return self._solve("uaamg_poisson_solve_mg", "uaamg_poisson_solve_mg_device", in_out_pressure, in_rhs)

    def solveMultigridPCGResident(self, out_pressure, pure_multigrid: bool = False) -> int:
        """solveMultigridPCG (or solvePureMultigrid) from a zero pressure with
        the rhs built at creation (a level 0 made by
        createPressurePoissonLaplacianWithRhs); the pressure is written to
        ``out_pressure`` (numpy or a torch CUDA tensor)."""
        L, h = self._configure()
        it = C.c_int(0)
        if isinstance(out_pressure, np.ndarray):
            assert out_pressure.dtype == np.float32 and out_pressure.flags["C_CONTIGUOUS"]
            fn = "uaamg_poisson_solve_mg_resident" if pure_multigrid else "uaamg_poisson_solve_pcg_resident"
            rc = getattr(L, fn)(h, out_pressure.ctypes.data, C.byref(it))
        else:
            assert not pure_multigrid, "the device form is PCG only"
            fn = "uaamg_poisson_solve_pcg_resident_device"
            with _lib.torch_ordered("poisson", h, out_pressure):
                rc = L.uaamg_poisson_solve_pcg_resident_device(h, out_pressure.data_ptr(), C.byref(it))
        _lib.check(rc, fn)
        self.mIterationTaken = int(it.value)
        return int(rc)

    # --- mixed-precision form (no counterpart in the reference): the
    # preconditioner's hierarchy in FP16/BF16 with FP32 arithmetic, FP32 outer
    # CG with FP64 dots, true-residual replacement, FP64 coarsest solve
    PRECISIONS = {"fp16": 1, "bf16": 2}

    def prepare_mixed(self, precision: str = "fp16") -> float:
        """Build the 16-bit hierarchy and the FP64 coarsest inverse; returns
        the time it took (ms)."""
        L, h = self._configure()
        ms = C.c_double(0.0)
        _lib.check(L.uaamg_poisson_prepare_mixed(h, self.PRECISIONS[precision], C.byref(ms)), "prepare_mixed")
        return float(ms.value)

    def set_residual_replacement(self, every: int) -> None:
        _lib.check(_lib.lib().uaamg_poisson_set_residual_replacement(self.mMultigridHierarchy._h, int(every)),
                   "set_residual_replacement")

    def solveMultigridPCGMixed(self, in_out_pressure, in_rhs, precision: str = "fp16") -> int:
        L, h = self._configure()
        it = C.c_int(0)
        prec = self.PRECISIONS[precision]
        if isinstance(in_out_pressure, np.ndarray):
            assert in_out_pressure.dtype == np.float32 and in_out_pressure.flags["C_CONTIGUOUS"]
            rhs = np.ascontiguousarray(in_rhs, np.float32)
            rc = L.uaamg_poisson_solve_pcg_mixed(h, prec, in_out_pressure.ctypes.data, rhs.ctypes.data, C.byref(it))
        else:
            with _lib.torch_ordered("poisson", h, in_out_pressure, in_rhs):
                rc = L.uaamg_poisson_solve_pcg_mixed_device(h, prec, in_out_pressure.data_ptr(), in_rhs.data_ptr(),
                                                            C.byref(it))
        _lib.check(rc, "solve_pcg_mixed")
        self.mIterationTaken = int(it.value)
        return int(rc)

    def true_residual_fp64(self, d_x, d_b) -> tuple[float, float]:
        """(|b - A x|_inf, |b|_inf) in FP64 from the FP32 level-0 matrix (device tensors)."""
        out = (C.c_double * 2)()
        h = self.mMultigridHierarchy._h
        with _lib.torch_ordered("poisson", h, d_x, d_b):
            _lib.check(_lib.lib().uaamg_poisson_true_residual_fp64(h, d_x.data_ptr(), d_b.data_ptr(), out),
                       "true_residual_fp64")
        return float(out[0]), float(out[1])

    def solve_fp64_reference(self, d_rhs, d_x, rel_tol: float = 1e-12, max_iter: int = 200):
        """The FP64 reference solution of the level-0 system (torch CUDA
        tensors: d_rhs float32 [n, 512], d_x float64 [n, 512] out): flexible
        FP64 PCG with the FP32 W-cycle as preconditioner, to a true relative
        2-norm residual of rel_tol.  Returns (status, iterations, residual)."""
        L, h = self._configure()
        it = C.c_int(0)
        rr = C.c_double(0.0)
        with _lib.torch_ordered("poisson", h, d_rhs, d_x):
            rc = L.uaamg_poisson_solve_fp64_reference(h, d_rhs.data_ptr(), d_x.data_ptr(), float(rel_tol),
                                                      int(max_iter), C.byref(it), C.byref(rr))
        _lib.check(rc, "solve_fp64_reference")
        return int(rc), int(it.value), float(rr.value)

    def precondition(self, r: np.ndarray) -> np.ndarray:
        L, h = self._configure()
        z = np.zeros_like(r, dtype=np.float32)
        r = np.ascontiguousarray(r, np.float32)
        _lib.check(L.uaamg_poisson_precondition(h, r.ctypes.data, z.ctypes.data), "precondition")
        return z

    def profile_pcg(self, d_pressure, d_rhs, max_classes: int = 64):
        """One solve with CUDA events around every kernel (device tensors).
        Returns {kernel class: (total ms, launches)}."""
        L, h = self._configure()
        names = C.create_string_buffer(64 * max_classes)
        ms = np.zeros(max_classes, np.float64)
        cnt = np.zeros(max_classes, np.int64)
        nc = C.c_int(0)
        with _lib.torch_ordered("poisson", h, d_pressure, d_rhs):
            rc = L.uaamg_poisson_profile_pcg(h, d_pressure.data_ptr(), d_rhs.data_ptr(), max_classes,
                                             C.addressof(names), ms.ctypes.data, cnt.ctypes.data, C.byref(nc))
        _lib.check(rc, "profile_pcg")
        return self._prof_table(names, ms, cnt, nc.value)

    def profile_pcg_mixed(self, d_pressure, d_rhs, precision: str = "fp16", max_classes: int = 64):
        """profile_pcg of the mixed-precision form."""
        L, h = self._configure()
        names = C.create_string_buffer(64 * max_classes)
        ms = np.zeros(max_classes, np.float64)
        cnt = np.zeros(max_classes, np.int64)
        nc = C.c_int(0)
        with _lib.torch_ordered("poisson", h, d_pressure, d_rhs):
            rc = L.uaamg_poisson_profile_pcg_mixed(h, self.PRECISIONS[precision], d_pressure.data_ptr(),
                                                   d_rhs.data_ptr(), max_classes, C.addressof(names),
                                                   ms.ctypes.data, cnt.ctypes.data, C.byref(nc))
        _lib.check(rc, "profile_pcg_mixed")
        return self._prof_table(names, ms, cnt, nc.value)

    def _prof_table(self, names, ms, cnt, n):
        self.mIterationTaken = int(_lib.lib().uaamg_poisson_iterations(self.mMultigridHierarchy._h))
        raw = names.raw
        out = {}
        for k in range(n):
            nm = raw[64 * k: 64 * k + 64].split(b"\0", 1)[0].decode()
            out[nm] = (float(ms[k]), int(cnt[k]))
        return out

    @property
    def final_residual(self) -> float:
        return float(_lib.lib().uaamg_poisson_final_residual(self.mMultigridHierarchy._h))

    @property
    def kernel_launches(self) -> int:
        return int(_lib.lib().uaamg_poisson_kernel_launches(self.mMultigridHierarchy._h))

    def set_stream(self, stream_ptr: int | None) -> None:
        _lib.check(_lib.lib().uaamg_poisson_set_stream(self.mMultigridHierarchy._h, stream_ptr), "set_stream")
