"""Python mirror of the reference's variational-viscosity interface over the C ABI.

Names and argument meaning follow SIMD_UAAMG/simd_viscosity3d.h:
``L_with_level.create_viscosity_matrix(viscosity, liquid_sdf, solid_sdf, dt,
rho)`` (h:85-88), ``get_zero_vec`` (h:139), ``build_rhs`` (h:126), the apply
family (``L_apply``, ``residual_apply``, ``Jacobi_apply``, ``XYZ_RBGS_apply``,
``ZYX_RBGS_apply``, ``restriction``, ``prolongation``, h:143-159) and
``simd_viscosity3d`` with ``m_max_iter`` / ``m_iteration`` / ``pcg_solve``
(h:273-318).  Grids are ``LeafGrid`` objects in one index space; vectors are
float32 [3, leaves, 512] arrays (numpy on the host, torch CUDA tensors for the
device path), zero off the DOFs.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .grids import LeafGrid
from .poisson import _as_c

MODES = {"normal": 0, "residual": 1, "jacobi": 2, "red_gs": 3, "black_gs": 4}
ARRAYS = ("diag", "invdiag", "neg_x", "neg_y", "neg_z", "T00", "T01", "T10", "T11")


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


class L_with_level:
    """Level 0 of the viscosity operator with its multigrid hierarchy on the GPU."""

    def __init__(self, handle: int, dt: float, rho: float, dx: float):
        self._h = handle
        self.m_dt = dt
        self.m_rho = rho
        self.m_dx = dx
        self.m_level = 0

    @staticmethod
    def create_viscosity_matrix(viscosity: LeafGrid, liquid_sdf: LeafGrid, solid_sdf: LeafGrid, dt: float,
                                rho: float, dx: float, stream: int | None = None) -> "L_with_level":
        """``stream``: a cudaStream_t (int) to build on; the handle keeps it."""
        L = _lib.lib()
        keep: list = []
        grids = (viscosity, liquid_sdf, solid_sdf)
        gs = [_as_c(g, keep) for g in grids]
        h = C.c_void_p()
        _lib.torch_inputs_ready(stream, grids)
        _lib.check(L.uaamg_viscosity_create_on_stream(*[C.byref(g) for g in gs], float(dt), float(rho), float(dx),
                                                      stream, C.byref(h)), "uaamg_viscosity_create")
        _lib.torch_after("viscosity", h.value, grids)
        return L_with_level(h.value, dt, rho, dx)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            try:
                _lib.lib().uaamg_viscosity_destroy(h)
            except Exception:  # interpreter shutdown: module globals already gone
                pass
            self._h = None

    # --- sizes and topology
    @property
    def m_ndof(self) -> int:
        return self.num_dof(0)

    def num_levels(self) -> int:
        return int(_lib.lib().uaamg_viscosity_num_levels(self._h))

    def num_dof(self, level: int = 0) -> int:
        return int(_lib.lib().uaamg_viscosity_num_dof(self._h, level))

    def leaf_count(self, level: int = 0) -> int:
        return int(_lib.lib().uaamg_viscosity_leaf_count(self._h, level))

    def topology(self, level: int = 0):
        n = self.leaf_count(level)
        o = np.zeros((n, 3), np.int32)
        m = np.zeros((3, n, 8), np.uint64)
        _lib.check(_lib.lib().uaamg_viscosity_topology(self._h, level, o.ctypes.data, m.ctypes.data), "topology")
        return o, m

    def dof_index(self, level: int = 0) -> np.ndarray:
        out = np.zeros((3, self.leaf_count(level), 512), np.int32)
        _lib.check(_lib.lib().uaamg_viscosity_dof_index(self._h, level, out.ctypes.data), "dof_index")
        return out

    def get_zero_vec(self, level: int = 0) -> np.ndarray:
        return np.zeros((3, self.leaf_count(level), 512), np.float32)

    # --- right-hand side and warm start
    def build_rhs(self, u: LeafGrid, v: LeafGrid, w: LeafGrid, solid_velocity: LeafGrid | None, out=None):
        keep: list = []
        gs = [_as_c(g, keep) for g in (u, v, w)]
        sv = C.byref(_as_c(solid_velocity, keep)) if solid_velocity is not None else None
        L = _lib.lib()
        if out is not None and not isinstance(out, np.ndarray):
            with _lib.torch_ordered("viscosity", self._h, out, u, v, w, solid_velocity):
                _lib.check(L.uaamg_viscosity_build_rhs_device(self._h, *[C.byref(g) for g in gs], sv,
                                                              out.data_ptr()), "build_rhs_device")
            return out
        _lib.torch_inputs_ready(None, u, v, w, solid_velocity)
        rhs = self.get_zero_vec() if out is None else out
        _lib.check(L.uaamg_viscosity_build_rhs(self._h, *[C.byref(g) for g in gs], sv, rhs.ctypes.data), "build_rhs")
        return rhs

    def gather_velocity(self, u: LeafGrid, v: LeafGrid, w: LeafGrid, out=None):
        """The velocity at every DOF: the warm start of the call site
        (FLIP_vdb.cpp:3188-3198)."""
        keep: list = []
        gs = [_as_c(g, keep) for g in (u, v, w)]
        L = _lib.lib()
        if out is not None and not isinstance(out, np.ndarray):
            with _lib.torch_ordered("viscosity", self._h, out, u, v, w):
                _lib.check(L.uaamg_viscosity_gather_velocity_device(self._h, *[C.byref(g) for g in gs],
                                                                    out.data_ptr()), "gather_velocity_device")
            return out
        _lib.torch_inputs_ready(None, u, v, w)
        x = self.get_zero_vec() if out is None else out
        _lib.check(L.uaamg_viscosity_gather_velocity(self._h, *[C.byref(g) for g in gs], x.ctypes.data),
                   "gather_velocity")
        return x

    def set_stream(self, stream_ptr) -> None:
        _lib.check(_lib.lib().uaamg_viscosity_set_stream(self._h, stream_ptr), "set_stream")

    # --- per-level operators
    def apply(self, level, mode, lhs, rhs=None, channel=0):
        out = np.zeros_like(lhs, dtype=np.float32)
        lhs = _f32(lhs)
        rhs = lhs if rhs is None else _f32(rhs)
        _lib.check(_lib.lib().uaamg_viscosity_level_apply(self._h, level, MODES[mode], int(channel), lhs.ctypes.data,
                                                          rhs.ctypes.data, out.ctypes.data), "level_apply")
        return out

    def L_apply(self, lhs, level=0):
        return self.apply(level, "normal", lhs)

    def residual_apply(self, lhs, rhs, level=0):
        return self.apply(level, "residual", lhs, rhs)

    def Jacobi_apply(self, lhs, rhs, level=0):
        return self.apply(level, "jacobi", lhs, rhs)

    def rbgs(self, level, lhs, rhs, order="xyz"):
        x = np.array(lhs, dtype=np.float32, copy=True)
        rhs = _f32(rhs)
        _lib.check(_lib.lib().uaamg_viscosity_level_rbgs(self._h, level, 0 if order == "xyz" else 1, x.ctypes.data,
                                                         rhs.ctypes.data), "level_rbgs")
        return x

    def XYZ_RBGS_apply(self, lhs, rhs, level=0):
        return self.rbgs(level, lhs, rhs, "xyz")

    def ZYX_RBGS_apply(self, lhs, rhs, level=0):
        return self.rbgs(level, lhs, rhs, "zyx")

    def restriction(self, fine, fine_level=0):
        out = np.zeros((3, self.leaf_count(fine_level + 1), 512), np.float32)
        fine = _f32(fine)
        _lib.check(_lib.lib().uaamg_viscosity_level_restrict(self._h, fine_level, fine.ctypes.data, out.ctypes.data),
                   "restrict")
        return out

    def prolongation(self, coarse, fine, fine_level=0):
        out = np.array(fine, dtype=np.float32, copy=True)
        coarse = _f32(coarse)
        _lib.check(_lib.lib().uaamg_viscosity_level_prolongate(self._h, fine_level, coarse.ctypes.data,
                                                               out.ctypes.data), "prolongate")
        return out

    def coefficients(self, level=0):
        """([3, 9, leaves, 512] effective values, [leaves] trimmed bits)."""
        n = self.leaf_count(level)
        coef = np.zeros((3, 9, n, 512), np.float32)
        trim = np.zeros(max(n, 1), np.uint32)
        _lib.check(_lib.lib().uaamg_viscosity_level_coefficients(self._h, level, coef.ctypes.data, trim.ctypes.data),
                   "coefficients")
        return coef, trim[:n]

    def solve_exact(self, rhs):
        out = np.zeros_like(rhs, dtype=np.float32)
        rhs = _f32(rhs)
        _lib.check(_lib.lib().uaamg_viscosity_coarsest_solve(self._h, rhs.ctypes.data, out.ctypes.data),
                   "coarsest_solve")
        return out


class simd_viscosity3d:
    """PCG with the mu-cycle (mu = 2, two red-black Gauss-Seidel sweeps) as
    preconditioner (simd_viscosity3d.h:273-318)."""

    SUCCESS = 0
    FAILED = 1

    def __init__(self, level0: L_with_level, liquid_velocity=None, solid_velocity=None):
        """simd_viscosity3d(level0, liquid_velocity, solid_velocity) (.cpp:3660-3689):
        liquid_velocity is a (u, v, w) triple of LeafGrids."""
        self.level0 = level0
        self.m_max_iter = 100
        self.m_iteration = 0
        self.use_graph = True
        self.m_rhs = None
        if liquid_velocity is not None:
            u, v, w = liquid_velocity
            self.m_rhs = level0.build_rhs(u, v, w, solid_velocity)

    def _configure(self):
        L = _lib.lib()
        h = self.level0._h
        _lib.check(L.uaamg_viscosity_set_max_iterations(h, int(self.m_max_iter)), "set_max_iterations")
        mode = self.use_graph if isinstance(self.use_graph, int) and not isinstance(self.use_graph, bool) \
            else (1 if self.use_graph else 0)
        _lib.check(L.uaamg_viscosity_set_graph_mode(h, mode), "set_graph_mode")
        return L, h

    def pcg_solve(self, in_lhs, tolerance: float, rhs=None) -> int:
        """Solves in place from the initial guess in_lhs (numpy or torch CUDA).
        Returns SUCCESS when the stopping test held, FAILED when the loop
        returned at m_max_iter - 1."""
        L, h = self._configure()
        rhs = self.m_rhs if rhs is None else rhs
        it = C.c_int(0)
        if isinstance(in_lhs, np.ndarray):
            assert in_lhs.dtype == np.float32 and in_lhs.flags["C_CONTIGUOUS"]
            rhs = _f32(rhs)
            rc = L.uaamg_viscosity_solve_pcg(h, in_lhs.ctypes.data, rhs.ctypes.data, float(tolerance), C.byref(it))
        else:
            with _lib.torch_ordered("viscosity", h, in_lhs, rhs):
                rc = L.uaamg_viscosity_solve_pcg_device(h, in_lhs.data_ptr(), rhs.data_ptr(), float(tolerance),
                                                        C.byref(it))
        _lib.check(rc, "pcg_solve")
        self.m_iteration = int(it.value)
        return int(rc)

    def solve_velocity(self, u: LeafGrid, v: LeafGrid, w: LeafGrid, solid_velocity: LeafGrid | None,
                       tolerance: float, out: np.ndarray | None = None):
        """The call site's viscosity step in one C-ABI call (FLIP_vdb.cpp:
        3178-3219; uaamg_viscosity_solve_velocity): the rhs and the warm start
        from the velocity, uploaded once, then PCG.  Returns (status, the solved
        DOF velocity [3, n, 512] in ``out`` or a new array); identical to
        build_rhs + gather_velocity + pcg_solve."""
        L, h = self._configure()
        keep: list = []
        gs = [_as_c(g, keep) for g in (u, v, w)]
        sv = C.byref(_as_c(solid_velocity, keep)) if solid_velocity is not None else None
        x = self.level0.get_zero_vec() if out is None else out
        assert x.dtype == np.float32 and x.flags["C_CONTIGUOUS"]
        it = C.c_int(0)
        _lib.torch_inputs_ready(None, u, v, w, solid_velocity)
        rc = L.uaamg_viscosity_solve_velocity(h, *[C.byref(g) for g in gs], sv, float(tolerance), x.ctypes.data,
                                              C.byref(it))
        _lib.check(rc, "solve_velocity")
        self.m_iteration = int(it.value)
        return int(rc), x

    def precondition(self, r: np.ndarray) -> np.ndarray:
        L, h = self._configure()
        z = np.zeros_like(r, dtype=np.float32)
        r = _f32(r)
        _lib.check(L.uaamg_viscosity_precondition(h, r.ctypes.data, z.ctypes.data), "precondition")
        return z

    def profile_pcg(self, d_lhs, d_rhs, tolerance: float, max_classes: int = 96):
        L, h = self._configure()
        names = C.create_string_buffer(64 * max_classes)
        ms = np.zeros(max_classes, np.float64)
        cnt = np.zeros(max_classes, np.int64)
        nc = C.c_int(0)
        with _lib.torch_ordered("viscosity", h, d_lhs, d_rhs):
            rc = L.uaamg_viscosity_profile_pcg(h, d_lhs.data_ptr(), d_rhs.data_ptr(), float(tolerance), max_classes,
                                               C.addressof(names), ms.ctypes.data, cnt.ctypes.data, C.byref(nc))
        _lib.check(rc, "profile_pcg")
        self.m_iteration = int(L.uaamg_viscosity_iterations(h))
        raw = names.raw
        out = {}
        for k in range(nc.value):
            nm = raw[64 * k: 64 * k + 64].split(b"\0", 1)[0].decode()
            out[nm] = (float(ms[k]), int(cnt[k]))
        return out

    @property
    def final_residual(self) -> float:
        return float(_lib.lib().uaamg_viscosity_final_residual(self.level0._h))

    @property
    def kernel_launches(self) -> int:
        return int(_lib.lib().uaamg_viscosity_kernel_launches(self.level0._h))
