"""ctypes binding of the CPU oracle (liboracle.so built from poisson_oracle.c and
viscosity_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
cpu_baseline / reference arm of bench.py, never by the uaamg_b200 package.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

SMOOTHERS = {"scheduled_jacobi": 0, "weighted_jacobi": 1, "rbgs": 2, "spai0": 3}
MODES = {"jacobi": 0, "residual": 1, "laplacian": 2, "red_gs": 3, "black_gs": 4, "spai0": 5}

f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
u64p = np.ctypeslib.ndpointer(dtype=np.uint64, flags="C_CONTIGUOUS")
u8p = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")


def build() -> str:
    path = os.path.join(_HERE, "liboracle.so")
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    if os.path.isdir(REFERENCE_ROOT):  # the reference's own helpers, where its sources are present
        subprocess.run(["make", "-s", "-C", _HERE, "ref", f"REF={REFERENCE_ROOT}"], check=True)
    return path


# Where build() finds the reference's sources; the built _ref/ libraries travel
# without them.
REFERENCE_ROOT = os.environ.get("UAAMG_REFERENCE_ROOT", "/root/reference")
REF_LIB = os.path.join(_HERE, "_ref", "libuaamg_ref.so")
REF_LIB_NATIVE = os.path.join(_HERE, "_ref", "libuaamg_ref_native.so")


def ref_lib(native: bool = False):
    """The reference's scalar helpers built from its own sources (None when
    oracle/_ref was not built)."""
    path = REF_LIB_NATIVE if native else REF_LIB
    if not os.path.exists(path):
        return None
    L = C.CDLL(path)
    L.ref_fraction_inside2.argtypes = [C.c_float] * 2
    L.ref_fraction_inside4.argtypes = [C.c_float] * 4
    L.ref_volume_fraction_tet.argtypes = [C.c_float] * 4
    L.ref_volume_fraction_cube.argtypes = [C.c_float] * 8
    for f in ("ref_fraction_inside2", "ref_fraction_inside4", "ref_volume_fraction_tet", "ref_volume_fraction_cube"):
        getattr(L, f).restype = C.c_float
    return L


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        vp = C.c_void_p
        L.orc_poisson_create.restype = vp
        L.orc_poisson_create.argtypes = [C.c_int64, i32p, u64p, f32p, C.c_float,
                                         C.c_int64, i32p, f32p, f32p, C.c_float, C.c_float, C.c_int]
        L.orc_poisson_free.argtypes = [vp]
        for fn in ("orc_num_levels",):
            getattr(L, fn).argtypes = [vp]
        L.orc_level_leaf_count.argtypes = [vp, C.c_int]
        L.orc_level_ndof.argtypes = [vp, C.c_int]
        L.orc_level_topology.argtypes = [vp, C.c_int, i32p, u64p]
        L.orc_level_coefficients.argtypes = [vp, C.c_int, f32p, f32p, f32p, f32p, u8p]
        L.orc_level_defaults.argtypes = [vp, C.c_int, f32p]
        g = [C.c_int64, i32p, f32p]
        L.orc_build_rhs.argtypes = [vp, *g, f32p, *g, C.c_float, *g, C.c_float, *g, C.c_float,
                                    *g, f32p, f32p]
        L.orc_apply.argtypes = [vp, C.c_int, C.c_int, C.c_float, C.c_float, f32p, f32p, f32p]
        L.orc_first_jacobi.argtypes = [vp, C.c_int, C.c_float, f32p, f32p]
        L.orc_first_spai0.argtypes = [vp, C.c_int, f32p, f32p]
        L.orc_first_rbgs.argtypes = [vp, C.c_int, C.c_int, C.c_float, f32p, f32p]
        L.orc_restrict.argtypes = [vp, C.c_int, f32p, f32p]
        L.orc_prolongate.argtypes = [vp, C.c_int, f32p, f32p, C.c_float]
        L.orc_coarsest_solve.argtypes = [vp, f32p, f32p]
        L.orc_precondition.argtypes = [vp, C.c_int, f32p, f32p]
        sig = [vp, f32p, f32p, C.c_float, C.c_int, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_float)]
        L.orc_solve_pcg.argtypes = sig
        L.orc_solve_mg.argtypes = sig
        L.orc_abs_max.argtypes = [vp, C.c_int, f32p]
        L.orc_abs_max.restype = C.c_float
        L.orc_dot.argtypes = [vp, C.c_int, f32p, f32p]
        L.orc_dot.restype = C.c_float
        L.orc_triplets.argtypes = [vp, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
        L.orc_triplets.restype = C.c_int64
        L.orc_dof_index.argtypes = [vp, C.c_int, i32p]
        L.orc_set_threads.argtypes = [C.c_int]
        L.orc_set_simd.argtypes = [C.c_int]
        # variational viscosity
        L.orc_visc_create.restype = vp
        L.orc_visc_create.argtypes = [C.c_int64, i32p, u64p, f32p, C.c_float,
                                      C.c_int64, i32p, f32p, C.c_float,
                                      C.c_int64, i32p, f32p, C.c_float,
                                      C.c_float, C.c_float, C.c_float, C.c_int]
        L.orc_visc_free.argtypes = [vp]
        L.orc_visc_num_levels.argtypes = [vp]
        for fn in ("orc_visc_leaf_count", "orc_visc_ndof"):
            getattr(L, fn).argtypes = [vp, C.c_int]
        L.orc_visc_topology.argtypes = [vp, C.c_int, i32p, u64p]
        L.orc_visc_coefficients.argtypes = [vp, C.c_int, f32p, C.c_void_p]
        L.orc_visc_defaults.argtypes = [vp, C.c_int, f32p]
        L.orc_visc_dof_index.argtypes = [vp, C.c_int, i32p]
        L.orc_visc_triplets.argtypes = [vp, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
        L.orc_visc_triplets.restype = C.c_int64
        L.orc_visc_build_rhs.argtypes = [vp, *g, C.c_float, *g, C.c_float, *g, C.c_float, *g, f32p, f32p]
        L.orc_visc_apply.argtypes = [vp, C.c_int, C.c_int, C.c_int, f32p, f32p, f32p]
        L.orc_visc_rbgs.argtypes = [vp, C.c_int, C.c_int, f32p, f32p]
        L.orc_visc_restrict.argtypes = [vp, C.c_int, f32p, f32p]
        L.orc_visc_prolongate.argtypes = [vp, C.c_int, f32p, f32p]
        L.orc_visc_coarsest_solve.argtypes = [vp, f32p, f32p]
        L.orc_visc_set_coarsest_order.argtypes = [vp, C.c_int]
        L.orc_visc_precondition.argtypes = [vp, f32p, f32p]
        L.orc_visc_pcg.argtypes = [vp, f32p, f32p, C.c_float, C.c_int, C.POINTER(C.c_int),
                                   C.POINTER(C.c_float)]
        L.orc_visc_abs_max.argtypes = [vp, C.c_int, f32p]
        L.orc_visc_abs_max.restype = C.c_float
        L.orc_visc_dot.argtypes = [vp, C.c_int, f32p, f32p]
        L.orc_visc_dot.restype = C.c_float
        L.orc_fraction_inside4.argtypes = [C.c_float] * 4
        L.orc_fraction_inside4.restype = C.c_float
        L.orc_fraction_inside2.argtypes = [C.c_float] * 2
        L.orc_fraction_inside2.restype = C.c_float
        L.orc_tet_fraction.argtypes = [C.c_float] * 4
        L.orc_tet_fraction.restype = C.c_float
        L.orc_cube_fraction.argtypes = [C.c_float] * 8
        L.orc_cube_fraction.restype = C.c_float
        L.orc_face_weights.argtypes = [C.c_int64, i32p, f32p, C.c_float, C.c_int64, i32p, vp, f32p]
        L.orc_pressure_gradient.argtypes = [C.c_int64, i32p, f32p, C.c_float, C.c_int64, i32p, f32p, f32p,
                                            C.c_int64, i32p, f32p, f32p, C.c_int64, i32p, u64p, f32p,
                                            C.c_float, C.c_float, C.c_float, C.c_int,
                                            C.c_int64, i32p, vp, f32p, f32p, u64p, f32p, f32p]
        L.orc_extrapolate_channel.argtypes = [C.c_int, C.c_int64, i32p, f32p, u64p, C.c_int64, i32p, u64p]
        L.orc_immerse_liquid_phi.argtypes = [C.c_int64, i32p, f32p, C.c_float, C.c_int64, i32p, vp, f32p,
                                             C.c_float, C.c_float, f32p]
        _LIB = L
    return _LIB


def _grid_args(g):
    return (g.leaf_count, g.origins, np.ascontiguousarray(g.values.reshape(-1), dtype=np.float32))


class OraclePoisson:
    """Oracle hierarchy for one Poisson system (level 0 + coarse levels)."""

    def __init__(self, phi, face_weights, dt, dx, hierarchy=True):
        L = lib()
        self._h = L.orc_poisson_create(phi.leaf_count, phi.origins, phi.masks,
                                       np.ascontiguousarray(phi.values.reshape(-1)),
                                       float(phi.background[0]), *_grid_args(face_weights),
                                       face_weights.background, float(dt), float(dx),
                                       1 if hierarchy else 0)
        self.num_levels = L.orc_num_levels(self._h)

    def __del__(self):
        if getattr(self, "_h", None):
            lib().orc_poisson_free(self._h)
            self._h = None

    def leaf_count(self, level=0):
        return lib().orc_level_leaf_count(self._h, level)

    def ndof(self, level=0):
        return lib().orc_level_ndof(self._h, level)

    def topology(self, level=0):
        n = self.leaf_count(level)
        o = np.zeros((n, 3), np.int32); m = np.zeros((n, 8), np.uint64)
        lib().orc_level_topology(self._h, level, o, m)
        return o, m

    def coefficients(self, level=0):
        n = self.leaf_count(level)
        arr = [np.zeros((n, 512), np.float32) for _ in range(4)]
        flags = np.zeros(n, np.uint8)
        lib().orc_level_coefficients(self._h, level, *arr, flags)
        return arr, flags

    def defaults(self, level=0):
        d = np.zeros(4, np.float32)
        lib().orc_level_defaults(self._h, level, d)
        return d

    def zeros(self, level=0):
        return np.zeros((self.leaf_count(level), 512), np.float32)

    def build_rhs(self, face_weights, vx, vy, vz, solid_velocity):
        out = self.zeros(0)
        lib().orc_build_rhs(self._h, *_grid_args(face_weights), face_weights.background,
                            *_grid_args(vx), float(vx.background[0]),
                            *_grid_args(vy), float(vy.background[0]),
                            *_grid_args(vz), float(vz.background[0]),
                            *_grid_args(solid_velocity), solid_velocity.background, out)
        return out

    def apply(self, level, mode, lhs, rhs=None, weight=6.0 / 7.0, w_sor=1.2):
        out = self.zeros(level)
        rhs = lhs if rhs is None else rhs
        lib().orc_apply(self._h, level, MODES[mode], weight, w_sor,
                        np.ascontiguousarray(lhs, np.float32), np.ascontiguousarray(rhs, np.float32), out)
        return out

    def first_jacobi(self, level, rhs, weight):
        out = self.zeros(level)
        lib().orc_first_jacobi(self._h, level, weight, np.ascontiguousarray(rhs, np.float32), out)
        return out

    def first_spai0(self, level, rhs):
        out = self.zeros(level)
        lib().orc_first_spai0(self._h, level, np.ascontiguousarray(rhs, np.float32), out)
        return out

    def first_rbgs(self, level, rhs, red_first=True, w_sor=1.2):
        out = self.zeros(level)
        lib().orc_first_rbgs(self._h, level, 1 if red_first else 0, w_sor,
                             np.ascontiguousarray(rhs, np.float32), out)
        return out

    def restrict(self, fine_level, fine):
        out = self.zeros(fine_level + 1)
        lib().orc_restrict(self._h, fine_level, np.ascontiguousarray(fine, np.float32), out)
        return out

    def prolongate(self, fine_level, coarse, fine, alpha=1.0):
        out = np.array(fine, dtype=np.float32, copy=True)
        lib().orc_prolongate(self._h, fine_level, np.ascontiguousarray(coarse, np.float32), out, alpha)
        return out

    def coarsest_solve(self, rhs):
        out = self.zeros(self.num_levels - 1)
        lib().orc_coarsest_solve(self._h, np.ascontiguousarray(rhs, np.float32), out)
        return out

    def precondition(self, r, smoother="scheduled_jacobi"):
        z = self.zeros(0)
        lib().orc_precondition(self._h, SMOOTHERS[smoother], np.ascontiguousarray(r, np.float32), z)
        return z

    def _solve(self, fn, x, b, tol, max_iter, smoother):
        x = np.array(x, dtype=np.float32, copy=True)
        it = C.c_int(0); res = C.c_float(0)
        st = fn(self._h, x, np.ascontiguousarray(b, np.float32), float(tol), int(max_iter),
                SMOOTHERS[smoother], C.byref(it), C.byref(res))
        return x, int(st), int(it.value), float(res.value)

    def solve_pcg(self, x, b, tol=1e-7, max_iter=100, smoother="scheduled_jacobi"):
        return self._solve(lib().orc_solve_pcg, x, b, tol, max_iter, smoother)

    def solve_mg(self, x, b, tol=1e-7, max_iter=100, smoother="scheduled_jacobi"):
        return self._solve(lib().orc_solve_mg, x, b, tol, max_iter, smoother)

    def abs_max(self, v, level=0):
        return float(lib().orc_abs_max(self._h, level, np.ascontiguousarray(v, np.float32)))

    def dot(self, a, b, level=0):
        return float(lib().orc_dot(self._h, level, np.ascontiguousarray(a, np.float32),
                                   np.ascontiguousarray(b, np.float32)))

    def triplets(self, level):
        n = lib().orc_triplets(self._h, level, None, None, None)
        r = np.zeros(n, np.int32); c = np.zeros(n, np.int32); v = np.zeros(n, np.float32)
        lib().orc_triplets(self._h, level, r.ctypes.data, c.ctypes.data, v.ctypes.data)
        return r, c, v

    def dof_index(self, level=0):
        out = np.zeros((self.leaf_count(level), 512), np.int32)
        lib().orc_dof_index(self._h, level, out)
        return out


VMODES = {"normal": 0, "residual": 1, "jacobi": 2, "red_gs": 3, "black_gs": 4}
VARRAYS = ("diag", "invdiag", "neg_x", "neg_y", "neg_z", "T00", "T01", "T10", "T11")


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


class OracleViscosity:
    """Oracle hierarchy for one variational viscosity system.  Vectors are
    float32 [3, leaf, 512] over a level's leaf set (0 at non-DOF voxels)."""

    def __init__(self, liquid_phi, solid_phi, viscosity, dt, rho, dx, hierarchy=True):
        L = lib()
        self._h = L.orc_visc_create(
            liquid_phi.leaf_count, liquid_phi.origins, liquid_phi.masks, _f32(liquid_phi.values.reshape(-1)),
            float(liquid_phi.background[0]),
            *_grid_args(solid_phi), float(solid_phi.background[0]),
            *_grid_args(viscosity), float(viscosity.background[0]),
            float(dt), float(rho), float(dx), 1 if hierarchy else 0)
        self.num_levels = L.orc_visc_num_levels(self._h)

    def __del__(self):
        if getattr(self, "_h", None):
            lib().orc_visc_free(self._h)
            self._h = None

    def leaf_count(self, level=0):
        return lib().orc_visc_leaf_count(self._h, level)

    def ndof(self, level=0):
        return lib().orc_visc_ndof(self._h, level)

    def zeros(self, level=0):
        return np.zeros((3, self.leaf_count(level), 512), np.float32)

    def topology(self, level=0):
        n = self.leaf_count(level)
        o = np.zeros((n, 3), np.int32)
        m = np.zeros((3, n, 8), np.uint64)
        lib().orc_visc_topology(self._h, level, o, m)
        return o, m

    def coefficients(self, level=0):
        """([3, 9, leaf, 512] effective values, [leaf] trimmed bits)."""
        n = self.leaf_count(level)
        coef = np.zeros((3, 9, n, 512), np.float32)
        trim = np.zeros(max(n, 1), np.uint32)
        lib().orc_visc_coefficients(self._h, level, coef, trim.ctypes.data)
        return coef, trim[:n]

    def defaults(self, level=0):
        d = np.zeros(27, np.float32)
        lib().orc_visc_defaults(self._h, level, d)
        return d.reshape(3, 9)

    def dof_index(self, level=0):
        out = np.zeros((3, self.leaf_count(level), 512), np.int32)
        lib().orc_visc_dof_index(self._h, level, out)
        return out

    def triplets(self, level):
        n = lib().orc_visc_triplets(self._h, level, None, None, None)
        r = np.zeros(n, np.int32); c = np.zeros(n, np.int32); v = np.zeros(n, np.float32)
        lib().orc_visc_triplets(self._h, level, r.ctypes.data, c.ctypes.data, v.ctypes.data)
        return r, c, v

    def build_rhs(self, u, v, w, solid_velocity):
        out = self.zeros(0)
        lib().orc_visc_build_rhs(self._h, *_grid_args(u), float(u.background[0]),
                                 *_grid_args(v), float(v.background[0]),
                                 *_grid_args(w), float(w.background[0]),
                                 *_grid_args(solid_velocity), _f32(solid_velocity.background), out)
        return out

    def apply(self, level, mode, lhs, rhs=None, channel=0):
        """normal/residual/jacobi: returns a new vector; red_gs/black_gs:
        returns a copy of lhs with channel ``channel`` updated."""
        rhs = lhs if rhs is None else rhs
        if mode in ("red_gs", "black_gs"):
            out = np.array(lhs, dtype=np.float32, copy=True)
        else:
            out = self.zeros(level)
        lib().orc_visc_apply(self._h, level, VMODES[mode], int(channel), _f32(lhs), _f32(rhs), out)
        return out

    def rbgs(self, level, lhs, rhs, order="xyz"):
        out = np.array(lhs, dtype=np.float32, copy=True)
        lib().orc_visc_rbgs(self._h, level, 0 if order == "xyz" else 1, out, _f32(rhs))
        return out

    def restrict(self, fine_level, fine):
        out = self.zeros(fine_level + 1)
        lib().orc_visc_restrict(self._h, fine_level, _f32(fine), out)
        return out

    def prolongate(self, fine_level, coarse, fine):
        out = np.array(fine, dtype=np.float32, copy=True)
        lib().orc_visc_prolongate(self._h, fine_level, _f32(coarse), out)
        return out

    ORDER_KERNEL, ORDER_SEQUENTIAL = 0, 1

    def set_coarsest_order(self, order: int):
        """Summation order of the coarsest CG: ORDER_KERNEL (the CUDA kernel's
        tree order, the default) or ORDER_SEQUENTIAL (plain sequential sums)."""
        lib().orc_visc_set_coarsest_order(self._h, int(order))

    def coarsest_solve(self, rhs):
        out = self.zeros(self.num_levels - 1)
        lib().orc_visc_coarsest_solve(self._h, _f32(rhs), out)
        return out

    def precondition(self, r):
        z = self.zeros(0)
        lib().orc_visc_precondition(self._h, _f32(r), z)
        return z

    def solve_pcg(self, x, b, tol=1e-6, max_iter=100):
        x = np.array(x, dtype=np.float32, copy=True)
        it = C.c_int(0); res = C.c_float(0)
        st = lib().orc_visc_pcg(self._h, x, _f32(b), float(tol), int(max_iter), C.byref(it), C.byref(res))
        return x, int(st), int(it.value), float(res.value)

    def abs_max(self, v, level=0):
        return float(lib().orc_visc_abs_max(self._h, level, _f32(v)))

    def dot(self, a, b, level=0):
        return float(lib().orc_visc_dot(self._h, level, _f32(a), _f32(b)))


def set_simd(on: bool) -> None:
    """The Poisson applier's AVX2 path (default) or the scalar per-voxel path
    (the same bits)."""
    lib().orc_set_simd(1 if on else 0)


def set_threads(n: int) -> None:
    lib().orc_set_threads(int(n))


# ---------------------------------------------------------------------------
# The steps either side of the pressure solve (projection_oracle.c)

def fraction_inside4(bl, br, tl, tr) -> float:
    """fraction_inside(bl, br, tl, tr) (levelset_util.cpp:23-100)."""
    return float(lib().orc_fraction_inside4(float(bl), float(br), float(tl), float(tr)))


def face_weights(solid_sdf, origins, masks=None) -> np.ndarray:
    """calculate_face_weights (FLIP_vdb.cpp:2669-2752) on the given topology:
    float32 [leaf][512][3]."""
    org = np.ascontiguousarray(origins, dtype=np.int32)
    n = org.shape[0]
    out = np.zeros((n, 512, 3), np.float32)
    m = None if masks is None else np.ascontiguousarray(masks, dtype=np.uint64)
    lib().orc_face_weights(*_grid_args(solid_sdf), float(solid_sdf.background.reshape(-1)[0]), n,
                           org.reshape(-1), None if m is None else m.ctypes.data, out.reshape(-1))
    return out


def pressure_gradient(liquid_phi, face_weights, solid_velocity, p_origins, p_masks, pressure, dt, dx, friction,
                      channel, velocity):
    """apply_pressure_gradient (FLIP_vdb.cpp:2571-2667) for one channel.  The
    pressure is given on its leaves (origins, DOF masks, values [leaf][512]).
    Returns (velocity, masks, update, reflected)."""
    v = np.ascontiguousarray(velocity.values.reshape(-1), dtype=np.float32)
    n = velocity.leaf_count
    vm = None if velocity.masks is None else np.ascontiguousarray(velocity.masks, dtype=np.uint64)
    out = np.zeros(n * 512, np.float32)
    upd = np.zeros(n * 512, np.float32)
    refl = np.zeros(n * 512, np.float32)
    mask = np.zeros(n * 8, np.uint64)
    lib().orc_pressure_gradient(
        *_grid_args(liquid_phi), float(liquid_phi.background.reshape(-1)[0]),
        *_grid_args(face_weights), _f32(face_weights.background),
        *_grid_args(solid_velocity), _f32(solid_velocity.background),
        int(np.asarray(p_origins).shape[0]), np.ascontiguousarray(p_origins, dtype=np.int32).reshape(-1),
        np.ascontiguousarray(p_masks, dtype=np.uint64).reshape(-1),
        np.ascontiguousarray(pressure, dtype=np.float32).reshape(-1),
        float(dt), float(dx), float(friction), int(channel),
        n, np.ascontiguousarray(velocity.origins, dtype=np.int32).reshape(-1),
        None if vm is None else vm.ctypes.data, v, out, mask, upd, refl)
    return out.reshape(n, 512), mask.reshape(n, 8), upd.reshape(n, 512), refl.reshape(n, 512)


def extrapolate_channel(n_layer, out_origins, values, masks, fill_leaf, fill_masks):
    """union_extrapolate's layers (vdb_velocity_extrapolator.cpp:611-659) for
    one channel; returns the updated (values, masks)."""
    org = np.ascontiguousarray(out_origins, dtype=np.int32).reshape(-1)
    v = np.array(values, dtype=np.float32, order="C").reshape(-1)
    m = np.array(masks, dtype=np.uint64, order="C").reshape(-1)
    fl = np.ascontiguousarray(fill_leaf, dtype=np.int32).reshape(-1)
    fm = np.ascontiguousarray(fill_masks, dtype=np.uint64).reshape(-1)
    n_out = org.size // 3
    lib().orc_extrapolate_channel(int(n_layer), n_out, org, v, m, fl.size, fl, fm)
    return v.reshape(n_out, 512), m.reshape(n_out, 8)


def immerse_liquid_phi(liquid_phi, solid_sdf, dx):
    """immerse_liquid_phi_in_solids' value passes (FLIP_vdb.cpp:2856-2938) on
    the liquid SDF's own leaves: float32 [leaf][512]."""
    n = liquid_phi.leaf_count
    out = np.zeros((n, 512), np.float32)
    m = None if liquid_phi.masks is None else np.ascontiguousarray(liquid_phi.masks, dtype=np.uint64)
    lib().orc_immerse_liquid_phi(*_grid_args(solid_sdf), float(solid_sdf.background.reshape(-1)[0]), n,
                                 np.ascontiguousarray(liquid_phi.origins, dtype=np.int32).reshape(-1),
                                 None if m is None else m.ctypes.data,
                                 np.ascontiguousarray(liquid_phi.values.reshape(-1), dtype=np.float32),
                                 float(liquid_phi.background.reshape(-1)[0]), float(dx), out.reshape(-1))
    return out
