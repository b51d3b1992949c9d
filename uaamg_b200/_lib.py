"""ctypes loader for libuaamg_b200.so (the C ABI declared in include/uaamg.h).

There is no CPU fallback: importing the solver classes without the built CUDA
library raises, so a missing extension can never silently turn into a
different code path.
"""
from __future__ import annotations

import contextlib
import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libuaamg_b200.so")

UAAMG_SUCCESS = 0
UAAMG_FAILED = 1


class UaamgError(RuntimeError):
    pass


class LeafGridC(C.Structure):
    _fields_ = [
        ("leaf_count", C.c_int64),
        ("origins", C.c_void_p),
        ("masks", C.c_void_p),
        ("values", C.c_void_p),
        ("components", C.c_int32),
        ("values_on_device", C.c_int32),
        ("background", C.c_float * 3),
    ]


class TuningC(C.Structure):
    _fields_ = [
        ("staged_min_leaves", C.c_int32),
        ("split_min_leaves", C.c_int32),
        ("pipe_min_leaves", C.c_int32),
        ("elem_ctas_per_sm", C.c_int32),
        ("bottom_cycle", C.c_int32),
    ]


class ServerOptionsC(C.Structure):
    _fields_ = [
        ("budget_bytes", C.c_int64),
        ("max_poisson", C.c_int32),
        ("max_viscosity", C.c_int32),
        ("admit_per_round", C.c_int32),
        ("batching", C.c_int32),
        ("keep_results", C.c_int32),
        ("pressure_tolerance", C.c_float),
        ("viscosity_tolerance", C.c_float),
    ]


class ServerStatsC(C.Structure):
    _fields_ = [(k, C.c_int64) for k in ("submitted", "queued", "resident", "done", "failed", "solves", "rounds",
                                         "batch_builds", "used_bytes", "peak_bytes", "pressure_solves",
                                         "pressure_busy_us")]


_lib = None

# (name, restype, argtypes) of every exported entry point in include/uaamg.h
vp, i32, i64, f32 = C.c_void_p, C.c_int, C.c_int64, C.c_float
pLG = C.POINTER(LeafGridC)
EXPORTS = [
    ("uaamg_poisson_create", i32, [pLG, pLG, f32, f32, C.POINTER(vp)]),
    ("uaamg_poisson_create_on_stream", i32, [pLG, pLG, f32, f32, vp, C.POINTER(vp)]),
    ("uaamg_poisson_create_with_rhs", i32, [pLG, pLG, pLG, pLG, pLG, pLG, f32, f32, vp, C.POINTER(vp)]),
    ("uaamg_poisson_solve_pcg_resident", i32, [vp, vp, C.POINTER(i32)]),
    ("uaamg_poisson_solve_pcg_resident_device", i32, [vp, vp, C.POINTER(i32)]),
    ("uaamg_poisson_solve_mg_resident", i32, [vp, vp, C.POINTER(i32)]),
    ("uaamg_poisson_copy_rhs", i32, [vp, vp]),
    ("uaamg_poisson_solve_fp64_reference", i32, [vp, vp, vp, C.c_double, i32, C.POINTER(i32),
                                                 C.POINTER(C.c_double)]),
    ("uaamg_packed3_from_vec3", i32, [pLG, vp, vp, vp]),
    ("uaamg_packed3_from_vec3_device", i32, [pLG, vp, vp, vp, vp]),
    ("uaamg_packed3_to_vec3_topology", i32, [pLG, pLG, pLG, C.POINTER(C.c_int64), vp, vp]),
    ("uaamg_packed3_to_vec3", i32, [pLG, pLG, pLG, vp]),
    ("uaamg_packed3_to_vec3_device", i32, [pLG, pLG, pLG, vp, vp]),
    ("uaamg_server_default_options", i32, [C.POINTER(ServerOptionsC)]),
    ("uaamg_server_create", i32, [C.POINTER(ServerOptionsC), C.POINTER(vp)]),
    ("uaamg_server_destroy", i32, [vp]),
    ("uaamg_server_submit_poisson", i32, [vp, pLG, pLG, pLG, f32, f32, i32, C.POINTER(C.c_int64)]),
    ("uaamg_server_submit_viscosity", i32, [vp, pLG, pLG, pLG, pLG, f32, f32, f32, i32, C.POINTER(C.c_int64)]),
    ("uaamg_server_push_velocity", i32, [vp, C.c_int64, pLG, pLG, pLG]),
    ("uaamg_server_wait", i32, [vp, C.c_int64, i32, C.c_double, C.POINTER(i32), C.POINTER(i32),
                                C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    ("uaamg_server_result", i32, [vp, C.c_int64, i32, C.POINTER(C.c_int64), vp]),
    ("uaamg_server_stats", i32, [vp, C.POINTER(ServerStatsC)]),
    ("uaamg_get_tuning", i32, [C.POINTER(TuningC)]),
    ("uaamg_set_tuning", i32, [C.POINTER(TuningC)]),
    ("uaamg_poisson_destroy", i32, [vp]),
    ("uaamg_poisson_set_smoother", i32, [vp, i32]),
    ("uaamg_poisson_set_max_iterations", i32, [vp, i32]),
    ("uaamg_poisson_set_relative_tolerance", i32, [vp, f32]),
    ("uaamg_poisson_iterations", i32, [vp]),
    ("uaamg_poisson_final_residual", f32, [vp]),
    ("uaamg_poisson_num_levels", i32, [vp]),
    ("uaamg_poisson_num_dof", i64, [vp, i32]),
    ("uaamg_poisson_leaf_count", i64, [vp, i32]),
    ("uaamg_poisson_dof_topology", i32, [vp, i32, vp, vp]),
    ("uaamg_poisson_dof_index", i32, [vp, i32, vp]),
    ("uaamg_poisson_build_rhs", i32, [vp, pLG, pLG, pLG, pLG, pLG, f32, vp]),
    ("uaamg_poisson_build_rhs_device", i32, [vp, pLG, pLG, pLG, pLG, pLG, f32, vp]),
    ("uaamg_face_weights", i32, [pLG, C.c_int64, vp, vp, vp]),
    ("uaamg_immerse_liquid_phi", i32, [pLG, pLG, C.c_float, vp]),
    ("uaamg_immerse_liquid_phi_device", i32, [pLG, pLG, C.c_float, vp, vp]),
    ("uaamg_extrapolate_channel", i32, [i32, C.c_int64, vp, vp, vp, C.c_int64, vp, vp]),
    ("uaamg_extrapolate_channel_device", i32, [i32, C.c_int64, vp, vp, vp, C.c_int64, vp, vp, vp]),
    ("uaamg_face_weights_device", i32, [pLG, C.c_int64, vp, vp, vp, vp]),
    ("uaamg_poisson_apply_pressure_gradient", i32, [vp, pLG, pLG, pLG, vp, f32, f32, i32, pLG, vp, vp, vp, vp]),
    ("uaamg_poisson_apply_pressure_gradient_device", i32,
     [vp, pLG, pLG, pLG, vp, f32, f32, i32, pLG, vp, vp, vp, vp]),
    ("uaamg_poisson_solve_pcg", i32, [vp, vp, vp, C.POINTER(C.c_int)]),
    ("uaamg_poisson_solve_pcg_device", i32, [vp, vp, vp, C.POINTER(C.c_int)]),
    ("uaamg_poisson_solve_mg", i32, [vp, vp, vp, C.POINTER(C.c_int)]),
    ("uaamg_poisson_solve_mg_device", i32, [vp, vp, vp, C.POINTER(C.c_int)]),
    ("uaamg_poisson_residual_norm_device", i32, [vp, vp, vp, vp, vp]),
    ("uaamg_poisson_residual_norm_noalloc", i32, [vp, vp, vp, vp, vp]),
    ("uaamg_poisson_level_apply", i32, [vp, i32, i32, f32, f32, vp, vp, vp]),
    ("uaamg_poisson_level_first_sweep", i32, [vp, i32, i32, f32, f32, vp, vp]),
    ("uaamg_poisson_level_restrict", i32, [vp, i32, vp, vp]),
    ("uaamg_poisson_level_prolongate", i32, [vp, i32, vp, vp, f32]),
    ("uaamg_poisson_level_coefficients", i32, [vp, i32, vp, vp, vp, vp, vp]),
    ("uaamg_poisson_coarsest_solve", i32, [vp, vp, vp]),
    ("uaamg_poisson_precondition", i32, [vp, vp, vp]),
    ("uaamg_poisson_profile_pcg", i32, [vp, vp, vp, i32, vp, vp, vp, C.POINTER(C.c_int)]),
    ("uaamg_poisson_set_stream", i32, [vp, vp]),
    ("uaamg_poisson_get_stream", i32, [vp, C.POINTER(vp)]),
    ("uaamg_poisson_set_graph_mode", i32, [vp, i32]),
    ("uaamg_poisson_kernel_launches", i64, [vp]),
    ("uaamg_solve_graph_cache_stats", i32, [C.POINTER(i64), C.POINTER(i64)]),
    ("uaamg_poisson_prepare_mixed", i32, [vp, i32, vp]),
    ("uaamg_poisson_set_residual_replacement", i32, [vp, i32]),
    ("uaamg_poisson_solve_pcg_mixed", i32, [vp, i32, vp, vp, C.POINTER(C.c_int)]),
    ("uaamg_poisson_solve_pcg_mixed_device", i32, [vp, i32, vp, vp, C.POINTER(C.c_int)]),
    ("uaamg_poisson_true_residual_fp64", i32, [vp, vp, vp, vp]),
    ("uaamg_poisson_profile_pcg_mixed", i32, [vp, i32, vp, vp, i32, vp, vp, vp, C.POINTER(C.c_int)]),
    ("uaamg_batch_create", i32, [i32, vp, C.POINTER(vp)]),
    ("uaamg_batch_destroy", i32, [vp]),
    ("uaamg_batch_size", i32, [vp]),
    ("uaamg_batch_set_smoother", i32, [vp, i32]),
    ("uaamg_batch_set_max_iterations", i32, [vp, i32]),
    ("uaamg_batch_set_relative_tolerance", i32, [vp, f32]),
    ("uaamg_batch_solve_pcg", i32, [vp, vp, vp, vp, vp]),
    ("uaamg_batch_solve_pcg_device", i32, [vp, vp, vp, vp, vp]),
    ("uaamg_batch_results", i32, [vp, vp, vp, vp]),
    ("uaamg_batch_set_stream", i32, [vp, vp]),
    ("uaamg_batch_get_stream", i32, [vp, C.POINTER(vp)]),
    ("uaamg_batch_set_graph_mode", i32, [vp, i32]),
    ("uaamg_batch_kernel_launches", i64, [vp]),
    ("uaamg_viscosity_create", i32, [pLG, pLG, pLG, f32, f32, f32, C.POINTER(vp)]),
    ("uaamg_viscosity_create_on_stream", i32, [pLG, pLG, pLG, f32, f32, f32, vp, C.POINTER(vp)]),
    ("uaamg_viscosity_destroy", i32, [vp]),
    ("uaamg_viscosity_set_max_iterations", i32, [vp, i32]),
    ("uaamg_viscosity_iterations", i32, [vp]),
    ("uaamg_viscosity_final_residual", f32, [vp]),
    ("uaamg_viscosity_num_levels", i32, [vp]),
    ("uaamg_viscosity_num_dof", i64, [vp, i32]),
    ("uaamg_viscosity_leaf_count", i64, [vp, i32]),
    ("uaamg_viscosity_topology", i32, [vp, i32, vp, vp]),
    ("uaamg_viscosity_dof_index", i32, [vp, i32, vp]),
    ("uaamg_viscosity_build_rhs", i32, [vp, pLG, pLG, pLG, pLG, vp]),
    ("uaamg_viscosity_build_rhs_device", i32, [vp, pLG, pLG, pLG, pLG, vp]),
    ("uaamg_viscosity_gather_velocity", i32, [vp, pLG, pLG, pLG, vp]),
    ("uaamg_viscosity_gather_velocity_device", i32, [vp, pLG, pLG, pLG, vp]),
    ("uaamg_viscosity_solve_pcg", i32, [vp, vp, vp, f32, C.POINTER(C.c_int)]),
    ("uaamg_viscosity_solve_pcg_device", i32, [vp, vp, vp, f32, C.POINTER(C.c_int)]),
    ("uaamg_viscosity_solve_velocity", i32, [vp, pLG, pLG, pLG, pLG, f32, vp, C.POINTER(C.c_int)]),
    ("uaamg_viscosity_level_apply", i32, [vp, i32, i32, i32, vp, vp, vp]),
    ("uaamg_viscosity_level_rbgs", i32, [vp, i32, i32, vp, vp]),
    ("uaamg_viscosity_level_restrict", i32, [vp, i32, vp, vp]),
    ("uaamg_viscosity_level_prolongate", i32, [vp, i32, vp, vp]),
    ("uaamg_viscosity_level_coefficients", i32, [vp, i32, vp, vp]),
    ("uaamg_viscosity_coarsest_solve", i32, [vp, vp, vp]),
    ("uaamg_viscosity_precondition", i32, [vp, vp, vp]),
    ("uaamg_viscosity_profile_pcg", i32, [vp, vp, vp, f32, i32, vp, vp, vp, C.POINTER(C.c_int)]),
    ("uaamg_viscosity_set_stream", i32, [vp, vp]),
    ("uaamg_viscosity_get_stream", i32, [vp, C.POINTER(vp)]),
    ("uaamg_viscosity_set_graph_mode", i32, [vp, i32]),
    ("uaamg_viscosity_kernel_launches", i64, [vp]),
    ("uaamg_last_error", C.c_char_p, []),
    ("uaamg_device_count", i32, []),
]


def lib():
    """Load the CUDA library (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise UaamgError(f"CUDA library not built: {LIB_PATH} (run __graft_entry__.build())")
        L = C.CDLL(LIB_PATH)
        for name, res, args in EXPORTS:
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(rc: int, what: str) -> int:
    if rc < 0:
        msg = lib().uaamg_last_error().decode(errors="replace")
        raise UaamgError(f"{what} failed ({rc}): {msg}")
    return rc


def ptr(a) -> int | None:
    """Address of a numpy array (host) or a torch tensor (host or device)."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        assert a.flags["C_CONTIGUOUS"]
        return a.ctypes.data
    return a.data_ptr()


# ----------------------------------------------------------------------------- torch stream ordering
# The library's handles run on streams of their own (non-blocking: not ordered
# with torch's streams).  The Python classes order every call that passes torch
# CUDA tensors with torch's current stream, so tensors torch is still writing
# are not read early and torch's kernels do not read outputs (or reuse input
# memory) before the library is done with them.
def is_cuda(*objs) -> bool:
    """True when an argument is, or holds (a LeafGrid's values, a list), a
    torch CUDA tensor."""
    for o in objs:
        if isinstance(o, (list, tuple)):
            if is_cuda(*o):
                return True
            continue
        if hasattr(o, "is_cuda"):  # a tensor (whose .values is a method, not data)
            if o.is_cuda:
                return True
            continue
        if getattr(getattr(o, "values", None), "is_cuda", False):  # a LeafGrid
            return True
    return False


def handle_stream(kind: str, h) -> int:
    """The stream a poisson / viscosity / batch handle's calls run on."""
    s = C.c_void_p()
    check(getattr(lib(), f"uaamg_{kind}_get_stream")(h, C.byref(s)), f"uaamg_{kind}_get_stream")
    return int(s.value or 0)


@contextlib.contextmanager
def torch_ordered(kind: str, h, *objs):
    """Around a call on handle ``h`` that reads or writes ``objs``: when one
    of them is a torch CUDA tensor, the handle's stream first waits for the
    work torch's current stream holds, and torch's current stream then waits
    for the call's work.  Both waits are device events; the host does not
    block."""
    if not is_cuda(*objs):
        yield
        return
    import torch
    cur = torch.cuda.current_stream()
    hs = handle_stream(kind, h)
    if hs == cur.cuda_stream:  # the handle runs on torch's stream: ordered already
        yield
        return
    ext = torch.cuda.ExternalStream(hs)
    ext.wait_stream(cur)
    try:
        yield
    finally:
        cur.wait_stream(ext)


def torch_inputs_ready(stream, *objs) -> None:
    """Before a call that takes torch CUDA tensors without a handle to order
    on (a creation on the new handle's own stream, a server submission):
    torch's current stream is synchronised, so the tensors are written."""
    if not stream and is_cuda(*objs):
        import torch
        torch.cuda.current_stream().synchronize()


def torch_after(kind: str, h, *objs) -> None:
    """After a creation that read torch CUDA tensors: torch's current stream
    waits for the new handle's stream (kernels still reading the inputs)."""
    if is_cuda(*objs):
        import torch
        cur = torch.cuda.current_stream()
        hs = handle_stream(kind, h)
        if hs != cur.cuda_stream:
            cur.wait_stream(torch.cuda.ExternalStream(hs))
