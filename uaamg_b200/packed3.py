"""Python mirror of packed_FloatGrid3 (SIMD_UAAMG/packed3grids.h, .cpp:11-83)
over the C ABI (uaamg_packed3_* in include/uaamg.h).

The reference's call sites hold a face velocity as a staggered Vec3fGrid and
hand the solvers its three channels: ``from_vec3`` splits it into three
FloatGrids with the vec3 grid's leaf topology (component c at active voxels,
the channel's background elsewhere), ``to_vec3`` merges three channels back
over the union of their topologies.  Grids are ``LeafGrid`` objects with numpy
values (host path) or torch CUDA tensors (device path, enqueued on torch's
current stream); the conversion runs in CUDA kernels either way.  Leaf grids
are in index space, so the reference's -dx/2 transform shift of each channel
has nothing to act on.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .grids import LeafGrid
from .poisson import _as_c


def _is_device(values) -> bool:
    return getattr(values, "is_cuda", False)


def _with_values(origins, masks, values, background) -> LeafGrid:
    """A LeafGrid around already-shaped values (numpy or a torch tensor)."""
    comps = 1 if values.ndim == 2 else 3
    g = LeafGrid(origins=np.zeros((0, 3), np.int32),
                 values=np.zeros((0, 512) if comps == 1 else (0, 512, 3), np.float32),
                 background=background)
    g.origins = np.ascontiguousarray(origins, dtype=np.int32).reshape(-1, 3)
    g.masks = None if masks is None else np.ascontiguousarray(masks, dtype=np.uint64).reshape(-1, 8)
    g.values = values
    return g


def _stream():
    import torch
    return torch.cuda.current_stream().cuda_stream


class packed_FloatGrid3:  # noqa: N801 - the reference's class name
    def __init__(self):
        self.v: list[LeafGrid | None] = [None, None, None]

    def from_vec3(self, in_v: LeafGrid, topologycopy: bool = False) -> None:
        """packed_FloatGrid3::from_vec3 (packed3grids.cpp:11-43)."""
        if in_v.components != 3:
            raise ValueError("from_vec3 takes a 3-component grid")
        n = in_v.leaf_count
        bg = np.asarray(in_v.background, np.float32).reshape(3)
        dev = _is_device(in_v.values)
        if dev:
            import torch
            outs = [torch.empty((n, 512), dtype=torch.float32, device=in_v.values.device) for _ in range(3)]
        else:
            outs = [np.empty((n, 512), np.float32) for _ in range(3)]
        if topologycopy:  # the channels' trees as built by the topology copy: every value the background
            for c in range(3):
                if dev:
                    outs[c].fill_(float(bg[c]))
                else:
                    outs[c].fill(bg[c])
        elif n:
            keep: list = []
            g = _as_c(in_v, keep)
            L = _lib.lib()
            if dev:
                _lib.check(L.uaamg_packed3_from_vec3_device(C.byref(g), *[o.data_ptr() for o in outs], _stream()),
                           "uaamg_packed3_from_vec3_device")
            else:
                _lib.check(L.uaamg_packed3_from_vec3(C.byref(g), *[o.ctypes.data for o in outs]),
                           "uaamg_packed3_from_vec3")
        self.v = [_with_values(in_v.origins, in_v.masks, outs[c], bg[c]) for c in range(3)]

    def to_vec3(self) -> LeafGrid:
        """packed_FloatGrid3::to_vec3 (packed3grids.cpp:46-83): background (0,0,0)."""
        if any(g is None for g in self.v):
            raise ValueError("to_vec3 needs all three channels")
        keep: list = []
        gs = [_as_c(g, keep) for g in self.v]
        L = _lib.lib()
        n = C.c_int64(0)
        _lib.check(L.uaamg_packed3_to_vec3_topology(*[C.byref(g) for g in gs], C.byref(n), None, None),
                   "uaamg_packed3_to_vec3_topology")
        org = np.zeros((n.value, 3), np.int32)
        masks = np.zeros((n.value, 8), np.uint64)
        if n.value:
            _lib.check(L.uaamg_packed3_to_vec3_topology(*[C.byref(g) for g in gs], C.byref(n), org.ctypes.data,
                                                        masks.ctypes.data), "uaamg_packed3_to_vec3_topology")
        filled = [g for g in self.v if g.leaf_count]
        dev = [_is_device(g.values) for g in filled]
        if dev and any(dev) != all(dev):
            raise ValueError("the channels' values must all be on the host or all on the device")
        if dev and all(dev):
            import torch
            vals = torch.empty((n.value, 512, 3), dtype=torch.float32, device=filled[0].values.device)
            if n.value:
                _lib.check(L.uaamg_packed3_to_vec3_device(*[C.byref(g) for g in gs], vals.data_ptr(), _stream()),
                           "uaamg_packed3_to_vec3_device")
        else:
            vals = np.zeros((n.value, 512, 3), np.float32)
            if n.value:
                _lib.check(L.uaamg_packed3_to_vec3(*[C.byref(g) for g in gs], vals.ctypes.data),
                           "uaamg_packed3_to_vec3")
        return _with_values(org, masks, vals, np.zeros(3, np.float32))

    def swap(self, other: "packed_FloatGrid3") -> None:
        self.v, other.v = other.v, self.v
