"""The steps either side of the pressure solve in a FLIP projection, on the GPU.

``calculate_face_weights`` produces the solid face fractions the Poisson
matrix reads (FLIP_Solver_OpenVDB::calculate_face_weights,
FLIP_vdb/FLIP_vdb.cpp:2669-2752); ``apply_pressure_gradient`` applies the
solved pressure to a velocity channel (FLIP_Solver_OpenVDB::
apply_pressure_gradient, FLIP_vdb.cpp:2571-2667).  Both run through the C ABI
(``uaamg_face_weights``, ``uaamg_poisson_apply_pressure_gradient``);
``face_weight_topology`` computes, on the host, the output topology the
reference gives the face weights: the liquid SDF's active voxels dilated by
two voxels over the 26-neighbourhood (FLIP_vdb.cpp:2672-2675).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .grids import LeafGrid, offsets_xyz, pack_masks, unpack_masks
from .poisson import LaplacianWithLevel, _as_c

# the FLIP solver's default boundary_friction_coefficient (FLIP_vdb.cpp:1886)
DEFAULT_FRICTION = 0.0


def face_weight_topology(liquid_phi: LeafGrid, layers: int = 2) -> tuple[np.ndarray, np.ndarray]:
    """Leaves (origins [n, 3]) and active masks ([n, 8]) of the liquid SDF's
    active voxels dilated ``layers`` times over the 26-neighbourhood
    (openvdb::tools::dilateActiveValues with NN_FACE_EDGE_VERTEX)."""
    from scipy.ndimage import binary_dilation

    org = np.asarray(liquid_phi.origins, dtype=np.int64)
    if org.shape[0] == 0:
        return np.zeros((0, 3), np.int32), np.zeros((0, 8), np.uint64)
    pad = 8 * (1 + (layers + 7) // 8)
    lo = org.min(axis=0) - pad
    hi = org.max(axis=0) + 8 + pad
    shape = tuple(int(v) for v in (hi - lo))
    act = np.zeros(shape, dtype=bool)
    xyz = offsets_xyz()
    on = unpack_masks(liquid_phi.masks)
    for i in range(org.shape[0]):
        g = org[i][None, :] + xyz - lo[None, :]
        a = on[i]
        act[g[a, 0], g[a, 1], g[a, 2]] = True
    if layers > 0:
        act = binary_dilation(act, structure=np.ones((3, 3, 3), dtype=bool), iterations=layers)
    nx, ny, nz = (s // 8 for s in shape)
    blk = act.reshape(nx, 8, ny, 8, nz, 8).transpose(0, 2, 4, 1, 3, 5).reshape(-1, 512)
    keep = blk.any(axis=1)
    ii, jj, kk = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    origins = (np.stack([ii.ravel(), jj.ravel(), kk.ravel()], axis=1) * 8 + lo[None, :])[keep]
    return origins.astype(np.int32), pack_masks(blk[keep])


def calculate_face_weights(solid_sdf: LeafGrid, origins: np.ndarray, masks: np.ndarray | None = None) -> np.ndarray:
    """Face weights [n, 512, 3] of the active voxels of the given topology
    ((1, 1, 1) elsewhere), from the solid SDF at the voxel corners."""
    keep: list = []
    org = np.ascontiguousarray(origins, dtype=np.int32).reshape(-1, 3)
    n = org.shape[0]
    out = np.empty((n, 512, 3), np.float32)
    m = None if masks is None else np.ascontiguousarray(masks, dtype=np.uint64).reshape(n, 8)
    g = _as_c(solid_sdf, keep)
    rc = _lib.lib().uaamg_face_weights(C.byref(g), n, org.ctypes.data if n else None,
                                       None if m is None or n == 0 else m.ctypes.data,
                                       out.ctypes.data if n else None)
    _lib.check(rc, "face_weights")
    return out


def face_weights_grid(solid_sdf: LeafGrid, liquid_phi: LeafGrid) -> LeafGrid:
    """The face-weight grid of the reference: the dilated liquid topology,
    background (1, 1, 1)."""
    origins, masks = face_weight_topology(liquid_phi)
    w = calculate_face_weights(solid_sdf, origins, masks)
    return LeafGrid(origins=origins, values=w, background=np.ones(3, np.float32), masks=masks)


def apply_pressure_gradient(lap: LaplacianWithLevel, liquid_phi: LeafGrid, face_weights: LeafGrid,
                            solid_velocity: LeafGrid, pressure: np.ndarray, dt: float, channel: int,
                            velocity: LeafGrid, friction: float = DEFAULT_FRICTION):
    """One velocity channel updated with the pressure solution of ``lap``
    (leaf-dense [leaf][512] on its level 0).  Returns (velocity [n, 512], the
    new active masks [n, 8], the update [n, 512], the reflected velocity
    [n, 512]); voxels without an update are inactive and keep their value."""
    keep: list = []
    n = velocity.leaf_count
    vel = np.empty((n, 512), np.float32)
    mask = np.empty((n, 8), np.uint64)
    upd = np.empty((n, 512), np.float32)
    refl = np.empty((n, 512), np.float32)
    p = np.ascontiguousarray(pressure, dtype=np.float32)
    gphi, gfw, gsv, gv = (_as_c(x, keep) for x in (liquid_phi, face_weights, solid_velocity, velocity))
    rc = _lib.lib().uaamg_poisson_apply_pressure_gradient(
        lap._h, C.byref(gphi), C.byref(gfw), C.byref(gsv), p.ctypes.data, float(dt), float(friction), int(channel),
        C.byref(gv), vel.ctypes.data, mask.ctypes.data, upd.ctypes.data, refl.ctypes.data)
    _lib.check(rc, "apply_pressure_gradient")
    return vel, mask, upd, refl
