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
``immerse_liquid_phi_in_solids`` adjusts the liquid SDF inside solids between
the two (FLIP_Solver_OpenVDB::immerse_liquid_phi_in_solids,
FLIP_vdb.cpp:2856-2942; ``uaamg_immerse_liquid_phi``).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .grids import LeafGrid
from .poisson import LaplacianWithLevel, _as_c
from .topology import dilate

# the FLIP solver's default boundary_friction_coefficient (FLIP_vdb.cpp:1886)
DEFAULT_FRICTION = 0.0


def face_weight_topology(liquid_phi: LeafGrid, layers: int = 2) -> tuple[np.ndarray, np.ndarray]:
    """Leaves (origins [n, 3]) and active masks ([n, 8]) of the liquid SDF's
    active voxels dilated ``layers`` times over the 26-neighbourhood
    (openvdb::tools::dilateActiveValues with NN_FACE_EDGE_VERTEX)."""
    return dilate(liquid_phi, layers, neighbours=26)


def calculate_face_weights(solid_sdf: LeafGrid, origins: np.ndarray, masks: np.ndarray | None = None) -> np.ndarray:
    """Face weights [n, 512, 3] of the active voxels of the given topology
    ((1, 1, 1) elsewhere), from the solid SDF at the voxel corners."""
    keep: list = []
    org = np.ascontiguousarray(origins, dtype=np.int32).reshape(-1, 3)
    n = org.shape[0]
    out = np.empty((n, 512, 3), np.float32)
    m = None if masks is None else np.ascontiguousarray(masks, dtype=np.uint64).reshape(n, 8)
    g = _as_c(solid_sdf, keep)
    _lib.torch_inputs_ready(None, solid_sdf)
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


def immerse_liquid_phi_values(liquid_phi: LeafGrid, solid_sdf: LeafGrid, dx: float) -> np.ndarray:
    """The value passes of immerse_liquid_phi_in_solids (FLIP_vdb.cpp:
    2856-2938) on the liquid SDF's own leaves, on the GPU: float32 [n, 512]."""
    keep: list = []
    n = liquid_phi.leaf_count
    out = np.empty((n, 512), np.float32)
    gs, gl = _as_c(solid_sdf, keep), _as_c(liquid_phi, keep)
    _lib.torch_inputs_ready(None, solid_sdf, liquid_phi)
    rc = _lib.lib().uaamg_immerse_liquid_phi(C.byref(gs), C.byref(gl), float(dx), out.ctypes.data if n else None)
    _lib.check(rc, "immerse_liquid_phi")
    return out


def immerse_liquid_phi_in_solids(liquid_phi: LeafGrid, solid_sdf: LeafGrid, dx: float) -> LeafGrid:
    """FLIP_Solver_OpenVDB::immerse_liquid_phi_in_solids (FLIP_vdb.cpp:
    2856-2942): the liquid SDF with its values adjusted inside solids (GPU)
    and its topology dilated once over the 26-neighbourhood (:2881) and once
    over the 6 face neighbours (:2941).  The liquid's leaves come first, then
    the leaves the dilations add (background values, as OpenVDB creates them);
    returns a new grid."""
    from .topology import LeafIndex
    vals = immerse_liquid_phi_values(liquid_phi, solid_sdf, dx)
    org, masks = dilate(dilate(liquid_phi, 1, neighbours=26), 1, neighbours=6)
    j = LeafIndex(liquid_phi.origins).find(org)
    n = liquid_phi.leaf_count
    out_masks = np.zeros((n, 8), np.uint64)
    out_masks[j[j >= 0]] = masks[j >= 0]
    new = j < 0
    bg = float(liquid_phi.background.reshape(-1)[0])
    return LeafGrid(origins=np.concatenate([liquid_phi.origins.astype(np.int32), org[new]], axis=0),
                    values=np.concatenate([vals, np.full((int(new.sum()), 512), bg, np.float32)], axis=0),
                    background=liquid_phi.background.copy(),
                    masks=np.concatenate([out_masks, masks[new]], axis=0))


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
    _lib.torch_inputs_ready(None, liquid_phi, face_weights, solid_velocity, velocity)
    rc = _lib.lib().uaamg_poisson_apply_pressure_gradient(
        lap._h, C.byref(gphi), C.byref(gfw), C.byref(gsv), p.ctypes.data, float(dt), float(friction), int(channel),
        C.byref(gv), vel.ctypes.data, mask.ctypes.data, upd.ctypes.data, refl.ctypes.data)
    _lib.check(rc, "apply_pressure_gradient")
    return vel, mask, upd, refl
