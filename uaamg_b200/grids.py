"""Flattened sparse-voxel grids: the host-side data format of the drop-in boundary.

The reference keeps every field in an OpenVDB tree of 8^3 leaves
(``openvdb::FloatGrid`` / ``Vec3fGrid``; see SIMD_UAAMG/simd_vdb_poisson.h:54-65).
This package does not depend on OpenVDB, so a grid crosses the boundary as its
leaf list, which is exactly the payload of an OpenVDB ``LeafNode<T,3>``:

* ``origins``  int32 [n, 3]  leaf origins (multiples of 8, index space)
* ``masks``    uint64 [n, 8] value masks (bit ``off & 63`` of word ``off >> 6``)
* ``values``   float32 [n, 512] or [n, 512, 3], voxel offset ``64*x + 8*y + z``
* ``background`` value returned for coordinates outside every leaf

Active tiles are not representable; a caller voxelizes them first
(``tree().voxelizeActiveTiles()`` in OpenVDB terms).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

LEAF_DIM = 8
LEAF_SIZE = 512


@dataclass
class LeafGrid:
    origins: np.ndarray
    values: np.ndarray
    background: np.ndarray
    masks: np.ndarray | None = None
    components: int = field(init=False)

    def __post_init__(self) -> None:
        self.origins = np.ascontiguousarray(self.origins, dtype=np.int32).reshape(-1, 3)
        n = self.origins.shape[0]
        v = np.ascontiguousarray(self.values, dtype=np.float32)
        if v.ndim == 2:
            self.components = 1
            v = v.reshape(n, LEAF_SIZE)
        else:
            self.components = int(v.shape[-1])
            v = v.reshape(n, LEAF_SIZE, self.components)
        self.values = v
        bg = np.atleast_1d(np.asarray(self.background, dtype=np.float32)).reshape(-1)
        if bg.size == 1 and self.components == 3:
            bg = np.repeat(bg, 3)
        self.background = np.ascontiguousarray(bg, dtype=np.float32)
        if self.masks is None:
            self.masks = np.full((n, 8), np.uint64(0xFFFFFFFFFFFFFFFF), dtype=np.uint64)
        self.masks = np.ascontiguousarray(self.masks, dtype=np.uint64).reshape(n, 8)
        if np.any(self.origins % LEAF_DIM):
            raise ValueError("leaf origins must be multiples of 8")

    @property
    def leaf_count(self) -> int:
        return int(self.origins.shape[0])


def offsets_xyz() -> np.ndarray:
    """Local (x, y, z) of every voxel offset 0..511 (offset = 64x + 8y + z)."""
    off = np.arange(LEAF_SIZE)
    return np.stack([off >> 6, (off >> 3) & 7, off & 7], axis=1)


def dense_to_leaves(dense: np.ndarray, origin=(0, 0, 0), background=0.0,
                    active: np.ndarray | None = None) -> LeafGrid:
    """Cut a dense [X, Y, Z(, C)] array whose voxel (0,0,0) sits at index
    ``origin`` into 8^3 leaves. Sizes need not be multiples of 8; the padding
    takes the background value and is inactive."""
    dense = np.asarray(dense, dtype=np.float32)
    comps = 1 if dense.ndim == 3 else dense.shape[3]
    X, Y, Z = dense.shape[:3]
    o = np.asarray(origin, dtype=np.int64)
    if np.any(o % LEAF_DIM):
        raise ValueError("dense origin must be a multiple of 8")
    nx, ny, nz = (-(-X // 8), -(-Y // 8), -(-Z // 8))
    pad = [(0, nx * 8 - X), (0, ny * 8 - Y), (0, nz * 8 - Z)] + ([(0, 0)] if comps > 1 else [])
    bg = np.broadcast_to(np.asarray(background, dtype=np.float32), (comps,))
    if comps == 1:
        padded = np.pad(dense, pad, constant_values=float(bg[0]))
    else:
        padded = np.stack([np.pad(dense[..., c], pad[:3], constant_values=float(bg[c]))
                           for c in range(comps)], axis=-1)
    act = np.ones((X, Y, Z), dtype=bool) if active is None else np.asarray(active, dtype=bool)
    act = np.pad(act, pad[:3], constant_values=False)
    # [nx,8,ny,8,nz,8,(C)] -> [nx,ny,nz,8,8,8,(C)]
    if comps == 1:
        blk = padded.reshape(nx, 8, ny, 8, nz, 8).transpose(0, 2, 4, 1, 3, 5)
        values = blk.reshape(-1, LEAF_SIZE)
    else:
        blk = padded.reshape(nx, 8, ny, 8, nz, 8, comps).transpose(0, 2, 4, 1, 3, 5, 6)
        values = blk.reshape(-1, LEAF_SIZE, comps)
    ablk = act.reshape(nx, 8, ny, 8, nz, 8).transpose(0, 2, 4, 1, 3, 5).reshape(-1, LEAF_SIZE)
    masks = pack_masks(ablk)
    ii, jj, kk = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    origins = np.stack([ii.ravel(), jj.ravel(), kk.ravel()], axis=1) * 8 + o[None, :]
    return LeafGrid(origins=origins.astype(np.int32), values=values, background=bg.copy(), masks=masks)


def pack_masks(active: np.ndarray) -> np.ndarray:
    """bool [n, 512] -> uint64 [n, 8] OpenVDB value masks."""
    a = np.asarray(active, dtype=bool).reshape(-1, 8, 64)
    weights = (np.uint64(1) << np.arange(64, dtype=np.uint64))
    return (a.astype(np.uint64) * weights[None, None, :]).sum(axis=2, dtype=np.uint64)


def unpack_masks(masks: np.ndarray) -> np.ndarray:
    """uint64 [n, 8] -> bool [n, 512]."""
    m = np.asarray(masks, dtype=np.uint64).reshape(-1, 8, 1)
    bits = (m >> np.arange(64, dtype=np.uint64)[None, None, :]) & np.uint64(1)
    return bits.reshape(-1, LEAF_SIZE).astype(bool)


def leaves_to_dense(origins: np.ndarray, values: np.ndarray, lo, shape, fill=0.0) -> np.ndarray:
    """Scatter leaf-dense values [n, 512] into a dense array of ``shape`` whose
    voxel (0,0,0) is at index ``lo``; voxels outside ``shape`` are dropped."""
    out = np.full(shape, fill, dtype=np.float32)
    xyz = offsets_xyz()
    lo = np.asarray(lo)
    for i in range(origins.shape[0]):
        g = origins[i][None, :] + xyz - lo[None, :]
        ok = np.all((g >= 0) & (g < np.asarray(shape)[None, :]), axis=1)
        out[g[ok, 0], g[ok, 1], g[ok, 2]] = values[i][ok]
    return out


def vdb_leaf_order(origins: np.ndarray) -> np.ndarray:
    """Permutation that sorts leaf origins in OpenVDB tree order (5-4-3 tree:
    RootNode map keyed by the 4096^3 tile origin, compared x, y, z; then the
    32^3 and 16^3 internal-node child offsets)."""
    o = np.asarray(origins, dtype=np.int64)
    r = o & ~np.int64(4095)
    i2 = (((o[:, 0] & 4095) >> 7) << 10) | (((o[:, 1] & 4095) >> 7) << 5) | ((o[:, 2] & 4095) >> 7)
    i1 = (((o[:, 0] & 127) >> 3) << 8) | (((o[:, 1] & 127) >> 3) << 4) | ((o[:, 2] & 127) >> 3)
    return np.lexsort((i1, i2, r[:, 2], r[:, 1], r[:, 0]))
